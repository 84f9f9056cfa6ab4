// Binary checkpoints of fields: the replacement for the reference's text
// dump (Baseline::Dump, src/diffusion3d/baseline.cc:62-70: one "%.7E" line
// per value, about 15 bytes and one printf per point -- 2 GB for a 512^3
// field).  A checkpoint is a 64-byte header and the raw field:
//
//   offset  size  field
//        0     8  magic "D3DCKPT1"
//        8     4  header bytes (64), uint32
//       12     4  dtype (0 FP32, 1 FP64), uint32
//       16     4  ndim (2 or 3), uint32
//       20    12  nx, ny, nz, int32 (nz = 1 in 2D)
//       32     8  step, int64 (the caller's step counter)
//       40     8  checksum: the sum of the payload's 32-bit words modulo
//                 2^64, uint64 (integer, so any reduction order gives the
//                 same value on the device or on a host)
//       48     8  payload bytes, uint64
//       56     4  flags, uint32 (bit 0: diffusion::Diffusion surface)
//       60     4  reserved (0)
//       64     -  the field, x fastest, little-endian
//
// Device <-> file traffic goes through two pinned staging buffers so the
// PCIe copy of one chunk overlaps the file write (or read) of the other.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "d3d_b200.h"
#include "d3d_kernels.h"

namespace d3d {
namespace {

constexpr char kMagic[8] = {'D', '3', 'D', 'C', 'K', 'P', 'T', '1'};
constexpr size_t kChunk = 64u << 20;  // bytes per staging buffer

struct Header {
  char magic[8];
  uint32_t header_bytes, dtype, ndim;
  int32_t nx, ny, nz;
  int64_t step;
  uint64_t checksum;
  uint64_t payload;
  uint32_t flags, reserved;
};
static_assert(sizeof(Header) == 64, "checkpoint header is 64 bytes");

Header make_header(const PlanShape& ps, long long step) {
  Header h;
  memset(&h, 0, sizeof h);
  memcpy(h.magic, kMagic, sizeof kMagic);
  h.header_bytes = sizeof h;
  h.dtype = (uint32_t)ps.dtype;
  h.ndim = (uint32_t)ps.ndim;
  h.nx = ps.nx;
  h.ny = ps.ny;
  h.nz = ps.nz;
  h.step = step;
  h.payload = (uint64_t)ps.n * dtype_size(ps.dtype);
  h.flags = ps.flip_y ? 1u : 0u;
  return h;
}

// Pinned staging pair and its events, released on scope exit (cudaFreeHost
// waits for copies still reading or writing a buffer).
struct Staging {
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~Staging() {
    for (int i = 0; i < 2; ++i) {
      if (ev[i]) cudaEventDestroy(ev[i]);
      if (buf[i]) cudaFreeHost(buf[i]);
    }
  }
  cudaError_t init(size_t bytes) {
    for (int i = 0; i < 2; ++i) {
      cudaError_t e = cudaMallocHost(&buf[i], bytes);
      if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
};

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

// Sum of `nwords` 32-bit words into *out (modulo 2^64): a grid-stride pass,
// a warp shuffle reduction, one 64-bit atomic per warp.
__global__ void __launch_bounds__(256)
    word_sum_kernel(const uint32_t* __restrict__ p, size_t nwords,
                    unsigned long long* out) {
  unsigned long long acc = 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nwords;
       i += stride)
    acc += __ldg(p + i);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// The header checksum of a device field; `scratch` holds at least 8 bytes.
int device_checksum(const PlanShape& ps, double* scratch, const void* field,
                    cudaStream_t s, uint64_t* out) {
  auto* acc = reinterpret_cast<unsigned long long*>(scratch);
  const size_t nwords = ps.n * dtype_size(ps.dtype) / 4;
  cudaError_t e = cudaMemsetAsync(acc, 0, sizeof *acc, s);
  if (e == cudaSuccess) {
    word_sum_kernel<<<148 * 8, 256, 0, s>>>(
        static_cast<const uint32_t*>(field), nwords, acc);
    e = cudaGetLastError();
  }
  unsigned long long v = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&v, acc, sizeof v, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_cuda_error(e, "checkpoint checksum");
  note_launches(1);
  *out = v;
  return D3D_OK;
}

}  // namespace

int checkpoint_save_host(const PlanShape& ps, const void* host_field,
                         long long step, const char* path) {
  Header h = make_header(ps, step);
  const uint32_t* w = static_cast<const uint32_t*>(host_field);
  uint64_t sum = 0;
  for (size_t i = 0, nw = h.payload / 4; i < nw; ++i) sum += w[i];
  h.checksum = sum;
  File out;
  out.f = fopen(path, "wb");
  if (!out.f) return set_error(D3D_E_IO, "cannot create %s", path);
  if (fwrite(&h, sizeof h, 1, out.f) != 1 ||
      fwrite(host_field, 1, h.payload, out.f) != h.payload ||
      fflush(out.f) != 0)
    return set_error(D3D_E_IO, "write failed: %s", path);
  return D3D_OK;
}

int checkpoint_save(const PlanShape& ps, double* scratch, const void* field,
                    long long step, const char* path, cudaStream_t s) {
  Header h = make_header(ps, step);
  int rc = device_checksum(ps, scratch, field, s, &h.checksum);
  if (rc) return rc;
  File out;
  out.f = fopen(path, "wb");
  if (!out.f) return set_error(D3D_E_IO, "cannot create %s", path);
  if (fwrite(&h, sizeof h, 1, out.f) != 1)
    return set_error(D3D_E_IO, "write failed: %s", path);
  const size_t total = h.payload;
  const size_t chunk = std::min(kChunk, std::max<size_t>(total, 1));
  Staging st;
  cudaError_t e = st.init(chunk);
  if (e != cudaSuccess) return set_cuda_error(e, "pinned staging");
  const char* src = static_cast<const char*>(field);
  const size_t nchunks = (total + chunk - 1) / chunk;
  auto issue = [&](size_t i) {
    const size_t off = i * chunk, len = std::min(chunk, total - off);
    cudaError_t r = cudaMemcpyAsync(st.buf[i & 1], src + off, len,
                                    cudaMemcpyDeviceToHost, s);
    if (r == cudaSuccess) r = cudaEventRecord(st.ev[i & 1], s);
    return r;
  };
  if (nchunks > 0 && (e = issue(0)) != cudaSuccess)
    return set_cuda_error(e, "D2H copy");
  for (size_t i = 0; i < nchunks; ++i) {
    // Chunk i+1 copies while chunk i is written; its buffer held chunk
    // i-1, which is already in the file.
    if (i + 1 < nchunks && (e = issue(i + 1)) != cudaSuccess)
      return set_cuda_error(e, "D2H copy");
    if ((e = cudaEventSynchronize(st.ev[i & 1])) != cudaSuccess)
      return set_cuda_error(e, "D2H copy");
    const size_t len = std::min(chunk, total - i * chunk);
    if (fwrite(st.buf[i & 1], 1, len, out.f) != len)
      return set_error(D3D_E_IO, "write failed: %s", path);
  }
  if (fflush(out.f) != 0)
    return set_error(D3D_E_IO, "write failed: %s", path);
  return D3D_OK;
}

int checkpoint_load(const PlanShape& ps, double* scratch, const char* path,
                    void* field, long long* step, cudaStream_t s) {
  File in;
  in.f = fopen(path, "rb");
  if (!in.f) return set_error(D3D_E_IO, "cannot open %s", path);
  Header h;
  if (fread(&h, sizeof h, 1, in.f) != 1 ||
      memcmp(h.magic, kMagic, sizeof kMagic) != 0 ||
      h.header_bytes != sizeof h)
    return set_error(D3D_E_IO, "%s is not a d3d checkpoint", path);
  const uint64_t want = (uint64_t)ps.n * dtype_size(ps.dtype);
  if (h.dtype != (uint32_t)ps.dtype || h.ndim != (uint32_t)ps.ndim ||
      h.nx != ps.nx || h.ny != ps.ny || h.nz != ps.nz || h.payload != want)
    return set_error(D3D_E_INVALID,
                     "%s holds a %uD %dx%dx%d %s field; the plan is %dD "
                     "%dx%dx%d %s",
                     path, h.ndim, h.nx, h.ny, h.nz,
                     h.dtype ? "FP64" : "FP32", ps.ndim, ps.nx, ps.ny, ps.nz,
                     ps.dtype ? "FP64" : "FP32");
  // Bit 0 of flags: the field is in the diffusion::Diffusion surface's
  // order.  Same shape, other surface: refused, not silently reordered.
  if ((h.flags & 1u) != (ps.flip_y ? 1u : 0u))
    return set_error(D3D_E_INVALID,
                     "%s was saved from a %s plan; this plan is a %s plan",
                     path, (h.flags & 1u) ? "diffusion::Diffusion"
                                          : "diffusion3d",
                     ps.flip_y ? "diffusion::Diffusion" : "diffusion3d");
  const size_t total = h.payload;
  const size_t chunk = std::min(kChunk, std::max<size_t>(total, 1));
  Staging st;
  cudaError_t e = st.init(chunk);
  if (e != cudaSuccess) return set_cuda_error(e, "pinned staging");
  char* dst = static_cast<char*>(field);
  const size_t nchunks = (total + chunk - 1) / chunk;
  for (size_t i = 0; i < nchunks; ++i) {
    // The buffer's previous copy (chunk i-2) must finish before the file
    // overwrites it; chunk i-1 copies meanwhile.
    if (i >= 2 && (e = cudaEventSynchronize(st.ev[i & 1])) != cudaSuccess)
      return set_cuda_error(e, "H2D copy");
    const size_t off = i * chunk, len = std::min(chunk, total - off);
    if (fread(st.buf[i & 1], 1, len, in.f) != len)
      return set_error(D3D_E_IO, "%s is truncated", path);
    e = cudaMemcpyAsync(dst + off, st.buf[i & 1], len, cudaMemcpyHostToDevice,
                        s);
    if (e == cudaSuccess) e = cudaEventRecord(st.ev[i & 1], s);
    if (e != cudaSuccess) return set_cuda_error(e, "H2D copy");
  }
  uint64_t sum = 0;
  int rc = device_checksum(ps, scratch, field, s, &sum);
  if (rc) return rc;
  if (sum != h.checksum)
    return set_error(D3D_E_IO,
                     "%s failed its checksum (%llu stored, %llu read)", path,
                     (unsigned long long)h.checksum, (unsigned long long)sum);
  if (step) *step = h.step;
  return D3D_OK;
}

}  // namespace d3d
