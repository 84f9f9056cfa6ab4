// One rank's z slab of a grid split across processes: the pass loop of the
// overlapped schedule, with the exchange left to the caller's transport
// (NCCL through torch.distributed, MPI, or host staging).  The reference
// runs one grid per process (src/diffusion3d/diffusion3d_cuda.cu:353-371)
// and has no multi-GPU path of its own.
//
// A pass of k <= halo steps (the owned planes are [lo, hi) of the local
// buffer, h = halo):
//   piece(down) = planes [lo-h, lo+2h), piece(up) = [hi-2h, hi+h);
//   k steps on each piece (its own small plan, clamped at the piece's
//   edges) leave its middle h planes exact: a clamp at a false edge makes
//   the plane beside it wrong, and each step spreads that by one plane;
//   those planes go to the neighbour while the owned planes run k steps;
//   the owned run is exact except h planes at each rank boundary, which
//   the pieces' planes overwrite; the received planes become the ghosts.
#include <cuda_runtime.h>

#include <new>

#include "d3d_b200.h"
#include "d3d_kernels.h"

struct d3d_slab_s {
  int nx = 0, ny = 0, halo = 0, dtype = D3D_F32, device = 0;
  int lo = 0, hi = 0, local_nz = 0;  // owned planes, local indices
  bool side[2] = {false, false};     // neighbour below / above
  size_t plane = 0;                  // bytes of one plane
  d3d_plan own = nullptr, piece = nullptr;
  void* pa[2] = {nullptr, nullptr};     // piece buffers (3 * halo planes)
  void* pb[2] = {nullptr, nullptr};
  void* ghost[2] = {nullptr, nullptr};  // landing buffers (halo planes)
};

namespace {

int slab_fail(int code, const char* msg) {
  return d3d::set_error(code, "%s", msg);
}

#define SLAB_TRY(call, what)                                           \
  do {                                                                 \
    cudaError_t e__ = (call);                                          \
    if (e__ != cudaSuccess) return d3d::set_cuda_error(e__, what);     \
  } while (0)

char* at(void* base, size_t bytes) { return static_cast<char*>(base) + bytes; }

}  // namespace

extern "C" {

int d3d_slab_create(int nx, int ny, int nz, int z0, int z1, int halo,
                    int dtype, d3d_slab* out, int* local_nz) {
  if (!out) return slab_fail(D3D_E_INVALID, "NULL output");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1 || z0 < 0 || z1 <= z0 || z1 > nz ||
      halo < 1 || (dtype != D3D_F32 && dtype != D3D_F64))
    return slab_fail(D3D_E_INVALID, "bad slab geometry");
  const bool down = z0 > 0, up = z1 < nz;
  if ((down && z0 < halo) || (up && nz - z1 < halo))
    return slab_fail(D3D_E_INVALID, "a neighbour holds fewer than halo planes");
  if ((down || up) && z1 - z0 < 2 * halo)
    return slab_fail(D3D_E_INVALID,
                     "a slab with a neighbour needs 2 x halo owned planes");
  d3d_slab s = new (std::nothrow) d3d_slab_s();
  if (!s) return slab_fail(D3D_E_OOM, "slab allocation");
  cudaGetDevice(&s->device);
  s->nx = nx;
  s->ny = ny;
  s->halo = halo;
  s->dtype = dtype;
  s->side[0] = down;
  s->side[1] = up;
  const int first = down ? z0 - halo : 0;
  s->lo = z0 - first;
  s->hi = z1 - first;
  s->local_nz = (up ? z1 + halo : nz) - first;
  s->plane = (size_t)nx * ny * (dtype == D3D_F64 ? 8 : 4);
  int rc = d3d_plan_create(nx, ny, z1 - z0, dtype, D3D_KERNEL_AUTO, 1,
                           &s->own);
  if (!rc && (down || up))
    rc = d3d_plan_create(nx, ny, 3 * halo, dtype, D3D_KERNEL_AUTO, 1,
                         &s->piece);
  for (int i = 0; i < 2 && !rc; ++i) {
    if (!s->side[i]) continue;
    rc = d3d_device_alloc(3 * halo * s->plane, &s->pa[i]);
    if (!rc) rc = d3d_device_alloc(3 * halo * s->plane, &s->pb[i]);
    if (!rc) rc = d3d_device_alloc(halo * s->plane, &s->ghost[i]);
  }
  if (rc) {
    const int code = rc;
    d3d_slab_destroy(s);  // keeps the failure's message
    return code;
  }
  if (local_nz) *local_nz = s->local_nz;
  *out = s;
  return D3D_OK;
}

int d3d_slab_run(d3d_slab s, void** f1, void** f2, const void* coeff,
                 int count, const d3d_slab_transport* t, void* stream) {
  if (!s || !f1 || !f2 || !*f1 || !*f2 || !coeff || count < 0)
    return slab_fail(D3D_E_INVALID, "NULL argument or negative count");
  if ((s->side[0] || s->side[1]) && (!t || !t->post || !t->wait))
    return slab_fail(D3D_E_INVALID, "a slab with neighbours needs a transport");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != s->device) return slab_fail(D3D_E_INVALID, "wrong device");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int h = s->halo;
  const size_t P = s->plane;
  for (int done = 0; done < count;) {
    const int k = count - done < h ? count - done : h;
    void* send[2] = {nullptr, nullptr};
    void* recv[2] = {nullptr, nullptr};
    for (int i = 0; i < 2; ++i) {
      if (!s->side[i]) continue;
      const int first = i == 0 ? s->lo - h : s->hi - 2 * h;
      SLAB_TRY(cudaMemcpyAsync(s->pa[i], at(*f1, first * P), 3 * h * P,
                               cudaMemcpyDeviceToDevice, st),
               "piece copy");
      void* a = s->pa[i];
      void* b = s->pb[i];
      int rc = d3d_run(s->piece, &a, &b, coeff, k, stream);
      if (rc) return rc;
      send[i] = at(a, h * P);  // the piece's middle planes: exact
      recv[i] = s->ghost[i];
    }
    if (s->side[0] || s->side[1]) {
      if (t->post(t->user, send, recv, h * P, stream) != 0)
        return slab_fail(D3D_E_TRANSPORT, "slab transport: post failed");
    }
    void* a = at(*f1, s->lo * P);
    void* b = at(*f2, s->lo * P);
    int rc = d3d_run(s->own, &a, &b, coeff, k, stream);
    if (rc) return rc;
    void* res = a == at(*f1, s->lo * P) ? *f1 : *f2;
    void* other = res == *f1 ? *f2 : *f1;
    if (s->side[0])
      SLAB_TRY(cudaMemcpyAsync(at(res, s->lo * P), send[0], h * P,
                               cudaMemcpyDeviceToDevice, st),
               "boundary planes");
    if (s->side[1])
      SLAB_TRY(cudaMemcpyAsync(at(res, (s->hi - h) * P), send[1], h * P,
                               cudaMemcpyDeviceToDevice, st),
               "boundary planes");
    if (s->side[0] || s->side[1]) {
      if (t->wait(t->user, stream) != 0)
        return slab_fail(D3D_E_TRANSPORT, "slab transport: wait failed");
    }
    if (s->side[0])
      SLAB_TRY(cudaMemcpyAsync(at(res, (s->lo - h) * P), s->ghost[0], h * P,
                               cudaMemcpyDeviceToDevice, st),
               "ghost planes");
    if (s->side[1])
      SLAB_TRY(cudaMemcpyAsync(at(res, s->hi * P), s->ghost[1], h * P,
                               cudaMemcpyDeviceToDevice, st),
               "ghost planes");
    *f1 = res;
    *f2 = other;
    done += k;
  }
  return D3D_OK;
}

int d3d_slab_destroy(d3d_slab s) {
  if (!s) return D3D_OK;
  if (s->own) d3d_plan_destroy(s->own);
  if (s->piece) d3d_plan_destroy(s->piece);
  for (int i = 0; i < 2; ++i) {
    if (s->pa[i]) d3d_device_free(s->pa[i]);
    if (s->pb[i]) d3d_device_free(s->pb[i]);
    if (s->ghost[i]) d3d_device_free(s->ghost[i]);
  }
  delete s;
  return D3D_OK;
}

}  // extern "C"
