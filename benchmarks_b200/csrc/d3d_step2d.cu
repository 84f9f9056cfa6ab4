// The 2D 5-point step of the reference's second plugin surface,
// diffusion::Diffusion with nd = 2 (src/diffusion/diffusion_openmp.cc:59-82,
// baseline.h:46-80):
//
//   f2[c] = cc*c + cw*w + ce*e + cs*s + cn*n,   s = y-1, n = y+1,
//
// clamped neighbours, summed left to right with every product and sum
// rounded on its own, so the result is bit-identical to the reference's
// CPU build.
//
// Design (HBM-bound: 8 B per FP32 update, 16 B per FP64 update).  Each warp
// owns a segment of 32*V consecutive columns (V values per lane) and marches
// down a chunk of rows.  A ring of R rows lives in registers: rows y-1, y,
// y+1 feed the update of row y and the next R-3 rows are already in flight,
// so every value crosses HBM once (plus the two chunk-boundary rows, L2
// hits while the neighbouring chunk runs) and no shared memory or barrier
// is needed.  x neighbours inside the segment come from the lane's own
// registers and warp shuffles; lanes 0 and 31 also load the one column just
// outside the segment.  Every replicated-boundary rule is an address or a
// loop-invariant select: the first loaded row is clamped to row 0, the row
// after the last to row ny-1, every column to [0, nx-1], and the lane that
// owns x = nx-1 takes its own value as e.
//
// Memory-level parallelism is what bounds the kernel: a lane's in-flight
// rows cost registers, so the variants trade ring depth against occupancy
// (kStep2dVariants), and short row chunks (6 rows by default) let each warp
// issue almost all of its loads at once.  Rows whose start is 16-byte
// aligned (nx a multiple of 16 / sizeof(T), aligned buffers) use one vector
// access per lane and row; other shapes keep the same 4 (FP32) or 2 (FP64)
// values per lane with one scalar access per value.
#include <algorithm>

#include "d3d_common.cuh"
#include "d3d_kernels.h"

namespace d3d {
namespace {

constexpr int kStep2dThreads = 256;

// One point, diffusion_openmp.cc:73-74.
template <typename T>
__device__ __forceinline__ T point5(const Coef<T>& k, T c, T w, T e, T s,
                                    T n) {
  T v = mul_rn(k.cc, c);
  v = add_rn(v, mul_rn(k.cw, w));
  v = add_rn(v, mul_rn(k.ce, e));
  v = add_rn(v, mul_rn(k.cs, s));
  v = add_rn(v, mul_rn(k.cn, n));
  return v;
}

// `point5` on two adjacent x positions (packed f32x2, exact products as in
// point2).
__device__ __forceinline__ uint64_t point5x2(const Coef2& k, uint64_t c,
                                             uint64_t w, uint64_t e,
                                             uint64_t s, uint64_t n) {
  uint64_t v = mul2_rn(k.cc, c, k.nz);
  v = add2_rn(v, mul2_rn(k.cw, w, k.nz));
  v = add2_rn(v, mul2_rn(k.ce, e, k.nz));
  v = add2_rn(v, mul2_rn(k.cs, s, k.nz));
  v = add2_rn(v, mul2_rn(k.cn, n, k.nz));
  return v;
}

// Packed coefficients for the FP32 pair path (unused for FP64).
template <typename T>
__device__ __forceinline__ Coef2 coef2_if(const Coef<T>& k) {
  if constexpr (sizeof(T) == 4) {
    return coef2(k);
  } else {
    return Coef2{};
  }
}

// V consecutive values of one row.
template <typename T, int V>
struct alignas(sizeof(T) * V) Vec {
  T e[V];
};

// One 16-byte load through the read-only path.
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> ld_vec(const T* p) {
  static_assert(sizeof(T) * V == 16, "16-byte vectors");
  Vec<T, V> r;
  if constexpr (sizeof(T) == 4) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    r.e[0] = v.x; r.e[1] = v.y; r.e[2] = v.z; r.e[3] = v.w;
  } else {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    r.e[0] = v.x; r.e[1] = v.y;
  }
  return r;
}

template <typename T, int V>
__device__ __forceinline__ void st_vec(T* p, const Vec<T, V>& r) {
  *reinterpret_cast<Vec<T, V>*>(p) = r;
}

// The V outputs of one lane from its centre, s (y-1) and n (y+1) values and
// the two x neighbours just outside its V columns.
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> seg5(const Coef<T>& k, const Coef2& k2,
                                          const Vec<T, V>& c,
                                          const Vec<T, V>& s,
                                          const Vec<T, V>& n, T wl, T er) {
  Vec<T, V> o;
  if constexpr (sizeof(T) == 4 && V == 4) {
    const uint64_t mid = pack2(c.e[1], c.e[2]);
    const uint64_t lo = point5x2(k2, pack2(c.e[0], c.e[1]),
                                 pack2(wl, c.e[0]), mid,
                                 pack2(s.e[0], s.e[1]), pack2(n.e[0], n.e[1]));
    const uint64_t hi = point5x2(k2, pack2(c.e[2], c.e[3]), mid,
                                 pack2(c.e[3], er), pack2(s.e[2], s.e[3]),
                                 pack2(n.e[2], n.e[3]));
    unpack2(lo, o.e[0], o.e[1]);
    unpack2(hi, o.e[2], o.e[3]);
  } else if constexpr (sizeof(T) == 4 && V == 2) {
    const uint64_t r = point5x2(k2, pack2(c.e[0], c.e[1]), pack2(wl, c.e[0]),
                                pack2(c.e[1], er), pack2(s.e[0], s.e[1]),
                                pack2(n.e[0], n.e[1]));
    unpack2(r, o.e[0], o.e[1]);
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) {
      const T w = i > 0 ? c.e[i - 1] : wl;
      const T e = i < V - 1 ? c.e[i + 1] : er;
      o.e[i] = point5(k, c.e[i], w, e, s.e[i], n.e[i]);
    }
  }
  return o;
}

// One warp = one (segment, row chunk) task; tasks are numbered segment
// fastest, so neighbouring warps read neighbouring columns of the same rows.
// R: rows in each lane's register ring (R-2 loads in flight).  VEC: one
// vector access per lane and row (needs nx % V == 0 and V*sizeof(T)-aligned
// buffers); otherwise V scalar accesses.
template <typename T, int V, int R, bool VEC>
__global__ void __launch_bounds__(kStep2dThreads)
    step2d_kernel(const T* __restrict__ src, T* __restrict__ dst, int nx,
                  int ny, Coef<T> k, int ychunk, int nseg) {
  constexpr int SW = 32 * V;
  static_assert(R >= 4, "rows y-1, y, y+1 and one in flight");
  const int lane = threadIdx.x & 31;
  const long long task =
      (long long)blockIdx.x * (kStep2dThreads / 32) + (threadIdx.x >> 5);
  const int seg = (int)(task % nseg);
  const long long chunk = task / nseg;
  if (chunk * ychunk >= ny) return;  // warp-uniform
  const int y0 = (int)(chunk * ychunk);
  const int y1 = min(ny, y0 + ychunk);

  const int xs = seg * SW;
  const int col = xs + V * lane;
  const bool valid = col < nx;  // the lane owns at least one column
  // Vector lanes past the edge read the last whole vector (never stored);
  // scalar lanes clamp each column, so a partial lane's columns past nx-1
  // hold f(nx-1), which is exactly the e neighbour x = nx-1 needs.
  const int lcol = VEC ? (valid ? col : nx - V) : col;
  const bool x_hi = valid && (col + V >= nx);  // owns x = nx-1
  const bool has_edge = (lane == 0) || (lane == 31);
  const int ecol = (lane == 0) ? max(xs - 1, 0) : min(xs + SW, nx - 1);
  int cl[V];  // scalar path: clamped column offsets from lcol
#pragma unroll
  for (int i = 0; i < V; ++i) cl[i] = min(col + i, nx - 1) - lcol;
  const Coef2 k2 = coef2_if<T>(k);

  Vec<T, V> ring[R];
  T edge[R];
  // Row r into a ring slot; r = y0-1 is clamped to row 0 and r = ny (the n
  // row of the last grid row) to row ny-1.  Rows past y1 are never needed.
  auto load = [&](int r, Vec<T, V>& v, T& ed) {
    if (r <= y1) {
      const T* row = src + (size_t)min(max(r, 0), ny - 1) * nx;
      if constexpr (VEC) {
        v = ld_vec<T, V>(row + lcol);
      } else {
#pragma unroll
        for (int i = 0; i < V; ++i) v.e[i] = __ldg(row + lcol + cl[i]);
      }
      if (has_edge) ed = __ldg(row + ecol);
    }
  };

  // Slot of row r: (r - y0 + 1) % R.  Rows y0-1 .. y0+R-3 first.
#pragma unroll
  for (int i = 0; i < R - 1; ++i) load(y0 - 1 + i, ring[i], edge[i]);

  T* out = dst + (size_t)y0 * nx + col;
  for (int yb = y0; yb < y1; yb += R) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int y = yb + i;
      if (y < y1) {
        // Row y+R-2 reuses the slot of row y-2.
        load(y + R - 2, ring[(i + R - 1) % R], edge[(i + R - 1) % R]);
        const Vec<T, V>& s = ring[i % R];
        const Vec<T, V>& c = ring[(i + 1) % R];
        const Vec<T, V>& n = ring[(i + 2) % R];
        T wl = __shfl_up_sync(0xffffffffu, c.e[V - 1], 1);
        T er = __shfl_down_sync(0xffffffffu, c.e[0], 1);
        if (lane == 0) wl = edge[(i + 1) % R];
        if (lane == 31) er = edge[(i + 1) % R];
        if (x_hi) er = c.e[V - 1];
        const Vec<T, V> o = seg5<T, V>(k, k2, c, s, n, wl, er);
        if constexpr (VEC) {
          if (valid) st_vec<T, V>(out, o);
        } else {
#pragma unroll
          for (int e = 0; e < V; ++e)
            if (col + e < nx) out[e] = o.e[e];
        }
        out += nx;
      }
    }
  }
}

int g_sms = 0;

int sm_count() {
  if (!g_sms) {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    g_sms = n > 0 ? n : 148;
  }
  return g_sms;
}

template <typename T, int V, int R, bool VEC>
cudaError_t launch2d_t(const void* f1, void* f2, int nx, int ny,
                       const void* coef, int ychunk_override,
                       cudaStream_t stream, LaunchInfo* info) {
  auto kern = step2d_kernel<T, V, R, VEC>;
  static int ctas_per_sm = 0;  // per instantiation; same on every device
  if (!ctas_per_sm) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &ctas_per_sm, kern, kStep2dThreads, 0);
    if (e != cudaSuccess) return e;
    if (ctas_per_sm < 1) ctas_per_sm = 1;
  }
  const int nseg = (nx + 32 * V - 1) / (32 * V);
  int ychunk = ychunk_override;
  if (ychunk <= 0) {
    // 6-row tasks (measured best on B200 from 4096^2 to 16384^2, FP32 and
    // FP64: a warp issues nearly all of a task's loads at once), shorter on
    // grids too small to give each resident warp one.
    const long long warps =
        (long long)sm_count() * ctas_per_sm * (kStep2dThreads / 32);
    const long long rows = (long long)ny * nseg;
    ychunk = (int)std::max<long long>(
        2, std::min<long long>(6, (rows + warps - 1) / warps));
  }
  ychunk = std::min(ychunk, ny);
  const long long nchunks = (ny + ychunk - 1) / ychunk;
  const long long tasks = nchunks * nseg;
  const long long blocks = (tasks + kStep2dThreads / 32 - 1) /
                           (kStep2dThreads / 32);
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  if (info) {
    info->grid_x = (int)blocks;
    info->grid_y = 1;
    info->grid_z = 1;
    info->block = kStep2dThreads;
    info->smem_bytes = 0;
    info->zchunk = ychunk;
    info->ctas_per_sm = ctas_per_sm;
  }
  kern<<<(unsigned)blocks, kStep2dThreads, 0, stream>>>(
      static_cast<const T*>(f1), static_cast<T*>(f2), nx, ny,
      coef_from<T>(coef), ychunk, nseg);
  return cudaGetLastError();
}

bool aligned(const void* p, size_t a) {
  return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0;
}

}  // namespace

int step2d_vector_width(const void* f1, const void* f2, int nx, int dtype) {
  const size_t es = dtype_size(dtype);
  for (int v = (int)(16 / es); v > 1; v /= 2)
    if (nx % v == 0 && aligned(f1, v * es) && aligned(f2, v * es)) return v;
  return 1;
}

namespace {

template <typename T, bool VEC>
cudaError_t launch2d_variant(int variant, const void* f1, void* f2, int nx,
                             int ny, const void* coef, int yc,
                             cudaStream_t s, LaunchInfo* info) {
  constexpr int V = 16 / sizeof(T);
  switch (variant) {
    case 0: return launch2d_t<T, V, 8, VEC>(f1, f2, nx, ny, coef, yc, s, info);
    case 1: return launch2d_t<T, V, 6, VEC>(f1, f2, nx, ny, coef, yc, s, info);
    case 2: return launch2d_t<T, V, 10, VEC>(f1, f2, nx, ny, coef, yc, s, info);
    case 3: return launch2d_t<T, V, 12, VEC>(f1, f2, nx, ny, coef, yc, s, info);
    case 4: return launch2d_t<T, V, 4, VEC>(f1, f2, nx, ny, coef, yc, s, info);
    case 5: return launch2d_t<T, V, 16, VEC>(f1, f2, nx, ny, coef, yc, s, info);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

const Step2dVariant kStep2dVariants[kNumStep2dVariants] = {
    {8}, {6}, {10}, {12}, {4}, {16}};

int default_step2d_variant() { return 0; }

cudaError_t launch_step2d(const void* f1, void* f2, int nx, int ny,
                          const void* coef, int dtype, int variant,
                          int ychunk_override, cudaStream_t stream,
                          LaunchInfo* info) {
  const bool vec = step2d_vector_width(f1, f2, nx, dtype) * dtype_size(dtype)
                   == 16;
  const int yc = ychunk_override;
  if (dtype == kF64)
    return vec ? launch2d_variant<double, true>(variant, f1, f2, nx, ny, coef,
                                                yc, stream, info)
               : launch2d_variant<double, false>(variant, f1, f2, nx, ny,
                                                 coef, yc, stream, info);
  return vec ? launch2d_variant<float, true>(variant, f1, f2, nx, ny, coef, yc,
                                             stream, info)
             : launch2d_variant<float, false>(variant, f1, f2, nx, ny, coef,
                                              yc, stream, info);
}

}  // namespace d3d
