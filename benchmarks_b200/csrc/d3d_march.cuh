// The any-shape tile march shared by the generic single-grid kernel and the
// multi-grid batch/server kernel.
//
// A 256-thread CTA owns a BX x BY xy tile and marches planes [z0, z1) of
// one grid.  Each thread owns its interior cell and at most one cell of the
// tile's one-cell halo ring, and keeps the next kQ planes of both in a
// register queue (kQ loads in flight per cell).  Per plane it publishes the
// current values into one of two shared halo planes (a single
// __syncthreads per plane), takes n/s/w/e from shared memory and b/c/t
// from its queue.  Every load address is clamped into the grid -- the
// reference's replicated-neighbour rule -- so no value is ever selected and
// any nx, ny, nz and alignment work.  Each point is d3d::point.
#pragma once

#include "d3d_common.cuh"

namespace d3d {

template <int BX, int BY>
struct MarchTile {
  static constexpr int THREADS = BX * BY;
  static constexpr int W = BX + 2;
  static constexpr int H = BY + 2;
  static constexpr int E = W * H;
  static constexpr int HALO = E - BX * BY;
  static_assert(THREADS == 256, "tile marches run 256 threads");
  static_assert(HALO <= THREADS, "one halo cell per thread at most");
};

constexpr int kMarchQ = 4;  // planes in each thread's register queue

template <typename T>
struct MarchPair {
  T own, halo;
};

// FLIP: the y-1 neighbour is summed before y+1 (diffusion::Diffusion)
// instead of after it (diffusion3d).
template <typename T, int BX, int BY, bool FLIP = false>
__device__ __forceinline__ void march_tile(const T* __restrict__ src,
                                           T* __restrict__ dst, int nx,
                                           int ny, int nz, int x0, int y0,
                                           int z0, int z1, const Coef<T>& k,
                                           T (*stage)[MarchTile<BX, BY>::E]) {
  using TL = MarchTile<BX, BY>;
  const int tid = threadIdx.x;
  const int tx = tid % BX, ty = tid / BX;
  const int xg = x0 + tx, yg = y0 + ty;
  // Interior cell: stage index and clamped in-plane offset.
  const int own_s = (ty + 1) * TL::W + (tx + 1);
  const int own_g = min(yg, ny - 1) * nx + min(xg, nx - 1);
  // Halo cell h = tid (if any): the border of the W x H box.
  const bool has_halo = tid < TL::HALO;
  int lx, ly;
  if (tid < TL::W) {
    lx = tid;
    ly = 0;
  } else if (tid < 2 * TL::W) {
    lx = tid - TL::W;
    ly = TL::H - 1;
  } else if (tid < 2 * TL::W + TL::H - 2) {
    lx = 0;
    ly = 1 + tid - 2 * TL::W;
  } else {
    lx = TL::W - 1;
    ly = 1 + tid - 2 * TL::W - (TL::H - 2);
  }
  const int halo_s = ly * TL::W + lx;
  const int hx = min(max(x0 - 1 + lx, 0), nx - 1);
  const int hy = min(max(y0 - 1 + ly, 0), ny - 1);
  const int halo_g = hy * nx + hx;
  const bool store_ok = xg < nx && yg < ny;
  const size_t plane = (size_t)nx * ny;
  // n is y-1 and s is y+1 (diffusion3d); FLIP swaps them.
  constexpr int nrow = FLIP ? -TL::W : TL::W;

  // Load pointers step one plane per call and stop at the last plane the
  // chunk needs (plane z1 is the t of plane z1-1); later calls re-read it.
  const int plim = min(z1, nz - 1);
  int pn = z0;  // plane the next load reads
  const T* po = src + (size_t)z0 * plane + own_g;
  const T* ph = src + (size_t)z0 * plane + halo_g;
  auto load_next = [&]() -> MarchPair<T> {
    MarchPair<T> v;
    v.own = __ldg(po);
    v.halo = has_halo ? __ldg(ph) : T(0);
    if (pn < plim) {
      po += plane;
      ph += plane;
    }
    ++pn;
    return v;
  };

  MarchPair<T> q[kMarchQ];
#pragma unroll
  for (int i = 0; i < kMarchQ; ++i) q[i] = load_next();
  // b of the first plane: plane z0-1, or plane 0 itself at the bottom.
  T b = (z0 > 0) ? __ldg(src + (size_t)(z0 - 1) * plane + own_g) : q[0].own;
  T* out = dst + (size_t)z0 * plane + (size_t)min(yg, ny - 1) * nx +
           min(xg, nx - 1);

  // One plane: publish `cur` into stage `st`, refill the slot with the next
  // plane in line, compute, store.
  auto plane_step = [&](T* st, MarchPair<T>& cur, const MarchPair<T>& next) {
    st[own_s] = cur.own;
    if (has_halo) st[halo_s] = cur.halo;
    const T c = cur.own;
    const T t = next.own;  // plane min(z+1, nz-1)
    cur = load_next();
    __syncthreads();
    const T w = st[own_s - 1];
    const T e = st[own_s + 1];
    const T n = st[own_s - nrow];
    const T s = st[own_s + nrow];
    const T v = point(k, c, w, e, s, n, b, t);
    if (store_ok) *out = v;
    out += plane;
    b = c;
  };

  // Unrolled kMarchQ (even) ways: queue slots and stage parity are
  // compile-time constants, so the queue stays in registers.
  for (int z = z0; z < z1; z += kMarchQ) {
    bool more = true;
#pragma unroll
    for (int i = 0; i < kMarchQ; ++i) {
      if (more) {
        plane_step(stage[i & 1], q[i], q[(i + 1) % kMarchQ]);
        more = (z + i + 1 < z1);
      }
    }
    if (!more) break;
  }
}


// ---------------------------------------------------------------------------
// FP32, two cells per thread: the same march with each thread owning an
// x-pair, so the stencil runs on packed f32x2 pairs (point2, exact) and the
// n/s neighbours are 8-byte shared loads.  The stage carries a two-column
// left pad (column c <-> x = x0 - 2 + c) so every thread's pair is 8-byte
// aligned; only columns 1 .. BX+2 are ever read.
// ---------------------------------------------------------------------------
template <int BX, int BY>
struct MarchTile2 {
  static constexpr int TX = BX / 2;  // threads per row
  static constexpr int THREADS = TX * BY;
  static constexpr int W = BX + 4;
  static constexpr int H = BY + 2;
  static constexpr int E = W * H;
  static constexpr int HALO = 2 * (BX + 2) + 2 * BY;
  static_assert(BX % 2 == 0, "pairs");
  static_assert(THREADS == 256, "tile marches run 256 threads");
  static_assert(HALO <= THREADS, "one halo cell per thread at most");
};

struct MarchQuad {
  float o0, o1, halo;
};

template <int BX, int BY, bool FLIP = false>
__device__ __forceinline__ void march_tile2(
    const float* __restrict__ src, float* __restrict__ dst, int nx, int ny,
    int nz, int x0, int y0, int z0, int z1, const Coef<float>& k,
    float (*stage)[MarchTile2<BX, BY>::E]) {
  using TL = MarchTile2<BX, BY>;
  const int tid = threadIdx.x;
  const int tx = tid % TL::TX, ty = tid / TL::TX;
  const int xg = x0 + 2 * tx, yg = y0 + ty;
  const int own_s = (ty + 1) * TL::W + 2 + 2 * tx;  // even: 8-byte aligned
  const int yc = min(yg, ny - 1);
  const int own_g0 = yc * nx + min(xg, nx - 1);
  const int own_g1 = yc * nx + min(xg + 1, nx - 1);
  const bool has_halo = tid < TL::HALO;
  int lx, ly;
  if (tid < BX + 2) {
    lx = 1 + tid;
    ly = 0;
  } else if (tid < 2 * (BX + 2)) {
    lx = 1 + tid - (BX + 2);
    ly = TL::H - 1;
  } else if (tid < 2 * (BX + 2) + BY) {
    lx = 1;
    ly = 1 + tid - 2 * (BX + 2);
  } else {
    lx = BX + 2;
    ly = 1 + tid - 2 * (BX + 2) - BY;
  }
  const int halo_s = ly * TL::W + lx;
  const int halo_g = min(max(y0 - 1 + ly, 0), ny - 1) * nx +
                     min(max(x0 - 2 + lx, 0), nx - 1);
  const bool store0 = xg < nx && yg < ny;
  const bool store1 = xg + 1 < nx && yg < ny;
  const size_t plane = (size_t)nx * ny;
  const Coef2 kk = coef2(k);
  constexpr int nrow = FLIP ? -TL::W : TL::W;  // as in march_tile

  const int plim = min(z1, nz - 1);
  int pn = z0;
  const float* pbase = src + (size_t)z0 * plane;
  auto load_next = [&]() -> MarchQuad {
    MarchQuad v;
    v.o0 = __ldg(pbase + own_g0);
    v.o1 = __ldg(pbase + own_g1);
    v.halo = has_halo ? __ldg(pbase + halo_g) : 0.0f;
    if (pn < plim) pbase += plane;
    ++pn;
    return v;
  };

  MarchQuad q[kMarchQ];
#pragma unroll
  for (int i = 0; i < kMarchQ; ++i) q[i] = load_next();
  float b0, b1;
  if (z0 > 0) {
    b0 = __ldg(src + (size_t)(z0 - 1) * plane + own_g0);
    b1 = __ldg(src + (size_t)(z0 - 1) * plane + own_g1);
  } else {
    b0 = q[0].o0;
    b1 = q[0].o1;
  }
  float* out = dst + (size_t)z0 * plane + own_g0;

  auto plane_step = [&](float* st, MarchQuad& cur, const MarchQuad& next) {
    *reinterpret_cast<float2*>(st + own_s) = make_float2(cur.o0, cur.o1);
    if (has_halo) st[halo_s] = cur.halo;
    const float c0 = cur.o0, c1 = cur.o1;
    const uint64_t t01 = pack2(next.o0, next.o1);
    const uint64_t b01 = pack2(b0, b1);
    cur = load_next();
    __syncthreads();
    const float w0 = st[own_s - 1];
    const float e1 = st[own_s + 2];
    const float2 n = *reinterpret_cast<const float2*>(st + own_s - nrow);
    const float2 sv = *reinterpret_cast<const float2*>(st + own_s + nrow);
    const uint64_t r = point2(kk, pack2(c0, c1), pack2(w0, c0),
                              pack2(c1, e1), pack2(sv.x, sv.y),
                              pack2(n.x, n.y), b01, t01);
    float o0, o1;
    unpack2(r, o0, o1);
    if (store0) out[0] = o0;
    if (store1) out[1] = o1;
    out += plane;
    b0 = c0;
    b1 = c1;
  };

  for (int z = z0; z < z1; z += kMarchQ) {
    bool more = true;
#pragma unroll
    for (int i = 0; i < kMarchQ; ++i) {
      if (more) {
        plane_step(stage[i & 1], q[i], q[(i + 1) % kMarchQ]);
        more = (z + i + 1 < z1);
      }
    }
    if (!more) break;
  }
}

}  // namespace d3d
