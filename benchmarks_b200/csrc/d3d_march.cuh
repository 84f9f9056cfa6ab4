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

template <typename T, int BX, int BY>
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

  auto load = [&](int p) -> MarchPair<T> {
    const T* pl = src + (size_t)min(p, nz - 1) * plane;
    MarchPair<T> v;
    v.own = __ldg(pl + own_g);
    v.halo = has_halo ? __ldg(pl + halo_g) : T(0);
    return v;
  };

  MarchPair<T> q0 = load(z0), q1 = load(min(z0 + 1, z1)),
               q2 = load(min(z0 + 2, z1)), q3 = load(min(z0 + 3, z1));
  // b of the first plane: plane z0-1, or plane 0 itself at the bottom.
  T b = (z0 > 0) ? __ldg(src + (size_t)(z0 - 1) * plane + own_g) : q0.own;

  // One plane: publish `cur`, refill its slot with plane z+kQ, compute.
  auto plane_step = [&](int z, MarchPair<T>& cur, const MarchPair<T>& next) {
    T* st = stage[z & 1];
    st[own_s] = cur.own;
    if (has_halo) st[halo_s] = cur.halo;
    const T c = cur.own;
    const T t = next.own;  // plane min(z+1, nz-1)
    cur = load(min(z + kMarchQ, z1));  // past the chunk: plane z1 again
    __syncthreads();
    const T w = st[own_s - 1];
    const T e = st[own_s + 1];
    const T n = st[own_s - TL::W];
    const T s = st[own_s + TL::W];
    const T v = point(k, c, w, e, s, n, b, t);
    if (store_ok) dst[(size_t)z * plane + (size_t)yg * nx + xg] = v;
    b = c;
  };

  for (int z = z0; z < z1; z += kMarchQ) {
    plane_step(z, q0, q1);
    if (z + 1 >= z1) break;
    plane_step(z + 1, q1, q2);
    if (z + 2 >= z1) break;
    plane_step(z + 2, q2, q3);
    if (z + 3 >= z1) break;
    plane_step(z + 3, q3, q0);
  }
}

}  // namespace d3d
