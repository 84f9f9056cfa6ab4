// Two fused time steps per HBM pass, FP32, with the single-step kernel's
// warp shape (d3d_step.cu): the K = 2 temporal-blocking kernel.
//
// The generic-K kernel (d3d_tb.cu) spreads each level's cells over the
// CTA's threads in any order, so x neighbours come from scalar shared loads
// and every cell carries a level mask; it runs about 31 instructions per
// update and only matches the single-step kernel.  Here every warp owns
// whole rows:
//
//   tile     128 output columns (a warp: 32 lanes x 4 floats) x 14 output
//            rows x a z-chunk; level 1 covers 16 rows (one halo row above
//            and below) and, through two scalar halo columns, x0-1 and
//            x0+128; level 0 is TMA-loaded as 136 x 18 boxes (x0-4 ..
//            x0+131, y0-2 .. y0+15) into a 4-plane shared ring (mbarriers);
//   warps    warp w owns level-1 rows 2w and 2w+1 of the 16 and the same
//            rows at level 2 (rows 1..14 only): warps 0 and 7 have one
//            level-2 row, and they compute the left and right level-1 halo
//            columns instead;
//   level 1  b, c of each owned row are in registers (three register sets
//            whose roles rotate with the plane, so nothing is copied), t is
//            one 16-byte shared load, n and s two more, w and e come from
//            warp shuffles (lanes 0 and 31 read one word beyond); the
//            result stays in registers and is also published to a 2-slot
//            shared ring for the rows above and below;
//   level 2  b, c, t are level 1's registers, n and s two shared loads from
//            the ring, w and e shuffles (lanes 0 and 31 read the halo
//            column); 128-bit stores to HBM.
//
// When level-0 plane q has landed, level 1 computes plane q-1 and level 2
// plane q-2, which reads only ring planes written in the previous
// iteration: one __syncthreads per plane.  Replicated boundaries are
// loop-invariant addresses and selects, as in the single-step kernel;
// z-clamps are register copies.  Every point is d3d::point (packed f32x2,
// exact products), so two fused steps are bit-identical to two single
// steps.  FLIP swaps the y-1 / y+1 offsets (the diffusion::Diffusion order).
#include <algorithm>
#include <type_traits>

#include "d3d_common.cuh"
#include "d3d_kernels.h"

namespace d3d {
namespace {

struct Tb2w {
  static constexpr int WARPS = 8;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int V = 4;                   // floats per lane
  static constexpr int BX = 128;                // output columns
  static constexpr int HX = 4;                  // box starts at x0 - HX
  static constexpr int P = BX + 2 * HX;         // 136: box / ring row pitch
  static constexpr int R1 = 16;                 // level-1 rows
  static constexpr int BY = R1 - 2;             // 14 output rows
  static constexpr int R0 = R1 + 2;             // 18 level-0 rows
  static constexpr int RPW = R1 / WARPS;        // 2 rows per warp
  // Level-0 ring planes: q-2, q-1, q in use and one load in flight, which
  // is a whole iteration (about 3.5 us at 512^3) ahead of its use; a power
  // of two keeps the stage and parity arithmetic to a mask and a shift.
  static constexpr int S0 = 4;
  static constexpr int STAGE_RAW = P * R0 * 4;  // 9792 bytes
  static constexpr int STAGE = (STAGE_RAW + 127) / 128 * 128;
  static constexpr int STAGE_ELEMS = STAGE / 4;
  static constexpr int RING = P * R1;           // floats per ring plane
  static constexpr int SMEM = S0 * STAGE + 2 * RING * 4 + S0 * 8 + 256;
  static_assert(R1 % WARPS == 0, "whole rows per warp");
};

// MINB = 2: two CTAs per SM at <= 128 registers without spilling (a
// three-CTA build spills and measured 20% slower on B200).
template <bool FLIP, int MINB>
__global__ void __launch_bounds__(Tb2w::THREADS, MINB)
    steps_tb2w_kernel(const __grid_constant__ CUtensorMap src,
                      float* __restrict__ dst, int nx, int ny, int nz,
                      Coef<float> k, int zchunk, unsigned* __restrict__ dev_err) {
  using C = Tb2w;
  constexpr int V = C::V, P = C::P, S0 = C::S0, RPW = C::RPW;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  float* stages = reinterpret_cast<float*>(base);
  float* ring = reinterpret_cast<float*>(base + S0 * C::STAGE);
  uint64_t* bars =
      reinterpret_cast<uint64_t*>(base + S0 * C::STAGE + 2 * C::RING * 4);

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int x0 = blockIdx.x * C::BX;
  const int y0 = blockIdx.y * C::BY;
  const int z0 = blockIdx.z * zchunk;
  const int z1 = min(nz, z0 + zchunk);
  if (z0 >= z1) return;
  // Level-1 planes [lo1, hi1], level-0 planes [lo0, hi0].
  const int lo1 = max(z0 - 1, 0), hi1 = min(z1, nz - 1);
  const int lo0 = max(z0 - 2, 0), hi0 = min(z1 + 1, nz - 1);

  // p >= lo0 always: unsigned arithmetic makes these a mask and a shift.
  auto stage_of = [&](int p) { return (int)((unsigned)(p - lo0) % S0); };
  auto parity_of = [&](int p) { return ((unsigned)(p - lo0) / S0) & 1u; };
  auto stage_ptr = [&](int p) {
    return stages + stage_of(p) * C::STAGE_ELEMS;
  };
  auto ring_ptr = [&](int p) { return ring + (p & 1) * C::RING; };
  auto issue = [&](int p) {
    const int s = stage_of(p);
    mbar_arrive_expect_tx(&bars[s], C::STAGE_RAW);
    tma_load_3d(stages + s * C::STAGE_ELEMS, &src, &bars[s], x0 - C::HX,
                y0 - 2, p);
  };

  if (threadIdx.x == 0) {
    tma_prefetch_desc(&src);
    for (int s = 0; s < S0; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int issued_hi = min(hi0, lo0 + S0 - 1);  // same value in every thread
  if (threadIdx.x == 0)
    for (int p = lo0; p <= issued_hi; ++p) issue(p);

  // Loop-invariant addressing.  Level-1 row r (0..15) is y = y0 - 1 + r,
  // level-0 row r + 1 of a stage and ring row r.  Column col = HX + V*lane.
  const int col = C::HX + V * lane;
  const int xg = x0 + V * lane;
  const bool x_lo = (x0 == 0);               // lane 0's w is its own c
  const bool x_hi = (xg + V - 1 == nx - 1);  // this lane's e is its own c
  int c0[RPW], n0[RPW], s0[RPW];  // stage offsets (level 1's inputs)
  int c1[RPW], n1[RPW], s1[RPW];  // ring offsets (level 2's inputs)
  size_t g_off[RPW];
  bool l2row[RPW], store_ok[RPW];
#pragma unroll
  for (int i = 0; i < RPW; ++i) {
    const int r = warp * RPW + i;
    const int y = y0 - 1 + r;
    c0[i] = (r + 1) * P + col;
    n0[i] = (y == 0 ? r + 1 : r) * P + col;
    s0[i] = (y == ny - 1 ? r + 1 : r + 2) * P + col;
    c1[i] = r * P + col;
    n1[i] = (y == 0 ? r : r - 1) * P + col;
    s1[i] = (y == ny - 1 ? r : r + 1) * P + col;
    if constexpr (FLIP) {
      int t = n0[i]; n0[i] = s0[i]; s0[i] = t;
      t = n1[i]; n1[i] = s1[i]; s1[i] = t;
    }
    l2row[i] = (r >= 1 && r <= C::R1 - 2);
    g_off[i] = (size_t)max(y, 0) * nx + xg;
    store_ok[i] = l2row[i] && y < ny && xg < nx;
  }
  // Halo columns of level 1: warp 0 lanes 0..15 take x0-1 (column HX-1) of
  // row `lane`, warp 7 lanes 0..15 take x0+128 (column HX+BX).
  const bool halo = (warp == 0 || warp == C::WARPS - 1) && lane < C::R1;
  const int hcol = (warp == 0) ? C::HX - 1 : C::HX + C::BX;
  const int hx = x0 + hcol - C::HX;  // its x
  const int hy = y0 - 1 + lane;      // its y (row `lane`)
  const int hc = (lane + 1) * P + hcol;
  int hw = hc - 1, he = hc + 1;
  if (hx <= 0) hw = hc;              // only x = 0 can be a left edge here
  if (hx >= nx - 1) he = hc;
  int hn = (hy == 0 ? lane + 1 : lane) * P + hcol;
  int hs = (hy == ny - 1 ? lane + 1 : lane + 2) * P + hcol;
  if constexpr (FLIP) {
    const int t = hn; hn = hs; hs = t;
  }
  const int hring = lane * P + hcol;
  const size_t plane = (size_t)nx * ny;
  const Coef2 kk = coef2(k);

  // Register sets: L0[set][row] level-0 planes, L1[set][row] level-1
  // planes; in iteration q the roles are b, c, t = planes q-2, q-1, q (L0)
  // and q-3, q-2, q-1 (L1).
  V16<float> L0[3][RPW], L1[3][RPW];

  // The chunk's first iteration: level 1 computes plane lo1.
  const int qs = lo1 + 1, qe = z1 + 1;
  int qf = -1;  // the iteration whose wait ran out
  {
    // Thread 0 makes every mbarrier wait; the CTA barrier releases the rest,
    // which then issue nothing while the plane is in flight.
    bool ok = true;
    if (threadIdx.x == 0)
      for (int p = lo0; p <= min(qs, hi0); ++p)
        ok = ok && mbar_wait_bounded(&bars[stage_of(p)], parity_of(p));
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
      qf = lo0 - 1;  // drain every plane issued
    }
  }
  if (qf < 0) {
    // Roles at q = qs with rot 0: b = set 0, c = set 1, t = set 2.
    const float* sc = stage_ptr(lo1);
    const float* sb = stage_ptr(max(lo1 - 1, 0));
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
      L0[1][i] = ld16_shared(sc + c0[i]);
      L0[0][i] = ld16_shared(sb + c0[i]);
    }

    auto iter = [&](auto rot, int q) -> bool {
      constexpr int RB = (decltype(rot)::value + 0) % 3;
      constexpr int RC = (decltype(rot)::value + 1) % 3;
      constexpr int RT = (decltype(rot)::value + 2) % 3;
      const int p1 = q - 1, p2 = q - 2;
      // ---- level 1: plane p1 ------------------------------------------
      if (p1 <= hi1) {
        const float* sc = stage_ptr(p1);
        // t: plane p1+1, or at the top plane nz-1 the plane itself.
        const float* st = stage_ptr(min(p1 + 1, hi0));
        float* ob = ring_ptr(p1);
#pragma unroll
        for (int i = 0; i < RPW; ++i) {
          L0[RT][i] = ld16_shared(st + c0[i]);
          const V16<float>& c = L0[RC][i];
          const V16<float> n = ld16_shared(sc + n0[i]);
          const V16<float> s = ld16_shared(sc + s0[i]);
          float wl = __shfl_up_sync(0xffffffffu, c.e[V - 1], 1);
          float er = __shfl_down_sync(0xffffffffu, c.e[0], 1);
          wl = ld_shared_if(lane == 0 && !x_lo, sc + c0[i] - 1, wl);
          if (lane == 0 && x_lo) wl = c.e[0];
          er = ld_shared_if(lane == 31, sc + c0[i] + V, er);
          if (x_hi) er = c.e[V - 1];
          const V16<float> o =
              point_seg<float>(kk, c, n, s, L0[RB][i], L0[RT][i], wl, er);
          L1[RT][i] = o;
          *reinterpret_cast<V16<float>*>(ob + c1[i]) = o;
        }
        if (halo) {
          const float* sb = stage_ptr(max(p1 - 1, 0));
          const float v = point(k, sc[hc], sc[hw], sc[he], sc[hs], sc[hn],
                                sb[hc], st[hc]);
          ob[hring] = v;
        }
      } else {
#pragma unroll
        for (int i = 0; i < RPW; ++i) L1[RT][i] = L1[RC][i];  // plane nz
      }
      // ---- level 2: plane p2 ------------------------------------------
      if (p2 >= z0) {
        const float* rc = ring_ptr(p2);
        float* out = dst + (size_t)p2 * plane;
#pragma unroll
        for (int i = 0; i < RPW; ++i) {
          if (!l2row[i]) continue;  // warp-uniform
          const V16<float>& c = L1[RC][i];
          const V16<float> n = ld16_shared(rc + n1[i]);
          const V16<float> s = ld16_shared(rc + s1[i]);
          float wl = __shfl_up_sync(0xffffffffu, c.e[V - 1], 1);
          float er = __shfl_down_sync(0xffffffffu, c.e[0], 1);
          wl = ld_shared_if(lane == 0 && !x_lo, rc + c1[i] - 1, wl);
          if (lane == 0 && x_lo) wl = c.e[0];
          er = ld_shared_if(lane == 31, rc + c1[i] + V, er);
          if (x_hi) er = c.e[V - 1];
          const V16<float> o =
              point_seg<float>(kk, c, n, s, L1[RB][i], L1[RT][i], wl, er);
          if (store_ok[i]) st16_global(out + g_off[i], o);
        }
      }
      // Plane -1 is plane 0: the plane just produced at z = 0 is also the
      // b of its next consumer (the c set becomes next iteration's b set).
      if (p1 == 0) {
#pragma unroll
        for (int i = 0; i < RPW; ++i) L1[RC][i] = L1[RT][i];
      }
      // Level 1 of the next iteration needs level-0 plane q+1 (its t).
      bool ok2 = true;
      if (threadIdx.x == 0 && q + 1 <= hi0)
        ok2 = mbar_wait_bounded(&bars[stage_of(q + 1)], parity_of(q + 1));
      if (!__syncthreads_and(ok2)) {
        if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
        return false;
      }
      // Plane q-2 is free now (its last reader was this iteration's halo).
      if (q - 2 >= lo0 && q - 2 + S0 <= hi0) {
        if (threadIdx.x == 0) issue(q - 2 + S0);
        issued_hi = q - 2 + S0;
      }
      return true;
    };

    for (int q = qs; q <= qe; q += 3) {
      if (!iter(std::integral_constant<int, 0>(), q)) { qf = q; break; }
      if (q + 1 > qe) break;
      if (!iter(std::integral_constant<int, 1>(), q + 1)) { qf = q + 1; break; }
      if (q + 2 > qe) break;
      if (!iter(std::integral_constant<int, 2>(), q + 2)) { qf = q + 2; break; }
    }
  }
  if (qf < 0) return;

  // A wait ran out: let every load issued and not yet waited for land
  // (bounded) before the CTA exits.  Waited so far: planes <= qf.
  if (threadIdx.x == 0) {
    for (int p = max(qf + 1, lo0); p <= issued_hi; ++p) {
      bool done = false;
      for (unsigned i = 0; i < (kMaxWaitIters >> 4) && !done; ++i)
        done = mbar_try_wait(&bars[stage_of(p)], parity_of(p));
      if (!done) {
        atomicOr(dev_err, kDevDrainTimeout);
        break;
      }
    }
  }
  __syncthreads();
}

template <bool FLIP, int MINB>
cudaError_t launch_tb2w_t(const CUtensorMap& src, void* f2, int nx, int ny,
                          int nz, const void* coef, int zchunk_override,
                          cudaStream_t stream, unsigned* dev_err,
                          LaunchInfo* info) {
  using C = Tb2w;
  auto kern = steps_tb2w_kernel<FLIP, MINB>;
  cudaError_t e = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
  if (e != cudaSuccess) return e;
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, C::THREADS,
                                                C::SMEM);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int gx = (nx + C::BX - 1) / C::BX;
  const int gy = (ny + C::BY - 1) / C::BY;
  int zchunk = zchunk_override;
  if (zchunk <= 0) {
    // The longest chunk of 256, 128 or 96 planes whose CTAs fill at least
    // one wave and leave the last wave empty or at least 90% full: longer
    // chunks recompute fewer halo planes, a part-filled last wave idles
    // SMs.  Sustained on B200 (Gpt-updates/s): 512^3 (whole waves at all
    // three) 842.5 / 839.7 / 825.9 at 256 / 128 / 96; 768^3 851 at 96
    // (last wave 92% full) against 828 at 128 and 802 at 256; 1024^3 858 at
    // 256.
    const long cap = (long)sms * std::max(occ, 1);
    const long tiles = (long)gx * gy;
    for (int z : {256, 128, 96}) {
      const long ctas = tiles * ((nz + z - 1) / z);
      const long rem = ctas % cap;
      if (ctas >= cap && (rem == 0 || rem * 10 >= cap * 9)) {
        zchunk = std::min(nz, z);
        break;
      }
    }
  }
  if (zchunk <= 0) {
    // Otherwise (measured on B200): 96 planes from nz = 512 on, 32 at
    // 384^3 (743 against 573-695 for 48-128), 16 for shorter grids, which
    // need more chunks to keep CTAs in flight.  Shallow grids of wide
    // planes, whose tiles alone fill two waves, take 128-plane chunks
    // instead of short ones (a z slab of a 1024^2 grid, 130 planes: 840 at
    // 128 against 751 at 16).
    if (nz < 512 && (long)gx * gy >= 2L * sms * std::max(occ, 1))
      zchunk = std::min(nz, 128);
    else
      zchunk = std::min(nz, nz >= 512 ? 96 : nz >= 384 ? 32 : 16);
  }
  const int gz = (nz + zchunk - 1) / zchunk;
  if (info) *info = LaunchInfo{gx, gy, gz, C::THREADS, C::SMEM, zchunk, occ};
  kern<<<dim3(gx, gy, gz), C::THREADS, C::SMEM, stream>>>(
      src, static_cast<float*>(f2), nx, ny, nz, coef_from<float>(coef),
      zchunk, dev_err);
  return cudaGetLastError();
}

}  // namespace

int tb2w_box_x() { return Tb2w::P; }
int tb2w_box_y() { return Tb2w::R0; }

cudaError_t launch_steps_tb2w(const CUtensorMap& src, void* f2, int nx,
                              int ny, int nz, const void* coef,
                              int zchunk_override, int flip_y,
                              cudaStream_t stream, unsigned* dev_err,
                              LaunchInfo* info) {
  return flip_y ? launch_tb2w_t<true, 2>(src, f2, nx, ny, nz, coef,
                                         zchunk_override, stream, dev_err,
                                         info)
                : launch_tb2w_t<false, 2>(src, f2, nx, ny, nz, coef,
                                          zchunk_override, stream, dev_err,
                                          info);
}

}  // namespace d3d
