// Multi-grid TMA step over pitched grids: the solve server's step kernel.
//
// The server keeps every solve in its device arena with a row pitch
// px = nx rounded up to 4 floats (16 bytes), so any grid, whatever its nx,
// can be read with TMA box loads (a tensor map's row stride must be a
// multiple of 16 bytes).  The pad columns x in [nx, px) hold copies of
// column nx-1 -- the replicated x boundary of the reference
// (diffusion3d_openmp.cc:52-53, `e = (x == nx-1) ? c : c + 1`) stored in
// memory -- and every step rewrites them from its own output.  The e
// neighbour of x = nx-1 is then read like any other neighbour and equals
// the centre value, so results are bit-identical to the unpadded field.
//
// Work items are (grid, tile) pairs as in the march kernel (d3d_batch.cu):
// tile = slab * tiles_xy + xy tile.  Each CTA runs the z-march of the
// single-grid TMA kernel (d3d_step.cu) on one tile of one z slab: one
// thread issues a 3-D box load per plane into a ring of S shared stages
// completed through mbarriers (bounded waits), b/c/t of each thread's
// 16-byte segments live in registers, x neighbours come from shuffles
// within the row's lanes, y neighbours from shared memory, and every output
// segment is one 16-byte store.  A row of the tile is LPR lanes wide
// (LPR = 32: 128-column tiles; LPR = 16: 64-column tiles, two rows per warp
// instruction), which bounds the columns wasted on narrow grids.  The strip
// form (pitched_strip_kernel, below; the server's default) maps threads
// onto whole rows instead, so almost no lane falls outside its grid.
//
// The two tensor maps of each grid (its a and b buffers) sit in the work
// descriptors in global memory, rewritten by the host between launches; the
// issuing thread acquires each map through the tensormap proxy before use.
#include <algorithm>
#include <cstdio>

#include "d3d_common.cuh"
#include "d3d_kernels.h"

namespace d3d {

template <int LPR, int BY, int S>
struct PitchedCfg {
  static constexpr int WARPS = 8;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int V = 4;             // floats per 16-byte segment
  static constexpr int BX = LPR * V;      // tile width
  static constexpr int HX = V;            // 16-byte x halo on each side
  static constexpr int P = BX + 2 * HX;   // shared row pitch (floats)
  static constexpr int R = BY + 2;        // rows per stage (1-row y halo)
  static constexpr int SEGR = 32 / LPR;   // rows per warp instruction
  static constexpr int RPW = BY / WARPS;  // tile rows per warp
  static constexpr int NR = RPW / SEGR;   // row sets per thread
  static constexpr int STAGE_BYTES_RAW = P * R * 4;
  static constexpr int STAGE_BYTES = (STAGE_BYTES_RAW + 127) / 128 * 128;
  static constexpr int STAGE_ELEMS = STAGE_BYTES / 4;
  static constexpr int SMEM = S * STAGE_BYTES + S * 8 + 128;
  static_assert(LPR == 32 || LPR == 16, "a tile row is 16 or 32 lanes");
  static_assert(BY % WARPS == 0 && RPW % SEGR == 0 && NR >= 1,
                "every warp owns whole row sets");
  static_assert(P <= 256 && R <= 256, "TMA box dimensions are at most 256");
  static_assert(S >= 4, "the ring keeps planes z, z+1, z+2 and one in flight");
};

__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

template <int LPR, int BY, int S>
__global__ void __launch_bounds__(256)
    pitched_step_kernel(const PitchedDesc* __restrict__ descs,
                        const int2* __restrict__ items, int parity,
                        unsigned* __restrict__ dev_err) {
  using C = PitchedCfg<LPR, BY, S>;
  constexpr int V = C::V;
  constexpr int NR = C::NR;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  float* stages = reinterpret_cast<float*>(base);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * C::STAGE_BYTES);

  const int2 it = items[blockIdx.x];
  const PitchedDesc* dp = descs + it.x;
  const CUtensorMap* src = &dp->map[parity];
  float* __restrict__ dst = parity ? dp->a : dp->b;
  const int nx = dp->nx, px = dp->px, ny = dp->ny, nz = dp->nz;
  const int txy = it.y % dp->tiles_xy, zs = it.y / dp->tiles_xy;
  const int x0 = (txy % dp->tiles_x) * C::BX;
  const int y0 = (txy / dp->tiles_x) * BY;
  const int z0 = zs * dp->zc;
  const int z1 = min(nz, z0 + dp->zc);
  if (z0 >= z1) return;
  const Coef<float> k{dp->k[0], dp->k[1], dp->k[2], dp->k[3],
                      dp->k[4], dp->k[5], dp->k[6], dp->k[7]};
  const int pbase = z0 > 0 ? z0 - 1 : 0;  // first plane loaded (b of z0)
  const int plast = min(z1, nz - 1);      // last plane needed (t of z1-1)

  auto stage_of = [&](int p) { return (int)((unsigned)(p - pbase) % S); };
  auto parity_of = [&](int p) { return ((unsigned)(p - pbase) / S) & 1u; };
  auto stage_ptr = [&](int p) { return stages + stage_of(p) * C::STAGE_ELEMS; };
  auto issue = [&](int p) {
    const int s = stage_of(p);
    mbar_arrive_expect_tx(&bars[s], C::STAGE_BYTES_RAW);
    tma_load_3d(stages + s * C::STAGE_ELEMS, src, &bars[s], x0 - C::HX,
                y0 - 1, p);
  };

  if (threadIdx.x == 0) {
    tensormap_acquire(src);
    tma_prefetch_desc(src);
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int p = pbase; p <= plast && p < pbase + S; ++p) issue(p);
  }

  // Addressing.  Boundary rules are addresses, as in the single-grid
  // kernel: y = 0 / ny-1 read the centre row as n / s, x = 0 reads its own
  // value as w; x = nx-1 reads the pad (a copy of itself) as e, or, when nx
  // fills its last segment, takes its own value for the lane's er.
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sl = lane % LPR, sub = lane / LPR;
  const int xg = x0 + V * sl;
  const int col = C::HX + V * sl;
  const bool x_hi = (xg + V - 1 == nx - 1);
  // The segment that holds x = nx-1 followed by pads: its pad outputs are
  // replaced by the value at nx-1 so the pads stay copies of that column.
  const bool x_cross = (xg < nx) && (xg + V > nx);
  const int jh = nx - 1 - xg;  // index of x = nx-1 in that segment
  int c_off[NR], n_off[NR], s_off[NR];
  size_t g_off[NR];
  bool store_ok[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const int row = warp * C::RPW + r * C::SEGR + sub;
    const int yg = y0 + row;
    c_off[r] = (row + 1) * C::P + col;
    n_off[r] = (yg == 0) ? c_off[r] : row * C::P + col;
    s_off[r] = (yg >= ny - 1) ? c_off[r] : (row + 2) * C::P + col;
    g_off[r] = (size_t)yg * px + xg;
    store_ok[r] = (yg < ny) && (xg < px);
  }
  const int wl_adj = (xg == 0) ? 0 : -1;
  const size_t plane = (size_t)px * ny;
  const Coef2 kk = coef2(k);

  V16<float> q0[NR], q1[NR], q2[NR];
  int drain_lo = pbase, drain_hi = min(plast, pbase + S - 1);

  bool ok = mbar_wait_bounded(&bars[stage_of(z0)], parity_of(z0));
  if (z0 > 0) ok = ok && mbar_wait_bounded(&bars[stage_of(z0 - 1)],
                                           parity_of(z0 - 1));
  if (z0 + 1 <= plast)
    ok = ok && mbar_wait_bounded(&bars[stage_of(z0 + 1)], parity_of(z0 + 1));
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
    goto drain;
  }
  {
    const float* sc = stage_ptr(z0);
    const float* sb = stage_ptr(pbase);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      q1[r] = ld16_shared(sc + c_off[r]);
      q0[r] = ld16_shared(sb + c_off[r]);
    }
  }
  __syncthreads();
  if (z0 > 0 && threadIdx.x == 0 && pbase + S <= plast) issue(pbase + S);

  {
    auto step = [&](int z, const V16<float>* vb, const V16<float>* vc,
                    V16<float>* vt) -> bool {
      const float* sc = stage_ptr(z);
      const float* st = stage_ptr(min(z + 1, nz - 1));
      float* out = dst + (size_t)z * plane;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        vt[r] = ld16_shared(st + c_off[r]);
        const V16<float> n = ld16_shared(sc + n_off[r]);
        const V16<float> s = ld16_shared(sc + s_off[r]);
        float wl = __shfl_up_sync(0xffffffffu, vc[r].e[V - 1], 1, LPR);
        float er = __shfl_down_sync(0xffffffffu, vc[r].e[0], 1, LPR);
        if (sl == 0) wl = sc[c_off[r] + wl_adj];
        if (sl == LPR - 1) er = sc[c_off[r] + V];
        if (x_hi) er = vc[r].e[V - 1];
        V16<float> o = point_seg<float>(kk, vc[r], n, s, vb[r], vt[r], wl, er);
        if (x_cross) {
          if (jh < 1) o.e[1] = o.e[0];
          if (jh < 2) o.e[2] = o.e[1];
          o.e[3] = o.e[2];
        }
        if (store_ok[r]) st16_global(out + g_off[r], o);
      }
      bool ok2 = true;
      if (z + 2 <= plast && z + 1 < z1)
        ok2 = mbar_wait_bounded(&bars[stage_of(z + 2)], parity_of(z + 2));
      if (!__syncthreads_and(ok2)) {
        if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
        return false;
      }
      if (threadIdx.x == 0 && z + S <= plast) issue(z + S);
      return true;
    };

    int zf = -1;
    for (int z = z0; z < z1; z += 3) {
      if (!step(z, q0, q1, q2)) { zf = z; break; }
      if (z + 1 >= z1) break;
      if (!step(z + 1, q1, q2, q0)) { zf = z + 1; break; }
      if (z + 2 >= z1) break;
      if (!step(z + 2, q2, q0, q1)) { zf = z + 2; break; }
    }
    if (zf >= 0) {
      drain_lo = zf + 2;
      drain_hi = min(plast, zf + S - 1);
      goto drain;
    }
  }
  return;

drain:
  // A wait ran out: let every load issued and not yet waited for land
  // before the CTA's shared memory is released.  Bounded as well.
  if (threadIdx.x == 0) {
    for (int p = drain_lo; p <= drain_hi; ++p) {
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

// ---------------------------------------------------------------------------
// Strip form.  A CTA covers `rows` whole rows of one piece of the grid's
// width (the whole pitch when it is at most kStripMaxW columns, else
// near-equal pieces) and a z slab.  Thread i takes the strip's (row,
// segment) pairs with linear index r * 256 + i (r < NR), so nearly every
// lane owns a real segment whatever the width: the tile forms above leave
// a quarter of their lanes outside grids 32..256 wide.  x neighbours are
// shuffles between lanes of one row; a segment at a row or warp edge reads
// its neighbour word from the staged plane instead.  The box, and so the
// stage, is (4 * segs + 8) x (rows + 2) floats, set per grid.
// ---------------------------------------------------------------------------
template <int NR, int MINB>
__global__ void __launch_bounds__(256, MINB)
    pitched_strip_kernel(const PitchedDesc* __restrict__ descs,
                         const int2* __restrict__ items, int parity,
                         unsigned* __restrict__ dev_err) {
  constexpr int S = 4, V = 4, HX = 4;
  constexpr int STAGE = strip_stage_bytes(NR);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  float* stages = reinterpret_cast<float*>(base);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * STAGE);

  const int2 it = items[blockIdx.x];
  const PitchedDesc* dp = descs + it.x;
  const CUtensorMap* src = &dp->map[parity];
  float* __restrict__ dst = parity ? dp->a : dp->b;
  const int nx = dp->nx, px = dp->px, ny = dp->ny, nz = dp->nz;
  const int segs = dp->seg_w, rows = dp->rows;
  const int pw = V * segs + 2 * HX;  // shared row pitch = box width
  const unsigned box_bytes = (unsigned)(pw * (rows + 2)) * 4u;
  const int txy = it.y % dp->tiles_xy, zs = it.y / dp->tiles_xy;
  const int x0 = (txy % dp->tiles_x) * V * segs;
  const int y0 = (txy / dp->tiles_x) * rows;
  const int z0 = zs * dp->zc;
  const int z1 = min(nz, z0 + dp->zc);
  if (z0 >= z1) return;
  const Coef<float> k{dp->k[0], dp->k[1], dp->k[2], dp->k[3],
                      dp->k[4], dp->k[5], dp->k[6], dp->k[7]};
  const int pbase = z0 > 0 ? z0 - 1 : 0;
  const int plast = min(z1, nz - 1);

  auto stage_of = [&](int p) { return (int)((unsigned)(p - pbase) % S); };
  auto parity_of = [&](int p) { return ((unsigned)(p - pbase) / S) & 1u; };
  auto stage_ptr = [&](int p) {
    return stages + stage_of(p) * (STAGE / 4);
  };
  auto issue = [&](int p) {
    const int s = stage_of(p);
    mbar_arrive_expect_tx(&bars[s], box_bytes);
    tma_load_3d(stages + s * (STAGE / 4), src, &bars[s], x0 - HX, y0 - 1,
                p);
  };

  if (threadIdx.x == 0) {
    tensormap_acquire(src);
    tma_prefetch_desc(src);
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int p = pbase; p <= plast && p < pbase + S; ++p) issue(p);
  }

  // Addressing.  Lanes past the strip's rows x segs pairs keep in-box
  // offsets (their row is clamped) and store nothing.  w: x = 0 takes the
  // centre value; a row's first segment and lane 0 read the word before
  // the segment.  e: x = nx-1 in a full last segment takes the centre
  // value, a padded one reads its pad (a copy of nx-1); a row's last
  // segment and lane 31 read the word after the segment.
  const int lane = threadIdx.x & 31;
  // g_off: within one plane (px * ny < 2^31 points, checked at submit).
  int c_off[NR], n_off[NR], s_off[NR], jh[NR], g_off[NR];
  bool store_ok[NR], w_sm[NR], w_own[NR], e_sm[NR], e_own[NR], cross[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const int L = r * 256 + (int)threadIdx.x;
    int row = L / segs;
    const int seg = L - row * segs;
    const bool valid = row < rows;
    row = min(row, rows - 1);
    const int yg = y0 + row, xg = x0 + V * seg;
    c_off[r] = (row + 1) * pw + HX + V * seg;
    n_off[r] = (yg == 0) ? c_off[r] : c_off[r] - pw;
    s_off[r] = (yg >= ny - 1) ? c_off[r] : c_off[r] + pw;
    g_off[r] = yg * px + xg;
    store_ok[r] = valid && yg < ny && xg < px;
    w_own[r] = (xg == 0);
    w_sm[r] = !w_own[r] && (seg == 0 || lane == 0);
    e_own[r] = (xg + V - 1 == nx - 1);
    e_sm[r] = !e_own[r] && (seg == segs - 1 || lane == 31);
    cross[r] = (xg < nx) && (xg + V > nx);
    jh[r] = nx - 1 - xg;
  }
  const size_t plane = (size_t)px * ny;
  const Coef2 kk = coef2(k);

  V16<float> q0[NR], q1[NR], q2[NR];
  int drain_lo = pbase, drain_hi = min(plast, pbase + S - 1);

  bool ok = mbar_wait_bounded(&bars[stage_of(z0)], parity_of(z0));
  if (z0 > 0) ok = ok && mbar_wait_bounded(&bars[stage_of(z0 - 1)],
                                           parity_of(z0 - 1));
  if (z0 + 1 <= plast)
    ok = ok && mbar_wait_bounded(&bars[stage_of(z0 + 1)], parity_of(z0 + 1));
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
    goto drain;
  }
  {
    const float* sc = stage_ptr(z0);
    const float* sb = stage_ptr(pbase);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      q1[r] = ld16_shared(sc + c_off[r]);
      q0[r] = ld16_shared(sb + c_off[r]);
    }
  }
  __syncthreads();
  if (z0 > 0 && threadIdx.x == 0 && pbase + S <= plast) issue(pbase + S);

  {
    auto step = [&](int z, const V16<float>* vb, const V16<float>* vc,
                    V16<float>* vt) -> bool {
      const float* sc = stage_ptr(z);
      const float* st = stage_ptr(min(z + 1, nz - 1));
      float* out = dst + (size_t)z * plane;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        vt[r] = ld16_shared(st + c_off[r]);
        const V16<float> n = ld16_shared(sc + n_off[r]);
        const V16<float> s = ld16_shared(sc + s_off[r]);
        float wl = __shfl_up_sync(0xffffffffu, vc[r].e[V - 1], 1);
        float er = __shfl_down_sync(0xffffffffu, vc[r].e[0], 1);
        wl = ld_shared_if(w_sm[r], sc + c_off[r] - 1, wl);
        if (w_own[r]) wl = vc[r].e[0];
        er = ld_shared_if(e_sm[r], sc + c_off[r] + V, er);
        if (e_own[r]) er = vc[r].e[V - 1];
        V16<float> o = point_seg<float>(kk, vc[r], n, s, vb[r], vt[r], wl, er);
        if (cross[r]) {
          if (jh[r] < 1) o.e[1] = o.e[0];
          if (jh[r] < 2) o.e[2] = o.e[1];
          o.e[3] = o.e[2];
        }
        if (store_ok[r]) st16_global(out + g_off[r], o);
      }
      bool ok2 = true;
      if (z + 2 <= plast && z + 1 < z1)
        ok2 = mbar_wait_bounded(&bars[stage_of(z + 2)], parity_of(z + 2));
      if (!__syncthreads_and(ok2)) {
        if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
        return false;
      }
      if (threadIdx.x == 0 && z + S <= plast) issue(z + S);
      return true;
    };

    int zf = -1;
    for (int z = z0; z < z1; z += 3) {
      if (!step(z, q0, q1, q2)) { zf = z; break; }
      if (z + 1 >= z1) break;
      if (!step(z + 1, q1, q2, q0)) { zf = z + 1; break; }
      if (z + 2 >= z1) break;
      if (!step(z + 2, q2, q0, q1)) { zf = z + 2; break; }
    }
    if (zf >= 0) {
      drain_lo = zf + 2;
      drain_hi = min(plast, zf + S - 1);
      goto drain;
    }
  }
  return;

drain:
  if (threadIdx.x == 0) {
    for (int p = drain_lo; p <= drain_hi; ++p) {
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

// ---------------------------------------------------------------------------
// Two fused steps per pass, strip form.  For grids whose pitch fits one
// piece (px <= kStripMaxW) a strip spans whole rows, so the intermediate
// level needs a y halo (one row above and below) and a z halo, and no x
// halo at all.  Level 0 is TMA-loaded as (4 * segs + 8) x (rows + 4)
// boxes into a 4-stage ring; level 1 is computed over rows + 2 rows into a
// 4-slot shared ring; level 2 reads its b, c, t, n, s from that ring and
// stores to HBM.  Both levels map threads linearly onto their own (row,
// segment) pairs, so neither wastes lanes.  In iteration q level 1 makes
// plane q-1 and level 2 plane q-3, which reads only ring planes written in
// earlier iterations: one block barrier per plane.  Every operand is a
// shared-memory load (no register queues, since the two levels' thread
// maps differ by a row), so a fused pair issues more instructions than two
// single strip steps; on B200 the batch autotuner measures it (temporal-
// block depth 2) against the single-step kinds per size class.
// ---------------------------------------------------------------------------
template <int NR>
__global__ void __launch_bounds__(256, 4 / NR)
    pitched_strip2_kernel(const PitchedDesc* __restrict__ descs,
                          const int2* __restrict__ items, int parity,
                          unsigned* __restrict__ dev_err) {
  constexpr int S0 = 4, V = 4, HX = 4, NR1 = NR + 1;
  constexpr int STAGE = strip2_slot_bytes(NR);  // level-0 stage
  constexpr int SLOT = strip2_slot_bytes(NR);   // level-1 ring slot
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  float* stages = reinterpret_cast<float*>(base);
  float* ring = reinterpret_cast<float*>(base + S0 * STAGE);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + S0 * STAGE + 4 * SLOT);

  const int2 it = items[blockIdx.x];
  const PitchedDesc* dp = descs + it.x;
  const CUtensorMap* src = &dp->map[parity];
  float* __restrict__ dst = parity ? dp->a : dp->b;
  const int nx = dp->nx, px = dp->px, ny = dp->ny, nz = dp->nz;
  const int segs = dp->seg_w, rows = dp->rows;
  const int pw = V * segs + 2 * HX;  // row pitch of stages and ring
  const unsigned box_bytes = (unsigned)(pw * (rows + 4)) * 4u;
  const int y0 = (it.y % dp->tiles_xy) * rows;
  const int z0 = (it.y / dp->tiles_xy) * dp->zc;
  const int z1 = min(nz, z0 + dp->zc);
  if (z0 >= z1) return;
  const Coef<float> k{dp->k[0], dp->k[1], dp->k[2], dp->k[3],
                      dp->k[4], dp->k[5], dp->k[6], dp->k[7]};
  // Level-1 planes [lo1, hi1], level-0 planes [lo0, hi0].
  const int lo1 = max(z0 - 1, 0), hi1 = min(z1, nz - 1);
  const int lo0 = max(z0 - 2, 0), hi0 = min(z1 + 1, nz - 1);

  auto stage_of = [&](int p) { return (int)((unsigned)(p - lo0) % S0); };
  auto parity_of = [&](int p) { return ((unsigned)(p - lo0) / S0) & 1u; };
  auto stage_ptr = [&](int p) { return stages + stage_of(p) * (STAGE / 4); };
  auto ring_ptr = [&](int p) { return ring + (p & 3) * (SLOT / 4); };
  auto issue = [&](int p) {
    const int s = stage_of(p);
    mbar_arrive_expect_tx(&bars[s], box_bytes);
    tma_load_3d(stages + s * (STAGE / 4), src, &bars[s], -HX, y0 - 2, p);
  };

  if (threadIdx.x == 0) {
    tensormap_acquire(src);
    tma_prefetch_desc(src);
    for (int s = 0; s < S0; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int issued_hi = min(hi0, lo0 + S0 - 1);  // same value in every thread
  if (threadIdx.x == 0)
    for (int p = lo0; p <= issued_hi; ++p) issue(p);

  // Addressing shared by both levels for a (row r of the ring / stage
  // frame, segment): offset r * pw + HX + 4 * seg.  Level-1 row r1 is
  // y = y0 - 1 + r1 (stage row r1 + 1, ring row r1); level-2 row r2 is
  // y = y0 + r2 (ring row r2 + 1).  Rules: y = 0 / ny-1 read the centre
  // row as n / s; x = 0 takes the centre value as w; x = nx-1 in a full
  // last segment takes the centre value as e, a padded one reads its pad;
  // a row's or warp's edge segment reads the word beside it.
  const int lane = threadIdx.x & 31;
  struct Cell {
    int c, n, s;     // offsets within a stage or ring plane
    bool w_sm, w_own, e_sm, e_own, cross, live;
    int jh;
  };
  auto make_cell = [&](int L, int nrows, int frame_row0, int yoff,
                       size_t* g_off) {
    Cell cl;
    int row = L / segs;
    const int seg = L - row * segs;
    cl.live = row < nrows;
    row = min(row, nrows - 1);
    const int y = yoff + row, xg = V * seg;
    cl.c = (frame_row0 + row) * pw + HX + V * seg;
    cl.n = (y == 0) ? cl.c : cl.c - pw;
    cl.s = (y >= ny - 1) ? cl.c : cl.c + pw;
    cl.w_own = (xg == 0);
    cl.w_sm = !cl.w_own && (seg == 0 || lane == 0);
    cl.e_own = (xg + V - 1 == nx - 1);
    cl.e_sm = !cl.e_own && (seg == segs - 1 || lane == 31);
    cl.cross = (xg < nx) && (xg + V > nx);
    cl.jh = nx - 1 - xg;
    if (g_off) {
      *g_off = (size_t)y * px + xg;
      cl.live = cl.live && y < ny && xg < px;
    }
    return cl;
  };
  Cell c1[NR1], c2[NR];
  size_t g_off[NR];
#pragma unroll
  for (int j = 0; j < NR1; ++j)
    c1[j] = make_cell(j * 256 + (int)threadIdx.x, rows + 2, 1, y0 - 1,
                      nullptr);
#pragma unroll
  for (int r = 0; r < NR; ++r)
    c2[r] = make_cell(r * 256 + (int)threadIdx.x, rows, 1, y0, &g_off[r]);
  const size_t plane = (size_t)px * ny;
  const Coef2 kk = coef2(k);

  // One segment from a plane frame: c, n, s, w, e from plane `pc`, b and t
  // from planes `pb`, `pt` (same offsets).
  auto seg_point = [&](const Cell& cl, const float* pc, const float* pb,
                       const float* pt) {
    const V16<float> c = ld16_shared(pc + cl.c);
    const V16<float> n = ld16_shared(pc + cl.n);
    const V16<float> s = ld16_shared(pc + cl.s);
    const V16<float> b = ld16_shared(pb + cl.c);
    const V16<float> t = ld16_shared(pt + cl.c);
    float wl = __shfl_up_sync(0xffffffffu, c.e[V - 1], 1);
    float er = __shfl_down_sync(0xffffffffu, c.e[0], 1);
    wl = ld_shared_if(cl.w_sm, pc + cl.c - 1, wl);
    if (cl.w_own) wl = c.e[0];
    er = ld_shared_if(cl.e_sm, pc + cl.c + V, er);
    if (cl.e_own) er = c.e[V - 1];
    V16<float> o = point_seg<float>(kk, c, n, s, b, t, wl, er);
    if (cl.cross) {
      if (cl.jh < 1) o.e[1] = o.e[0];
      if (cl.jh < 2) o.e[2] = o.e[1];
      o.e[3] = o.e[2];
    }
    return o;
  };

  const int qs = lo1 + 1, qe = z1 + 2;
  int qf = -1;  // the iteration whose wait ran out
  {
    bool ok = true;
    for (int p = lo0; p <= min(qs, hi0); ++p)
      ok = ok && mbar_wait_bounded(&bars[stage_of(p)], parity_of(p));
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
      qf = lo0 - 1;
    }
  }
  if (qf < 0) {
    for (int q = qs; q <= qe; ++q) {
      const int p1 = q - 1, p2 = q - 3;
      if (p1 <= hi1) {  // level 1: plane p1 into the ring
        const float* pc = stage_ptr(p1);
        const float* pb = stage_ptr(max(p1 - 1, 0));
        const float* pt = stage_ptr(min(p1 + 1, nz - 1));
        float* out = ring_ptr(p1);
#pragma unroll
        for (int j = 0; j < NR1; ++j) {
          const V16<float> o = seg_point(c1[j], pc, pb, pt);
          if (c1[j].live)
            *reinterpret_cast<V16<float>*>(out + c1[j].c - pw) = o;
        }
      }
      if (p2 >= z0) {  // level 2: plane p2 to HBM
        const float* pc = ring_ptr(p2);
        const float* pb = ring_ptr(max(p2 - 1, 0));
        const float* pt = ring_ptr(min(p2 + 1, nz - 1));
        float* out = dst + (size_t)p2 * plane;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const V16<float> o = seg_point(c2[r], pc, pb, pt);
          if (c2[r].live) st16_global(out + g_off[r], o);
        }
      }
      // Level 1 of the next iteration needs level-0 plane q+1.
      bool ok2 = true;
      if (q + 1 <= hi0)
        ok2 = mbar_wait_bounded(&bars[stage_of(q + 1)], parity_of(q + 1));
      if (!__syncthreads_and(ok2)) {
        if (threadIdx.x == 0) atomicOr(dev_err, kDevWaitTimeout);
        qf = q;
        break;
      }
      // Plane q-2 is free now (its last reader was this level-1 plane).
      if (q - 2 >= lo0 && q - 2 + S0 <= hi0) {
        if (threadIdx.x == 0) issue(q - 2 + S0);
        issued_hi = q - 2 + S0;
      }
    }
  }
  if (qf < 0) return;
  // A wait ran out: let every load issued and not yet waited for land
  // (bounded) before the CTA exits.
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

// Between the host's dense rows (nx floats) and the arena's pitched rows
// (px floats): `to_pitched` writes every x in [0, px) of dst from
// src[min(x, nx-1)], which also fills the pads; otherwise dst takes the
// first nx floats of each pitched row.  Blocks stride over rows.
__global__ void __launch_bounds__(128)
    repitch_kernel(const float* __restrict__ src, float* __restrict__ dst,
                   int nx, int px, long long rows, bool to_pitched) {
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    if (to_pitched) {
      const float* in = src + (size_t)r * nx;
      float* out = dst + (size_t)r * px;
      for (int x = threadIdx.x; x < px; x += blockDim.x)
        out[x] = in[min(x, nx - 1)];
    } else {
      const float* in = src + (size_t)r * px;
      float* out = dst + (size_t)r * nx;
      for (int x = threadIdx.x; x < nx; x += blockDim.x) out[x] = in[x];
    }
  }
}

namespace {

// (row lanes, rows per tile, planes in the ring).
const PitchedVariant kPitched[kNumPitchedVariants] = {
    {16, 16, 4}, {32, 16, 4}, {32, 32, 4}, {16, 32, 4}, {32, 8, 4}};

template <int LPR, int BY, int S>
cudaError_t launch_t(const PitchedDesc* descs, const int2* items, int n,
                     int parity, cudaStream_t s, unsigned* dev_err) {
  using C = PitchedCfg<LPR, BY, S>;
  auto kern = pitched_step_kernel<LPR, BY, S>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  kern<<<n, C::THREADS, C::SMEM, s>>>(descs, items, parity, dev_err);
  return cudaGetLastError();
}

}  // namespace

const PitchedVariant& pitched_variant(int v) { return kPitched[v]; }

int pitched_box_x(int v) { return kPitched[v].lanes * 4 + 8; }
int pitched_box_y(int v) { return kPitched[v].by + 2; }

cudaError_t launch_pitched_step(int variant, const PitchedDesc* descs,
                                const int2* items, int nitems, int parity,
                                cudaStream_t s, unsigned* dev_err) {
  if (nitems <= 0) return cudaSuccess;
  switch (variant) {
    case 0: return launch_t<16, 16, 4>(descs, items, nitems, parity, s, dev_err);
    case 1: return launch_t<32, 16, 4>(descs, items, nitems, parity, s, dev_err);
    case 2: return launch_t<32, 32, 4>(descs, items, nitems, parity, s, dev_err);
    case 3: return launch_t<16, 32, 4>(descs, items, nitems, parity, s, dev_err);
    case 4: return launch_t<32, 8, 4>(descs, items, nitems, parity, s, dev_err);
    default: return cudaErrorInvalidValue;
  }
}

// Many grids' repitch in one launch: block row blockIdx.y takes grids
// blockIdx.y, blockIdx.y + gridDim.y, ...; blockIdx.x strides their rows.
__global__ void __launch_bounds__(128)
    repitch_multi_kernel(const RepitchDesc* __restrict__ d, int n,
                         bool to_pitched) {
  for (int g = blockIdx.y; g < n; g += gridDim.y) {
    const RepitchDesc r = d[g];
    for (long long row = blockIdx.x; row < r.rows; row += gridDim.x) {
      if (to_pitched) {
        const float* in = r.dense + (size_t)row * r.nx;
        float* out = r.pitched + (size_t)row * r.px;
        for (int x = threadIdx.x; x < r.px; x += blockDim.x)
          out[x] = in[min(x, r.nx - 1)];
      } else {
        const float* in = r.pitched + (size_t)row * r.px;
        float* out = r.dense + (size_t)row * r.nx;
        for (int x = threadIdx.x; x < r.nx; x += blockDim.x) out[x] = in[x];
      }
    }
  }
}

cudaError_t launch_repitch_multi(const RepitchDesc* d, int n,
                                 bool to_pitched, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const dim3 grid(8, (unsigned)std::min(n, 65535));
  repitch_multi_kernel<<<grid, 128, 0, s>>>(d, n, to_pitched);
  return cudaGetLastError();
}

StripShape strip_shape(int px, int ny, int nr) {
  StripShape sh;
  sh.pieces = (px + kStripMaxW - 1) / kStripMaxW;
  const int w = ((px + sh.pieces - 1) / sh.pieces + 3) / 4 * 4;
  sh.segs = w / 4;
  sh.rows = std::max(1, std::min({64, ny, nr * 256 / sh.segs}));
  while (sh.rows > 1 && (w + 8) * (sh.rows + 2) * 4 > strip_stage_bytes(nr))
    --sh.rows;
  return sh;
}

cudaError_t launch_pitched_strip(int nr, const PitchedDesc* descs,
                                 const int2* items, int nitems, int parity,
                                 cudaStream_t s, unsigned* dev_err) {
  if (nitems <= 0) return cudaSuccess;
  auto go = [&](auto kern, int smem) {
    static bool attr_set[2] = {false, false};
    bool& set = attr_set[nr - 1];
    if (!set) {
      cudaError_t e = cudaFuncSetAttribute(
          kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      set = true;
    }
    kern<<<nitems, 256, smem, s>>>(descs, items, parity, dev_err);
    return cudaGetLastError();
  };
  // Register budgets: 64 a thread for one segment (4 CTAs/SM), 80 for two
  // (3 CTAs/SM; at 64 it spills and measured 6% slower on B200).
  if (nr == 1)
    return go(pitched_strip_kernel<1, 4>,
              4 * strip_stage_bytes(1) + 4 * 8 + 128);
  if (nr == 2)
    return go(pitched_strip_kernel<2, 3>,
              4 * strip_stage_bytes(2) + 4 * 8 + 128);
  return cudaErrorInvalidValue;
}

StripShape strip2_shape(int px, int ny, int nr) {
  StripShape sh{1, px / 4, 1};
  if (px > kStripMaxW) {  // no two-step form: the strip needs x halos
    sh.pieces = 0;
    return sh;
  }
  const int pw = px + 8;
  sh.rows = std::max(1, std::min({64, ny, nr * 256 / sh.segs}));
  while (sh.rows > 1 && pw * (sh.rows + 4) * 4 > strip2_slot_bytes(nr))
    --sh.rows;
  return sh;
}

cudaError_t launch_pitched_strip2(int nr, const PitchedDesc* descs,
                                  const int2* items, int nitems, int parity,
                                  cudaStream_t s, unsigned* dev_err) {
  if (nitems <= 0) return cudaSuccess;
  auto go = [&](auto kern, int smem) {
    static bool attr_set[2] = {false, false};
    bool& set = attr_set[nr - 1];
    if (!set) {
      cudaError_t e = cudaFuncSetAttribute(
          kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      set = true;
    }
    kern<<<nitems, 256, smem, s>>>(descs, items, parity, dev_err);
    return cudaGetLastError();
  };
  if (nr == 1)
    return go(pitched_strip2_kernel<1>, 8 * strip2_slot_bytes(1) + 4 * 8 + 128);
  if (nr == 2)
    return go(pitched_strip2_kernel<2>, 8 * strip2_slot_bytes(2) + 4 * 8 + 128);
  return cudaErrorInvalidValue;
}

cudaError_t launch_repitch(const float* src, float* dst, int nx, int px,
                           long long rows, bool to_pitched, cudaStream_t s) {
  if (rows <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>(rows, 148LL * 16);
  repitch_kernel<<<(unsigned)blocks, 128, 0, s>>>(src, dst, nx, px, rows,
                                                  to_pitched);
  return cudaGetLastError();
}

}  // namespace d3d
