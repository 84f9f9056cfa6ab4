// Cluster-resident multi-grid kernel: whole small grids live in shared
// memory for all of their steps.
//
// A batch of small grids (the 16..96-per-axis batch: at most 3.5 MiB per
// buffer) streams every grid through HBM once per step when each step is a
// launch: 8 bytes per point-update, whatever the kernel.  Here a thread-
// block cluster of C CTAs (C <= 16) holds one grid in its shared memory,
// split into z slabs of `pc` planes per CTA, and runs all of that grid's
// steps before it takes the next grid: HBM sees the grid once on the way in
// and once on the way out.  The launch is persistent: one launch per
// (cluster size, thread shape) class walks that class's grids, largest work
// first, through an atomic work counter, and records each grid's completed
// steps in a per-grid counter.
//
// One step (the reference's update, diffusion3d_openmp.cc:43-71, evaluated
// with d3d::point_seg: same order, same rounding):
//   1. cluster barrier: the previous step's planes (or the loaded input)
//      are complete in every CTA;
//   2. each thread pulls, for its own columns, the plane below its slab
//      (the b of its first plane) from the lower neighbour CTA's shared
//      memory into registers, and the plane above its slab (the t of its
//      last plane) into a one-plane halo buffer of its own CTA (DSMEM loads,
//      ld.shared::cluster; no TMA, no multicast);
//   3. cluster barrier: every pull is done, so planes may be overwritten
//      (each thread arrives right after its pulls and waits only before
//      its first write, so the new values of the first plane are computed
//      while the other CTAs arrive);
//   4. z-march over the slab, in place: b and c of each thread's 16-byte
//      segments ride in registers, t, n, s come from shared memory, x
//      neighbours from shuffles (lanes at a row or warp edge read the
//      staged word); a block barrier separates the reads of plane p from
//      the writes of its new values.
// Replicated boundaries: x = 0 and the last segment take their own value
// (the pads x in [nx, px) hold copies of column nx-1 and are rewritten each
// step), y = 0 / ny-1 read their own row, z = 0 / nz-1 their own plane.
//
// Synchronisation is the hardware cluster barrier only (every CTA of a
// cluster runs the same loop bounds, read from the same descriptor); no
// thread spins on a flag, so there is no wait to bound.  A CTA with no
// planes (nz < C * pc) still takes part in every barrier.
#include <algorithm>
#include <cstdio>

#include "d3d_common.cuh"
#include "d3d_kernels.h"

namespace d3d {

namespace {

// Every thread of every CTA of the cluster arrives (release) and waits
// (acquire): shared-memory accesses before the arrive, local or remote, are
// ordered before every access of the cluster after the wait.  The
// non-.aligned forms, so a warp need not be converged at the barrier.  A
// thread alternates arrive and wait; work between the two overlaps the
// other CTAs' arrival.
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire;" ::: "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  cluster_arrive();
  cluster_wait();
}

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// The shared::cluster address of `cta_addr` (a shared::cta address) in CTA
// `rank` of this cluster.
__device__ __forceinline__ uint32_t map_to_rank(uint32_t cta_addr,
                                                unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(r)
               : "r"(cta_addr), "r"(rank));
  return r;
}

__device__ __forceinline__ V16<float> ld16_cluster(uint32_t addr) {
  V16<float> v;
  asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.e[0]), "=f"(v.e[1]), "=f"(v.e[2]), "=f"(v.e[3])
               : "r"(addr)
               : "memory");
  return v;
}

__device__ __forceinline__ int ld_cluster_s32(uint32_t addr) {
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];"
               : "=r"(v)
               : "r"(addr)
               : "memory");
  return v;
}

__device__ __forceinline__ void st16_shared(float* p, const V16<float>& v) {
  *reinterpret_cast<int4*>(p) = *reinterpret_cast<const int4*>(&v);
}

// Flag bits of a thread's unit (one 16-byte segment of one row).
enum : unsigned {
  kValid = 1u,
  kWOwn = 2u,    // x = 0: w is the centre value
  kWSm = 4u,     // lane 0 inside a row: w is the staged word before
  kEOwn = 8u,    // last segment of the row: e is the centre value
  kESm = 16u,    // lane 31 inside a row: e is the staged word after
  kNOwn = 32u,   // y = 0: n is the own row
  kSOwn = 64u,   // y = ny-1: s is the own row
  kCross = 128u,  // the segment holds x = nx-1 followed by pads
  kPullN = 1024u,  // first row of a part not at y = 0: pulls the y halo below
  kPullS = 2048u   // last row of a part not at y = ny-1: pulls the one above
};
constexpr int kYBatch = 4;  // y-halo planes pulled per batch of loads

// PARTS: the grid's planes are cut into row parts (d.yparts > 1); without
// it the code for the y halo is left out.
template <int NT, int UMAX, bool PARTS>
__device__ __forceinline__ void resident_grid(const ResidentDesc& d,
                                              unsigned rank, float* sm,
                                              int* __restrict__ steps_done,
                                              int g) {
  const int tid = threadIdx.x, lane = tid & 31;
  const int nx = d.nx, ny = d.ny, nz = d.nz, px = d.px, S = d.segs;
  const int pc = d.pc;
  // Cluster rank = zk * yparts + yk: rows [y0, y0 + yn) of planes
  // [z0, z1).  With row parts (yparts > 1) a plane in shared memory is
  // rows + 2 rows of px floats: row 0 and row rows + 1 hold the
  // neighbouring parts' edge rows (the y halo), rows 1..yn this CTA's rows;
  // whole planes (yparts = 1) have no halo rows.  Every CTA of the grid has
  // the same layout (rows = ceil(ny / yparts)), so a neighbour's plane p
  // starts at the same offset.
  const int yparts = PARTS ? d.yparts : 1, rows = PARTS ? d.rows : ny;
  const int yk = (int)rank % yparts, zk = (int)rank / yparts;
  const int y0 = yk * rows;
  const int yn = max(0, min(ny, y0 + rows) - y0);
  const int hrow = PARTS ? 1 : 0;  // first row of the CTA's own rows
  const int plane = px * (rows + 2 * hrow);
  const int z0 = zk * pc;
  const int z1 = min(nz, z0 + pc);
  const int np = yn > 0 ? max(0, z1 - z0) : 0;
  float* halo = sm + pc * plane;  // the plane above the slab (t of z1-1)

  // Load the slab: rows of nx floats into rows of px, pads from nx-1.
  {
    const int nrow = np * yn;
    for (int r = tid >> 5; r < nrow; r += NT / 32) {
      const int zz = r / yn, yy = r - zz * yn;
      const float* in = d.in + ((size_t)(z0 + zz) * ny + y0 + yy) * nx;
      float* o = sm + zz * plane + (yy + hrow) * px;
      for (int x = lane; x < px; x += 32) o[x] = in[min(x, nx - 1)];
    }
  }

  // This thread's units u = tid + i * NT of the plane (S segments a row).
  const int units = S * yn;
  // Narrow thread shapes (2 units a thread) keep the rows above and below
  // as offsets and rotate three register sets through the b, c, t roles;
  // the wide ones (4 and 6 units) derive the row offsets from the flags and
  // keep only b in registers, loading c from shared memory each plane (one
  // more load a segment, two register sets fewer).
  constexpr bool kWide = UMAX > 2;
  int c_off[UMAX], n_off[UMAX], s_off[UMAX];
  unsigned fl[UMAX];  // flag bits; bits 8..9: index of x = nx-1 if kCross
#pragma unroll
  for (int i = 0; i < UMAX; ++i) {
    const int u = tid + i * NT;
    const bool valid = u < units;
    const int uu = valid ? u : 0;
    const int r = uu / S, seg = uu - r * S;  // r: row within the part
    const int yg = y0 + r, xg = 4 * seg;
    c_off[i] = (r + hrow) * px + xg;
    // y = 0 / ny-1 read their own row; a part's edge row reads the halo
    // row the pull fills.
    n_off[i] = yg == 0 ? c_off[i] : c_off[i] - px;
    s_off[i] = yg == ny - 1 ? c_off[i] : c_off[i] + px;
    unsigned f = valid ? kValid : 0u;
    if (seg == 0) f |= kWOwn;
    else if (lane == 0) f |= kWSm;
    if (seg == S - 1) f |= kEOwn;
    else if (lane == 31) f |= kESm;
    if (yg == 0) f |= kNOwn;
    if (yg == ny - 1) f |= kSOwn;
    if (valid && r == 0 && yg > 0) f |= kPullN;
    if (valid && r == yn - 1 && yg < ny - 1) f |= kPullS;
    if (xg + 4 > nx) f |= kCross | ((unsigned)(nx - 1 - xg) << 8);
    fl[i] = f;
  }
  const Coef<float> k{d.k[0], d.k[1], d.k[2], d.k[3],
                      d.k[4], d.k[5], d.k[6], d.k[7]};
  const Coef2 kk = coef2(k);
  const uint32_t sm_base = smem_u32(sm);
  // z neighbours: the same rows of the slabs below and above (ranks
  // -/+ yparts); y neighbours: the parts before and after (ranks -/+ 1).
  const uint32_t below =
      z0 > 0 ? map_to_rank(sm_base, rank - yparts) + 4u * (pc - 1) * plane
             : 0u;
  const uint32_t above = z1 < nz ? map_to_rank(sm_base, rank + yparts) : 0u;
  // The part before is full and ends with row `rows` of its layout; the
  // part after starts with row 1.  Their rows land in this CTA's rows 0
  // and yn + 1: for a first-row unit (row 1, c_off = px + x) the source is
  // the part before's row `rows` at x, for a last-row unit (row yn,
  // c_off = yn * px + x) the part after's row 1 at x.
  const uint32_t ybelow = yk > 0 ? map_to_rank(sm_base, rank - 1) : 0u;
  const uint32_t yabove =
      yk + 1 < yparts && y0 + yn < ny ? map_to_rank(sm_base, rank + 1) : 0u;

  // One plane of the march: b in vb, c in vc (narrow shapes; the wide ones
  // load it), t loaded and kept in vt for the next plane (narrow: three
  // register sets whose roles rotate, so nothing is copied; wide: vt is vb
  // and receives c), the new values held until every thread of the CTA has
  // read plane p, then stored over it.  Before the first store of a step,
  // every CTA's pulls must be done.
  V16<float> q0[UMAX], q1[UMAX], q2[UMAX], nv[UMAX];
  auto plane_step = [&](int p, const V16<float>* vb, const V16<float>* vc,
                        V16<float>* vt) {
    float* pl = sm + p * plane;
    const float* tp = p + 1 < np ? pl + plane : (z1 < nz ? halo : pl);
#pragma unroll
    for (int i = 0; i < UMAX; ++i) {
      const unsigned f = fl[i];
      const V16<float> c = kWide ? ld16_shared(pl + c_off[i]) : vc[i];
      const V16<float> t = ld16_shared(tp + c_off[i]);
      const int no = kWide ? c_off[i] - ((f & kNOwn) ? 0 : px) : n_off[i];
      const int sof = kWide ? c_off[i] + ((f & kSOwn) ? 0 : px) : s_off[i];
      const V16<float> n = ld16_shared(pl + no);
      const V16<float> so = ld16_shared(pl + sof);
      float wl = __shfl_up_sync(0xffffffffu, c.e[3], 1);
      float er = __shfl_down_sync(0xffffffffu, c.e[0], 1);
      wl = ld_shared_if(f & kWSm, pl + c_off[i] - 1, wl);
      if (f & kWOwn) wl = c.e[0];
      er = ld_shared_if(f & kESm, pl + c_off[i] + 4, er);
      if (f & kEOwn) er = c.e[3];
      V16<float> o = point_seg<float>(kk, c, n, so, vb[i], t, wl, er);
      if (f & kCross) {
        const unsigned jh = (f >> 8) & 3u;
        if (jh < 1) o.e[1] = o.e[0];
        if (jh < 2) o.e[2] = o.e[1];
        o.e[3] = o.e[2];
      }
      nv[i] = o;
      // Narrow: t goes to the set that is c next plane.  Wide: c is the b
      // of the next plane (vb and vt are the same set there).
      vt[i] = kWide ? c : t;
    }
    __syncthreads();  // plane p read everywhere in this CTA
    if (p == 0) cluster_wait();  // every pull of the cluster is done
#pragma unroll
    for (int i = 0; i < UMAX; ++i)
      if (fl[i] & kValid) st16_shared(pl + c_off[i], nv[i]);
  };

  cluster_arrive();  // the slab is loaded
  for (int s = 0; s < d.steps; ++s) {
    cluster_wait();  // planes of the previous step complete everywhere
    if (np > 0) {
#pragma unroll
      for (int i = 0; i < UMAX; ++i) {
        q0[i] = z0 > 0 ? ld16_cluster(below + 4u * c_off[i])
                       : ld16_shared(sm + c_off[i]);
        if (z1 < nz && (fl[i] & kValid))
          st16_shared(halo + c_off[i], ld16_cluster(above + 4u * c_off[i]));
      }
      // y halo of every plane of the slab: the row under a part's first
      // row, the row over its last row (old values, as the z halo), in
      // batches of kYBatch planes whose remote loads are all issued before
      // any is stored, so their latencies overlap.
#pragma unroll
      for (int i = 0; i < UMAX && PARTS; ++i) {
        if (!(fl[i] & (kPullN | kPullS))) continue;
        const bool dn = fl[i] & kPullN;
        const int dst = dn ? c_off[i] - px : c_off[i] + px;
        const uint32_t src =
            dn ? ybelow + 4u * (rows * px + c_off[i] - px)
               : yabove + 4u * (px + c_off[i] - yn * px);
        for (int p0 = 0; p0 < np; p0 += kYBatch) {
          V16<float> yv[kYBatch];
#pragma unroll
          for (int j = 0; j < kYBatch; ++j)
            if (p0 + j < np)
              yv[j] = ld16_cluster(src + 4u * (p0 + j) * plane);
#pragma unroll
          for (int j = 0; j < kYBatch; ++j)
            if (p0 + j < np) st16_shared(sm + (p0 + j) * plane + dst, yv[j]);
        }
      }
    }
    // This thread's pulls are done; the new values of plane 0 are computed
    // before the wait, so the other CTAs' arrival overlaps that work.
    cluster_arrive();
    if (np > 0) {
      if constexpr (!kWide) {
#pragma unroll
        for (int i = 0; i < UMAX; ++i) q1[i] = ld16_shared(sm + c_off[i]);
      }
      if constexpr (kWide) {
        // b in q0; each plane leaves its c there for the next.
        for (int p = 0; p < np; ++p) plane_step(p, q0, q1, q0);
      } else {
        for (int p = 0; p < np; p += 3) {
          plane_step(p, q0, q1, q2);
          if (p + 1 >= np) break;
          plane_step(p + 1, q1, q2, q0);
          if (p + 2 >= np) break;
          plane_step(p + 2, q2, q0, q1);
        }
      }
    } else {
      cluster_wait();
    }
    if (rank == 0 && tid == 0)
      *reinterpret_cast<volatile int*>(steps_done + g) = s + 1;
    cluster_arrive();  // this step's planes are written
  }
  cluster_wait();
  __syncthreads();
  // Store the slab: the first nx floats of each row.
  {
    const int nrow = np * yn;
    for (int r = tid >> 5; r < nrow; r += NT / 32) {
      const int zz = r / yn, yy = r - zz * yn;
      float* o = d.out + ((size_t)(z0 + zz) * ny + y0 + yy) * nx;
      const float* in = sm + zz * plane + (yy + hrow) * px;
      for (int x = lane; x < nx; x += 32) o[x] = in[x];
    }
  }
}

template <int NT, int UMAX, bool PARTS>
__global__ void __launch_bounds__(NT, (NT < 512 ? 512 / NT : 1))
    resident_kernel(const ResidentDesc* __restrict__ descs, int ngrids,
                    unsigned* __restrict__ queue,
                    int* __restrict__ steps_done) {
  extern __shared__ __align__(16) float sm[];
  __shared__ int next_grid;
  const unsigned rank = cluster_rank();
  for (;;) {
    if (rank == 0 && threadIdx.x == 0)
      next_grid = (int)atomicAdd(queue, 1u);
    cluster_sync_all();
    const int g = rank == 0 ? next_grid
                            : ld_cluster_s32(map_to_rank(
                                  smem_u32(&next_grid), 0));
    cluster_sync_all();  // everyone has read it before rank 0 rewrites it
    if (g >= ngrids) break;
    resident_grid<NT, UMAX, PARTS>(descs[g], rank, sm, steps_done,
                            descs[g].grid_id);
  }
}

// (threads, units a thread at most): a plane of S * ny 16-byte segments
// fits variant v when S * ny <= threads * units.
const ResidentVariant kResident[kNumResidentVariants] = {
    {128, 2}, {256, 2}, {512, 2}, {512, 4}, {384, 6}};

template <int NT, int UMAX, bool PARTS>
cudaError_t launch_v(const ResidentDesc* descs, int ngrids, unsigned* queue,
                     int* steps_done, int cluster, int nclusters,
                     size_t smem, cudaStream_t s) {
  auto kern = resident_kernel<NT, UMAX, PARTS>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nclusters * cluster));
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, descs, ngrids, queue, steps_done);
}

template <int NT, int UMAX, bool PARTS>
cudaError_t prepare_v() {
  auto kern = resident_kernel<NT, UMAX, PARTS>;
  cudaError_t e = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)kResidentSmemMax);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(
      kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

template <int NT, int UMAX, bool PARTS>
cudaError_t max_clusters_v(int cluster, size_t smem, int* out) {
  auto kern = resident_kernel<NT, UMAX, PARTS>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cluster);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaOccupancyMaxActiveClusters(out, kern, &cfg);
}

__global__ void set_counters_kernel(const int2* __restrict__ id_steps, int n,
                                    int* __restrict__ counters) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    counters[id_steps[i].x] = id_steps[i].y;
}

}  // namespace

const ResidentVariant& resident_variant(int v) {
  return kResident[v % kResidentParts];
}

bool resident_fit(int nx, int ny, int nz, ResidentFit* fit) {
  const int px = (nx + 3) / 4 * 4, segs = px / 4;
  // Candidates in order of preference: the narrow thread shapes (2 units a
  // thread; 128 and 256 threads take a share of the SM's shared memory so
  // that 512 threads run on an SM and one CTA's barrier waits overlap
  // another's work) with whole planes, then with planes cut into 2 or 4
  // row parts (each CTA holds its rows plus one halo row on each side); the
  // wide shapes (4 and 6 units a thread, whole planes) last.  The first
  // that covers a CTA's plane and needs at most 16 CTAs wins.  (On B200 the
  // wide shapes ran 80^3 at 450 Gpt/s against 710 for 64^3 on the 512-thread
  // narrow shape; a 256-thread shape with 4 units at half an SM measured
  // slower than 512 threads with 2 at a whole SM.)
  struct Cand {
    int v, yparts;
  };
  static const Cand cands[] = {{0, 1}, {1, 1}, {2, 1}, {0, 2}, {1, 2},
                               {2, 2}, {0, 4}, {1, 4}, {2, 4}, {3, 1},
                               {4, 1}};
  for (const Cand& cd : cands) {
    const ResidentVariant& rv = kResident[cd.v];
    if (cd.yparts > 1 && ny < 8 * cd.yparts) continue;
    const int rows = (ny + cd.yparts - 1) / cd.yparts;
    const long long units = (long long)segs * rows;
    if (units > (long long)rv.threads * rv.units) continue;
    const long long plane = (long long)px * (rows + (cd.yparts > 1 ? 2 : 0));
    const int per_sm = std::max(1, 512 / rv.threads);
    const size_t cap =
        std::min(kResidentSmemMax, (size_t)(233472 / per_sm) - 1024);
    const long long pmax = (long long)(cap / 4) / plane - 1;
    if (pmax < 1) continue;
    const int zparts = (int)((nz + pmax - 1) / pmax);
    if (zparts * cd.yparts > kResidentMaxCluster) continue;
    fit->cluster = zparts * cd.yparts;
    fit->variant = cd.v + (cd.yparts > 1 ? kResidentParts : 0);
    fit->yparts = cd.yparts;
    fit->rows = rows;
    fit->pc = (nz + zparts - 1) / zparts;
    fit->smem = (size_t)((fit->pc + 1) * plane * 4);
    fit->px = px;
    return true;
  }
  return false;
}

cudaError_t launch_set_counters(const int2* id_steps, int n, int* counters,
                                cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int blocks = std::min((n + 255) / 256, 148);
  set_counters_kernel<<<blocks, 256, 0, s>>>(id_steps, n, counters);
  return cudaGetLastError();
}

cudaError_t resident_prepare() {
  static int done_dev = -1;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (done_dev == dev) return cudaSuccess;
  if ((e = prepare_v<128, 2, false>()) != cudaSuccess) return e;
  if ((e = prepare_v<256, 2, false>()) != cudaSuccess) return e;
  if ((e = prepare_v<512, 2, false>()) != cudaSuccess) return e;
  if ((e = prepare_v<512, 4, false>()) != cudaSuccess) return e;
  if ((e = prepare_v<384, 6, false>()) != cudaSuccess) return e;
  if ((e = prepare_v<128, 2, true>()) != cudaSuccess) return e;
  if ((e = prepare_v<256, 2, true>()) != cudaSuccess) return e;
  if ((e = prepare_v<512, 2, true>()) != cudaSuccess) return e;
  done_dev = dev;
  return cudaSuccess;
}

cudaError_t resident_max_clusters(int variant, int cluster, size_t smem,
                                  int* out) {
  *out = 0;
  switch (variant) {
    case 0: return max_clusters_v<128, 2, false>(cluster, smem, out);
    case 1: return max_clusters_v<256, 2, false>(cluster, smem, out);
    case 2: return max_clusters_v<512, 2, false>(cluster, smem, out);
    case 3: return max_clusters_v<512, 4, false>(cluster, smem, out);
    case 4: return max_clusters_v<384, 6, false>(cluster, smem, out);
    case kResidentParts + 0: return max_clusters_v<128, 2, true>(cluster, smem, out);
    case kResidentParts + 1: return max_clusters_v<256, 2, true>(cluster, smem, out);
    case kResidentParts + 2: return max_clusters_v<512, 2, true>(cluster, smem, out);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_resident(int variant, const ResidentDesc* descs,
                            int ngrids, unsigned* queue, int* steps_done,
                            int cluster, int nclusters, size_t smem,
                            cudaStream_t s) {
  if (ngrids <= 0 || nclusters <= 0) return cudaSuccess;
  if (cluster < 1 || cluster > kResidentMaxCluster ||
      smem > kResidentSmemMax)
    return cudaErrorInvalidValue;
  switch (variant) {
    case 0: return launch_v<128, 2, false>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    case 1: return launch_v<256, 2, false>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    case 2: return launch_v<512, 2, false>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    case 3: return launch_v<512, 4, false>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    case 4: return launch_v<384, 6, false>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    case kResidentParts + 0: return launch_v<128, 2, true>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    case kResidentParts + 1: return launch_v<256, 2, true>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    case kResidentParts + 2: return launch_v<512, 2, true>(descs, ngrids, queue, steps_done, cluster, nclusters, smem, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace d3d
