// Batched solves: many independent FP32 grids advanced together.
//
// The reference runs one grid per process (Diffusion3DCUDA::RunKernel,
// diffusion3d_cuda.cu:353-371).  Here a batch of grids of different shapes,
// coefficients and step counts is advanced by one multi-grid step kernel
// per time step; all steps of a run are captured once into a CUDA graph and
// replayed as a single graph launch.
//
// Work list.  Grids are split into size classes by nx; each class has one
// kernel kind, picked by the autotuner from six: the march kernel below
// with one of four tile shapes (BX x BY, 256 threads) on the caller's dense
// fields, or the strip form of the pitched TMA kernel (d3d_pitched.cu, 1 or
// 2 row segments a thread) on pitched copies of the fields.  Within a
// class, grids are sorted by step count (descending) and every grid
// contributes one work item per xy tile (or strip), so the items still
// active at step s are a prefix of the class's list: step s launches
// exactly that prefix.  Pitched copies are filled from the caller's inputs
// at the start of the graph and the results written back at its end, one
// multi-grid repitch launch each way.
//
// March kernel: d3d::march_tile (d3d_march.cuh) over one z slab of the
// item's grid (the batch API uses one slab of all nz planes; the solve
// server's march option cuts large grids into several).  Each point is
// d3d::point: results are bit-identical to running each grid alone.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

#include "d3d_b200.h"
#include "d3d_common.cuh"
#include "d3d_kernels.h"
#include "d3d_march.cuh"

namespace d3d {

// PAIR: two cells per thread with packed arithmetic (march_tile2);
// otherwise one cell per thread (march_tile).
template <int BX, int BY, bool PAIR>
__global__ void __launch_bounds__(256)
    batch_step_kernel(const BatchDesc* __restrict__ descs,
                      const int2* __restrict__ items, int parity) {
  using TileT =
      std::conditional_t<PAIR, MarchTile2<BX, BY>, MarchTile<BX, BY>>;
  __shared__ __align__(16) float stage[2][TileT::E];
  const int2 it = items[blockIdx.x];
  const BatchDesc d = descs[it.x];
  const int txy = it.y % d.tiles_xy, zs = it.y / d.tiles_xy;
  const int bx = txy % d.tiles_x, by = txy / d.tiles_x;
  const int z0 = zs * d.zc, z1 = min(d.nz, z0 + d.zc);
  const float* src = parity ? d.b : d.a;
  float* dst = parity ? d.a : d.b;
  const Coef<float> k{d.k[0], d.k[1], d.k[2], d.k[3],
                      d.k[4], d.k[5], d.k[6], d.k[7]};
  if constexpr (PAIR)
    march_tile2<BX, BY>(src, dst, d.nx, d.ny, d.nz, bx * BX, by * BY, z0,
                        z1, k, stage);
  else
    march_tile<float, BX, BY>(src, dst, d.nx, d.ny, d.nz, bx * BX, by * BY,
                              z0, z1, k, stage);
}

// Shape 0 (32 x 16 cells as x-pairs) is the default, the autotuner's pick
// for every size class of the 16..96 batch on B200; it may pick another per
// class.
const BShape kBShapes[kNumBShapes] = {{32, 16}, {64, 8}, {32, 8}, {16, 16}};

cudaError_t launch_batch_step(int shape, const BatchDesc* descs,
                              const int2* items, int nitems, int parity,
                              cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  switch (shape) {
    case 0: batch_step_kernel<32, 16, true><<<nitems, 256, 0, s>>>(descs, items, parity); break;
    case 1: batch_step_kernel<64, 8, true><<<nitems, 256, 0, s>>>(descs, items, parity); break;
    case 2: batch_step_kernel<32, 8, false><<<nitems, 256, 0, s>>>(descs, items, parity); break;
    case 3: batch_step_kernel<16, 16, false><<<nitems, 256, 0, s>>>(descs, items, parity); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace d3d

// ---------------------------------------------------------------------------
// Host side of the batch API (C ABI in include/d3d_b200.h)
// ---------------------------------------------------------------------------
namespace {

using d3d::BatchDesc;
using d3d::kBShapes;
using d3d::kNumBShapes;
using d3d::PitchedDesc;

// Size classes by nx; the autotuner picks one kernel kind per class.
constexpr int kNumClasses = 4;
int class_of(int nx) {
  if (nx <= 24) return 0;
  if (nx <= 40) return 1;
  if (nx <= 72) return 2;
  return 3;
}

// Kernel kinds: 0..3 the march kernel's tile shapes (kBShapes) on the
// caller's dense fields; 4 and 5 the strip form of the pitched TMA kernel
// (1 or 2 segments a thread) on the batch's pitched copies; 6 and 7 its
// two-step form (temporal-block depth 2: fused step pairs, then one strip
// step for an odd step count), for classes whose grids are at most
// d3d::kStripMaxW floats wide.
constexpr int kStripKind = kNumBShapes;
constexpr int kStrip2Kind = kStripKind + 2;
// Kind 8 is batch-wide: every grid that fits runs on the cluster-resident
// kernel (d3d_resident.cu); the rest keep per-class kinds 0..7.
constexpr int kResidentKind = kStrip2Kind + 2;
constexpr int kNumKinds = kResidentKind + 1;
constexpr int kDefaultKind = kStripKind;  // before the autotuner runs
int kind_nr(int kind) {
  return kind >= kStrip2Kind ? kind - kStrip2Kind + 1
         : kind >= kStripKind ? kind - kStripKind + 1
                              : 0;
}
bool kind_two(int kind) { return kind >= kStrip2Kind; }

// One launch of the cluster-resident kernel: grids of one cluster size and
// thread shape, largest work first.
struct ResidentClass {
  int cluster = 1, variant = 0, nclusters = 0;
  size_t smem = 0;
  std::vector<int> grids;
  d3d::ResidentDesc* d_descs = nullptr;
  unsigned* d_queue = nullptr;
};
constexpr int kSideStreams = 4;

struct ClassPlan {
  std::vector<int> grids;  // batch indices, sorted by steps descending
  int kind = 0;
  int max_steps = 0;
  // Launch j (a step, or for two-step kinds a fused pair) covers the first
  // active[j] items.
  std::vector<int> active;
  void* d_descs = nullptr;  // BatchDesc or PitchedDesc, by kind
  int2* d_items = nullptr;
  int nitems = 0;
  // Two-step kinds: the single strip step of grids with an odd step count,
  // after pass j: items [one_lo[j], one_lo[j] + one_n[j]) of d_items1.
  PitchedDesc* d_descs1 = nullptr;
  int2* d_items1 = nullptr;
  std::vector<int> one_lo, one_n;
};

}  // namespace

struct d3d_batch_s {
  std::vector<d3d_batch_grid> grids;
  float* arena = nullptr;
  size_t arena_bytes = 0;
  int max_steps = 0;
  ClassPlan cls[kNumClasses];
  // Pitched copies (rows of ceil4(nx) floats) for strip-kind classes, and
  // the repitch lists that move those grids' inputs in and results out.
  float* pitched = nullptr;
  std::vector<unsigned long long> poff;  // per grid: pitched a; b follows
  d3d::RepitchDesc* d_rep_in = nullptr;
  d3d::RepitchDesc* d_rep_out = nullptr;
  int n_rep = 0;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capture_stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int device = 0;
  long long total_items = 0;
  unsigned long long launches_per_run = 0;
  // Cluster-resident kernel: which grids fit it, whether it is in use, its
  // launches, the per-grid step counters, and the side streams its
  // launches run on (forked from and joined back to the run's stream).
  std::vector<char> resident_ok;
  std::vector<d3d::ResidentDesc> rdesc;  // per grid (resident_ok ones)
  std::vector<int> rclass_of;            // per grid: index into rclasses
  std::vector<ResidentClass> rclasses;
  bool resident_on = false;
  // Only classes of at most this many CTAs a cluster run resident; the
  // larger grids keep the per-step kinds (the autotuner picks the bound).
  int res_max_cluster = d3d::kResidentMaxCluster;
  int* d_counters = nullptr;
  int2* d_classic_steps = nullptr;  // (grid, steps) of the per-step grids
  int n_classic = 0;
  cudaStream_t side[kSideStreams] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kSideStreams] = {};
};

namespace {

int bfail(int code, const char* msg) { return d3d::set_error(code, "%s", msg); }

int bcuda(cudaError_t e, const char* what) {
  return d3d::set_cuda_error(e, what);
}

#define B_TRY(call, what)                            \
  do {                                               \
    cudaError_t e__ = (call);                        \
    if (e__ != cudaSuccess) return bcuda(e__, what); \
  } while (0)

int pitch_of(int nx) { return (nx + 3) / 4 * 4; }
unsigned long long pitched_elems(const d3d_batch_grid& g) {
  const unsigned long long e = (unsigned long long)pitch_of(g.nx) * g.ny * g.nz;
  return (e + 63) / 64 * 64;  // 256-byte aligned buffers
}
float* pitched_buf(d3d_batch b, int gi, int which) {
  return b->pitched + b->poff[gi] + (which ? pitched_elems(b->grids[gi]) : 0);
}

// Whether every grid of a class fits the two-step form.
bool class_takes_two_step(const d3d_batch b, const ClassPlan& c) {
  for (int id : c.grids)
    if (pitch_of(b->grids[id].nx) > d3d::kStripMaxW) return false;
  return true;
}

// A strip-form descriptor of grid `id` (boxes of `rows + extra` rows).
int strip_desc(d3d_batch b, int id, const d3d::StripShape& sh, int extra,
               PitchedDesc* d) {
  const d3d_batch_grid& g = b->grids[id];
  const int px = pitch_of(g.nx);
  memset(d, 0, sizeof *d);
  d->a = pitched_buf(b, id, 0);
  d->b = pitched_buf(b, id, 1);
  for (int m = 0; m < 2; ++m) {
    cudaError_t e = d3d::encode_field_map(&d->map[m], m ? d->b : d->a, px,
                                          g.ny, g.nz, d3d::kF32,
                                          4 * sh.segs + 8, sh.rows + extra);
    if (e != cudaSuccess) return bcuda(e, "tensor map of a batch grid");
  }
  d->nx = g.nx;
  d->px = px;
  d->ny = g.ny;
  d->nz = g.nz;
  d->tiles_x = sh.pieces;
  d->tiles_xy = sh.pieces * ((g.ny + sh.rows - 1) / sh.rows);
  d->zc = g.nz;  // one slab: batches bring parallelism in grid count
  d->seg_w = sh.segs;
  d->rows = sh.rows;
  for (int j = 0; j < 7; ++j) d->k[j] = g.coeff[j];
  d->k[7] = -0.0f;
  return D3D_OK;
}

template <typename T>
int upload(const std::vector<T>& v, T** out, const char* what) {
  *out = nullptr;
  if (v.empty()) return D3D_OK;
  B_TRY(cudaMalloc(out, v.size() * sizeof(T)), what);
  B_TRY(cudaMemcpy(*out, v.data(), v.size() * sizeof(T),
                   cudaMemcpyHostToDevice),
        what);
  return D3D_OK;
}

void free_class(ClassPlan& c) {
  if (c.d_descs) cudaFree(c.d_descs);
  if (c.d_items) cudaFree(c.d_items);
  if (c.d_descs1) cudaFree(c.d_descs1);
  if (c.d_items1) cudaFree(c.d_items1);
  c.d_descs = nullptr;
  c.d_items = nullptr;
  c.d_descs1 = nullptr;
  c.d_items1 = nullptr;
}

// (Re)builds one class's descriptors and item lists for its current kind.
int build_class(d3d_batch b, ClassPlan& c) {
  free_class(c);
  const bool two = kind_two(c.kind);
  const int nr = kind_nr(c.kind);
  const int nlaunch = two ? c.max_steps / 2 : c.max_steps;
  c.active.assign(nlaunch, 0);
  c.one_lo.assign(c.max_steps / 2 + 1, 0);
  c.one_n.assign(c.max_steps / 2 + 1, 0);
  c.nitems = 0;
  if (c.grids.empty()) return D3D_OK;
  std::vector<BatchDesc> descs;
  std::vector<PitchedDesc> pdescs, pdescs1;
  std::vector<int2> items, items1;
  for (size_t gi = 0; gi < c.grids.size(); ++gi) {
    const int id = c.grids[gi];
    const d3d_batch_grid& g = b->grids[id];
    int tiles;
    if (two) {
      const int px = pitch_of(g.nx);
      PitchedDesc d, d1;
      int rc = strip_desc(b, id, d3d::strip2_shape(px, g.ny, nr), 4, &d);
      if (rc) return rc;
      rc = strip_desc(b, id, d3d::strip_shape(px, g.ny, 1), 2, &d1);
      if (rc) return rc;
      pdescs.push_back(d);
      pdescs1.push_back(d1);
      tiles = d.tiles_xy;
      if (g.steps & 1) {
        const int j = g.steps / 2;
        if (c.one_n[j] == 0) c.one_lo[j] = (int)items1.size();
        for (int t = 0; t < d1.tiles_xy; ++t)
          items1.push_back(make_int2((int)gi, t));
        c.one_n[j] += d1.tiles_xy;
      }
    } else if (nr) {
      PitchedDesc d;
      int rc = strip_desc(b, id, d3d::strip_shape(pitch_of(g.nx), g.ny, nr),
                          2, &d);
      if (rc) return rc;
      pdescs.push_back(d);
      tiles = d.tiles_xy;
    } else {
      const d3d::BShape sh = kBShapes[c.kind];
      BatchDesc d;
      d.a = b->arena + g.offset_a;
      d.b = b->arena + g.offset_b;
      d.nx = g.nx;
      d.ny = g.ny;
      d.nz = g.nz;
      d.tiles_x = (g.nx + sh.bx - 1) / sh.bx;
      d.tiles_xy = d.tiles_x * ((g.ny + sh.by - 1) / sh.by);
      d.zc = g.nz;
      for (int j = 0; j < 7; ++j) d.k[j] = g.coeff[j];
      d.k[7] = -0.0f;
      tiles = d.tiles_xy;
      descs.push_back(d);
    }
    for (int t = 0; t < tiles; ++t) items.push_back(make_int2((int)gi, t));
    // this grid's items are in launches [0, steps) (pairs: [0, steps/2))
    const int nl = two ? g.steps / 2 : g.steps;
    for (int j = 0; j < nl; ++j) c.active[j] += tiles;
  }
  c.nitems = (int)items.size();
  int rc;
  if (nr) {
    PitchedDesc* d = nullptr;
    rc = upload(pdescs, &d, "batch descriptors");
    c.d_descs = d;
  } else {
    BatchDesc* d = nullptr;
    rc = upload(descs, &d, "batch descriptors");
    c.d_descs = d;
  }
  if (!rc) rc = upload(items, &c.d_items, "batch items");
  if (!rc) rc = upload(pdescs1, &c.d_descs1, "batch descriptors");
  if (!rc) rc = upload(items1, &c.d_items1, "batch items");
  return rc;
}

// The pitched buffer (0: a, 1: b) holding grid `g`'s result under a kind:
// one step swaps the buffers, a fused pair swaps them once.
int result_buffer(const d3d_batch_grid& g, int kind) {
  const int swaps = kind_two(kind) ? g.steps / 2 + (g.steps & 1) : g.steps;
  return swaps & 1;
}

// The repitch lists of every grid (steps > 0) in a strip-kind class.
int build_repitch(d3d_batch b) {
  if (b->d_rep_in) cudaFree(b->d_rep_in);
  if (b->d_rep_out) cudaFree(b->d_rep_out);
  b->d_rep_in = b->d_rep_out = nullptr;
  b->n_rep = 0;
  std::vector<d3d::RepitchDesc> in, out;
  for (const ClassPlan& c : b->cls) {
    if (!kind_nr(c.kind)) continue;
    for (int id : c.grids) {
      const d3d_batch_grid& g = b->grids[id];
      if (g.steps == 0) continue;  // its result is its input
      const long long rows = (long long)g.ny * g.nz;
      in.push_back({b->arena + g.offset_a, pitched_buf(b, id, 0), g.nx,
                    pitch_of(g.nx), rows});
      out.push_back({b->arena + ((g.steps & 1) ? g.offset_b : g.offset_a),
                     pitched_buf(b, id, result_buffer(g, c.kind)), g.nx,
                     pitch_of(g.nx), rows});
    }
  }
  if (in.empty()) return D3D_OK;
  const size_t bytes = in.size() * sizeof(d3d::RepitchDesc);
  B_TRY(cudaMalloc(&b->d_rep_in, bytes), "cudaMalloc (repitch lists)");
  B_TRY(cudaMalloc(&b->d_rep_out, bytes), "cudaMalloc (repitch lists)");
  B_TRY(cudaMemcpy(b->d_rep_in, in.data(), bytes, cudaMemcpyHostToDevice),
        "H2D repitch lists");
  B_TRY(cudaMemcpy(b->d_rep_out, out.data(), bytes, cudaMemcpyHostToDevice),
        "H2D repitch lists");
  b->n_rep = (int)in.size();
  return D3D_OK;
}

cudaError_t launch_class_step(const ClassPlan& c, int nitems, int parity,
                              cudaStream_t s) {
  const int nr = kind_nr(c.kind);
  if (kind_two(c.kind))
    return d3d::launch_pitched_strip2(
        nr, static_cast<const PitchedDesc*>(c.d_descs), c.d_items, nitems,
        parity, s, d3d::device_error_word());
  if (nr)
    return d3d::launch_pitched_strip(
        nr, static_cast<const PitchedDesc*>(c.d_descs), c.d_items, nitems,
        parity, s, d3d::device_error_word());
  return d3d::launch_batch_step(c.kind,
                                static_cast<const BatchDesc*>(c.d_descs),
                                c.d_items, nitems, parity, s);
}

// All steps of all classes, in step order (class launches of one step are
// independent; steps depend on each other through the stream order).
int enqueue_run(d3d_batch b, cudaStream_t s, int only_class, int max_steps,
                unsigned long long* launches) {
  unsigned long long n = 0;
  for (int step = 0; step < max_steps; ++step) {
    for (int ci = 0; ci < kNumClasses; ++ci) {
      if (only_class >= 0 && ci != only_class) continue;
      ClassPlan& c = b->cls[ci];
      if (step >= c.max_steps) continue;
      if (kind_two(c.kind)) {
        // Pair j = step / 2 at even steps, then the odd grids' last step.
        if (step & 1) continue;
        const int j = step / 2;
        if (j < (int)c.active.size() && c.active[j] > 0) {
          B_TRY(launch_class_step(c, c.active[j], j & 1, s),
                "batch step launch");
          ++n;
        }
        if (c.one_n[j] > 0) {
          B_TRY(d3d::launch_pitched_strip(1, c.d_descs1,
                                          c.d_items1 + c.one_lo[j],
                                          c.one_n[j], j & 1, s,
                                          d3d::device_error_word()),
                "batch step launch");
          ++n;
        }
        continue;
      }
      if (c.active[step] == 0) continue;
      B_TRY(launch_class_step(c, c.active[step], step & 1, s),
            "batch step launch");
      ++n;
    }
  }
  if (launches) *launches = n;
  return D3D_OK;
}

void drop_graph(d3d_batch b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
}

// Which grids fit the cluster-resident kernel, and its launch classes:
// a grid with S = ceil(nx/4) row segments fits when a thread shape covers
// its S * ny segments a plane and a cluster of at most 16 CTAs holds its
// nz planes, pc a CTA plus one halo plane, in the shared memory a CTA may
// have.  Grids with 0 steps are their own result and never run.
int plan_resident(d3d_batch b) {
  const int n = (int)b->grids.size();
  b->resident_ok.assign(n, 0);
  b->rdesc.assign(n, d3d::ResidentDesc{});
  b->rclass_of.assign(n, -1);
  b->rclasses.clear();
  cudaError_t e = d3d::resident_prepare();
  if (e != cudaSuccess) {
    // Without the kernel's attributes every grid keeps the per-step kinds.
    cudaGetLastError();
    return D3D_OK;
  }
  std::vector<std::pair<int, int>> keys;  // (cluster, variant)
  for (int i = 0; i < n; ++i) {
    const d3d_batch_grid& g = b->grids[i];
    if (g.steps < 1) continue;
    d3d::ResidentFit fit;
    if (!d3d::resident_fit(g.nx, g.ny, g.nz, &fit)) continue;
    const int px = fit.px, segs = px / 4, cl = fit.cluster, v = fit.variant;
    const int pc = fit.pc;
    d3d::ResidentDesc& d = b->rdesc[i];
    d.in = b->arena + g.offset_a;
    d.out = b->arena + ((g.steps & 1) ? g.offset_b : g.offset_a);
    d.nx = g.nx;
    d.ny = g.ny;
    d.nz = g.nz;
    d.steps = g.steps;
    d.px = px;
    d.segs = segs;
    d.pc = pc;
    d.grid_id = i;
    d.yparts = fit.yparts;
    d.rows = fit.rows;
    for (int j = 0; j < 7; ++j) d.k[j] = g.coeff[j];
    d.k[7] = -0.0f;
    const std::pair<int, int> key(cl, v);
    int ci = -1;
    for (size_t j = 0; j < keys.size(); ++j)
      if (keys[j] == key) ci = (int)j;
    if (ci < 0) {
      ci = (int)keys.size();
      keys.push_back(key);
      b->rclasses.emplace_back();
      b->rclasses.back().cluster = cl;
      b->rclasses.back().variant = v;
    }
    ResidentClass& rc = b->rclasses[ci];
    rc.grids.push_back(i);
    rc.smem = std::max(rc.smem, fit.smem);
    b->rclass_of[i] = ci;
    b->resident_ok[i] = 1;
  }
  // Classes the GPU cannot schedule (no cluster of that size and shared
  // memory fits) hand their grids back to the per-step kinds.
  for (size_t ci = 0; ci < b->rclasses.size(); ++ci) {
    ResidentClass& rc = b->rclasses[ci];
    int maxc = 0;
    if (d3d::resident_max_clusters(rc.variant, rc.cluster, rc.smem,
                                   &maxc) != cudaSuccess) {
      cudaGetLastError();
      maxc = 0;
    }
    rc.nclusters = std::min<int>(maxc, (int)rc.grids.size());
    if (rc.nclusters < 1)
      for (int id : rc.grids) b->resident_ok[id] = 0;
  }
  std::vector<ResidentClass> kept;
  for (ResidentClass& rc : b->rclasses)
    if (rc.nclusters >= 1) kept.push_back(std::move(rc));
  b->rclasses = std::move(kept);
  for (size_t ci = 0; ci < b->rclasses.size(); ++ci) {
    ResidentClass& rc = b->rclasses[ci];
    // Largest work first: the last grids to start are the shortest.
    std::stable_sort(rc.grids.begin(), rc.grids.end(), [&](int x, int y) {
      const d3d_batch_grid &gx = b->grids[x], &gy = b->grids[y];
      return (double)gx.nx * gx.ny * gx.nz * gx.steps >
             (double)gy.nx * gy.ny * gy.nz * gy.steps;
    });
    std::vector<d3d::ResidentDesc> descs;
    for (int id : rc.grids) {
      descs.push_back(b->rdesc[id]);
      b->rclass_of[id] = (int)ci;
    }
    int r = upload(descs, &rc.d_descs, "resident descriptors");
    if (r) return r;
    B_TRY(cudaMalloc(&rc.d_queue, sizeof(unsigned)),
          "cudaMalloc (resident work counter)");
  }
  return D3D_OK;
}

void free_resident(d3d_batch b) {
  for (ResidentClass& rc : b->rclasses) {
    if (rc.d_descs) cudaFree(rc.d_descs);
    if (rc.d_queue) cudaFree(rc.d_queue);
    rc.d_descs = nullptr;
    rc.d_queue = nullptr;
  }
}

// Puts every grid (steps >= 0) into its size class, leaving out the grids
// the cluster-resident kernel runs when it is on, and rebuilds the classes'
// work lists and the repitch lists.
bool runs_resident(const d3d_batch b, int i) {
  return b->resident_on && b->resident_ok[i] &&
         b->rclasses[b->rclass_of[i]].cluster <= b->res_max_cluster;
}

bool class_resident(const d3d_batch b, const ResidentClass& rc) {
  return b->resident_on && rc.cluster <= b->res_max_cluster;
}

int assign_grids(d3d_batch b) {
  for (ClassPlan& c : b->cls) {
    c.grids.clear();
    c.max_steps = 0;
  }
  b->max_steps = 0;
  std::vector<int2> classic;
  for (int i = 0; i < (int)b->grids.size(); ++i) {
    if (runs_resident(b, i)) continue;
    ClassPlan& c = b->cls[class_of(b->grids[i].nx)];
    c.grids.push_back(i);
    c.max_steps = std::max(c.max_steps, b->grids[i].steps);
    b->max_steps = std::max(b->max_steps, b->grids[i].steps);
    classic.push_back(make_int2(i, b->grids[i].steps));
  }
  b->total_items = 0;
  for (ClassPlan& c : b->cls) {
    std::stable_sort(c.grids.begin(), c.grids.end(), [&](int x, int y) {
      return b->grids[x].steps > b->grids[y].steps;
    });
    int rc = build_class(b, c);
    if (rc) return rc;
    for (int a : c.active) b->total_items += a;
  }
  if (b->d_classic_steps) cudaFree(b->d_classic_steps);
  b->d_classic_steps = nullptr;
  b->n_classic = (int)classic.size();
  int rc = upload(classic, &b->d_classic_steps, "batch step counts");
  if (rc) return rc;
  return build_repitch(b);
}

// A whole run on stream s: the cluster-resident launches on side streams
// forked from s, the per-step launches of the other grids on s meanwhile,
// then s waits for the side streams.  Every grid's step counter is zeroed
// first; the resident kernel advances its grids' counters step by step,
// and one small launch after the per-step path sets the other grids'.
int enqueue_all(d3d_batch b, cudaStream_t s, unsigned long long* launches) {
  unsigned long long n = 0;
  B_TRY(cudaMemsetAsync(b->d_counters, 0, b->grids.size() * sizeof(int), s),
        "counter reset");
  bool used[kSideStreams] = {};
  if (b->resident_on && !b->rclasses.empty()) {
    B_TRY(cudaEventRecord(b->fork, s), "cudaEventRecord (fork)");
    for (size_t ci = 0, li = 0; ci < b->rclasses.size(); ++ci) {
      const ResidentClass& rc = b->rclasses[ci];
      if (!class_resident(b, rc)) continue;
      const int k = (int)(li++ % kSideStreams);
      if (!used[k]) {
        B_TRY(cudaStreamWaitEvent(b->side[k], b->fork, 0),
              "cudaStreamWaitEvent (fork)");
        used[k] = true;
      }
      B_TRY(cudaMemsetAsync(rc.d_queue, 0, sizeof(unsigned), b->side[k]),
            "work counter reset");
      B_TRY(d3d::launch_resident(rc.variant, rc.d_descs,
                                 (int)rc.grids.size(), rc.d_queue,
                                 b->d_counters, rc.cluster, rc.nclusters,
                                 rc.smem, b->side[k]),
            "resident launch");
      ++n;
    }
  }
  if (b->n_rep) {
    B_TRY(d3d::launch_repitch_multi(b->d_rep_in, b->n_rep, true, s),
          "repitch launch");
    ++n;
  }
  unsigned long long steps_launched = 0;
  int rc = enqueue_run(b, s, -1, b->max_steps, &steps_launched);
  if (rc) return rc;
  n += steps_launched;
  if (b->n_rep) {
    B_TRY(d3d::launch_repitch_multi(b->d_rep_out, b->n_rep, false, s),
          "repitch launch");
    ++n;
  }
  if (b->n_classic) {
    B_TRY(d3d::launch_set_counters(b->d_classic_steps, b->n_classic,
                                   b->d_counters, s),
          "counter launch");
    ++n;
  }
  for (int k = 0; k < kSideStreams; ++k) {
    if (!used[k]) continue;
    B_TRY(cudaEventRecord(b->join[k], b->side[k]), "cudaEventRecord (join)");
    B_TRY(cudaStreamWaitEvent(s, b->join[k], 0), "cudaStreamWaitEvent");
  }
  if (launches) *launches = n;
  return D3D_OK;
}

}  // namespace

extern "C" {

int d3d_batch_coefficients(int nx, int ny, int nz, float kappa,
                           float coeff7[7]) {
  if (nx < 1 || ny < 1 || nz < 1 || !(kappa > 0.0f) || !coeff7)
    return bfail(D3D_E_INVALID, "bad grid or kappa");
  const float l = 1.0f;
  const float dx = l / nx, dy = l / ny, dz = l / nz;
  const float h = std::min(dx, std::min(dy, dz));
  const float dt = (float)(0.1 * h * h / kappa);
  const float ce = kappa * dt / (dx * dx);
  const float cn = kappa * dt / (dy * dy);
  const float ct = kappa * dt / (dz * dz);
  const float cc = (float)(1.0 - (ce + ce + cn + cn + ct + ct));
  const float c[7] = {ce, ce, cn, cn, ct, ct, cc};
  memcpy(coeff7, c, sizeof c);
  return D3D_OK;
}

int d3d_batch_layout(d3d_batch_grid* grids, int n, size_t* arena_bytes) {
  if (!grids || n < 0 || !arena_bytes) return bfail(D3D_E_INVALID, "NULL");
  unsigned long long off = 0;  // elements
  for (int i = 0; i < n; ++i) {
    const unsigned long long pts =
        (unsigned long long)grids[i].nx * grids[i].ny * grids[i].nz;
    const unsigned long long padded = (pts + 63) / 64 * 64;  // 256 B
    grids[i].offset_a = off;
    grids[i].offset_b = off + padded;
    off += 2 * padded;
  }
  *arena_bytes = (size_t)off * sizeof(float);
  return D3D_OK;
}

int d3d_batch_create(const d3d_batch_grid* grids, int n, void* arena,
                     size_t arena_bytes, d3d_batch* out) {
  if (!grids || n < 1 || !arena || !out)
    return bfail(D3D_E_INVALID, "NULL argument or empty batch");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    const d3d_batch_grid& g = grids[i];
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || g.steps < 0)
      return bfail(D3D_E_INVALID, "bad grid dimensions or steps");
    if (((long long)g.nx + 3) / 4 * 4 * g.ny >= (1LL << 31))
      return bfail(D3D_E_INVALID, "grid plane too large");
    const unsigned long long pts = (unsigned long long)g.nx * g.ny * g.nz;
    if ((g.offset_a + pts) * 4 > arena_bytes ||
        (g.offset_b + pts) * 4 > arena_bytes)
      return bfail(D3D_E_INVALID, "grid buffer outside the arena");
    const unsigned long long a0 = g.offset_a, a1 = g.offset_a + pts;
    const unsigned long long b0 = g.offset_b, b1 = g.offset_b + pts;
    if (a0 < b1 && b0 < a1)
      return bfail(D3D_E_INVALID, "a grid's two buffers overlap");
  }
  d3d_batch b = new (std::nothrow) d3d_batch_s();
  if (!b) return bfail(D3D_E_OOM, "batch allocation");
  b->grids.assign(grids, grids + n);
  b->arena = static_cast<float*>(arena);
  b->arena_bytes = arena_bytes;
  cudaGetDevice(&b->device);
  // Pitched copies for the strip kinds, two buffers per grid.
  b->poff.resize(n);
  unsigned long long pe = 0;
  for (int i = 0; i < n; ++i) {
    b->poff[i] = pe;
    pe += 2 * pitched_elems(grids[i]);
  }
  // Without room for them the batch runs the march kinds only, on the
  // caller's fields.
  if (cudaMalloc(&b->pitched, pe * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    b->pitched = nullptr;
  }
  for (auto& c : b->cls) c.kind = b->pitched ? kDefaultKind : 0;
  int rc = plan_resident(b);
  if (!rc) rc = assign_grids(b);
  if (rc) {
    d3d_batch_destroy(b);
    return rc;
  }
  bool ok = cudaMalloc(&b->d_counters, n * sizeof(int)) == cudaSuccess &&
            cudaMemset(b->d_counters, 0, n * sizeof(int)) == cudaSuccess &&
            cudaEventCreate(&b->ev[0]) == cudaSuccess &&
            cudaEventCreate(&b->ev[1]) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) ==
                cudaSuccess;
  for (int k = 0; ok && k < kSideStreams; ++k)
    ok = cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking) ==
             cudaSuccess &&
         cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) ==
             cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    d3d_batch_destroy(b);
    return bfail(D3D_E_CUDA, "batch streams, events or step counters");
  }
  *out = b;
  return D3D_OK;
}

int d3d_batch_autotune(d3d_batch b, void* stream) {
  if (!b) return bfail(D3D_E_INVALID, "NULL batch");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  drop_graph(b);
  // Per-class kinds are tuned with every grid in its class.
  b->resident_on = false;
  int arc = assign_grids(b);
  if (arc) return arc;
  b->total_items = 0;
  for (int ci = 0; ci < kNumClasses; ++ci) {
    ClassPlan& c = b->cls[ci];
    if (c.grids.empty()) continue;
    const int probe_steps = std::min(c.max_steps, 8);  // pairs count 2
    if (probe_steps == 0) continue;
    float best = -1.0f;
    int best_kind = c.kind;
    for (int kind = 0; kind < kResidentKind; ++kind) {  // per-class kinds
      if (kind_nr(kind) && !b->pitched) continue;
      if (kind_two(kind) && !class_takes_two_step(b, c)) continue;
      c.kind = kind;
      int rc = build_class(b, c);
      if (rc) return rc;
      rc = enqueue_run(b, s, ci, 1, nullptr);  // warm-up
      if (rc) return rc;
      B_TRY(cudaEventRecord(b->ev[0], s), "cudaEventRecord");
      rc = enqueue_run(b, s, ci, probe_steps, nullptr);
      if (rc) return rc;
      B_TRY(cudaEventRecord(b->ev[1], s), "cudaEventRecord");
      B_TRY(cudaEventSynchronize(b->ev[1]), "cudaEventSynchronize");
      float ms = 0.0f;
      B_TRY(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]), "elapsed");
      if (best < 0.0f || ms < best) {
        best = ms;
        best_kind = kind;
      }
    }
    c.kind = best_kind;
    int rc = build_class(b, c);
    if (rc) return rc;
  }
  for (const ClassPlan& c : b->cls)
    for (int a : c.active) b->total_items += a;
  int rc = build_repitch(b);
  if (rc) return rc;
  // Then the whole run without the cluster-resident kernel and with it for
  // the grids it fits in clusters of at most 4, 8, 12 or 16 CTAs (the
  // others keep the kinds just picked): the per-step kinds are HBM-bound
  // and the resident kernel needs SMs but next to no HBM, so a split can
  // beat both ends.
  bool any = false;
  for (char ok : b->resident_ok) any = any || ok;
  if (!any) return D3D_OK;
  static const int bounds[] = {0, 4, 8, 12, d3d::kResidentMaxCluster};
  float times[5];
  for (float& t : times) t = -1.0f;
  for (int bi = 0; bi < 5; ++bi) {
    const int bound = bounds[bi];
    b->resident_on = bound > 0;
    b->res_max_cluster = bound > 0 ? bound : d3d::kResidentMaxCluster;
    if (bound > 0) {  // skip a bound that changes nothing
      bool fresh = false;
      for (const ResidentClass& c : b->rclasses)
        fresh = fresh || (c.cluster <= bound && c.cluster > bound - 4);
      if (!fresh) continue;
    }
    rc = assign_grids(b);
    if (rc) return rc;
    rc = enqueue_all(b, s, nullptr);  // warm-up
    if (rc) return rc;
    B_TRY(cudaEventRecord(b->ev[0], s), "cudaEventRecord");
    rc = enqueue_all(b, s, nullptr);
    if (rc) return rc;
    B_TRY(cudaEventRecord(b->ev[1], s), "cudaEventRecord");
    B_TRY(cudaEventSynchronize(b->ev[1]), "cudaEventSynchronize");
    B_TRY(cudaEventElapsedTime(&times[bi], b->ev[0], b->ev[1]), "elapsed");
  }
  // The fastest, except that a larger bound within 2% of it wins: more
  // grids resident means fewer launches a run (one persistent launch
  // instead of one per step), which costs host time the device timing
  // does not see.  (On B200 the 4096-grid batch ran 310 ms at bound 12
  // with 1008 launches and 314 ms at 16 with 185.)
  float best = -1.0f;
  for (float t : times)
    if (t >= 0.0f && (best < 0.0f || t < best)) best = t;
  int best_bound = 0;
  for (int bi = 0; bi < 5; ++bi)
    if (times[bi] >= 0.0f && times[bi] <= 1.02f * best)
      best_bound = bounds[bi];
  b->resident_on = best_bound > 0;
  b->res_max_cluster =
      best_bound > 0 ? best_bound : d3d::kResidentMaxCluster;
  return assign_grids(b);
}

int d3d_batch_set_kind(d3d_batch b, int kind) {
  if (!b) return bfail(D3D_E_INVALID, "NULL batch");
  if (kind < 0 || kind >= kNumKinds)
    return bfail(D3D_E_INVALID, "no such kernel kind");
  if (kind == kResidentKind) {
    // Every grid the cluster-resident kernel fits runs on it; the others
    // take the strip kind (the march kind without pitched copies).
    drop_graph(b);
    b->resident_on = true;
    b->res_max_cluster = d3d::kResidentMaxCluster;
    for (ClassPlan& c : b->cls) c.kind = b->pitched ? kDefaultKind : 0;
    return assign_grids(b);
  }
  if (kind_nr(kind) && !b->pitched)
    return bfail(D3D_E_UNSUPPORTED,
                 "no device memory was left for the pitched copies");
  if (kind_two(kind))
    for (int i = 0; i < (int)b->grids.size(); ++i)
      if (pitch_of(b->grids[i].nx) > d3d::kStripMaxW)
        return bfail(D3D_E_UNSUPPORTED,
                     "two-step kinds need grids at most 248 floats wide");
  drop_graph(b);
  b->resident_on = false;
  for (ClassPlan& c : b->cls) c.kind = kind;
  return assign_grids(b);
}

int d3d_batch_set_resident_max_cluster(d3d_batch b, int max_cluster) {
  if (!b) return bfail(D3D_E_INVALID, "NULL batch");
  if (max_cluster < 0 || max_cluster > d3d::kResidentMaxCluster)
    return bfail(D3D_E_INVALID, "max_cluster must be 0 to 16");
  drop_graph(b);
  b->resident_on = max_cluster > 0;
  b->res_max_cluster =
      max_cluster > 0 ? max_cluster : d3d::kResidentMaxCluster;
  return assign_grids(b);
}

int d3d_batch_run(d3d_batch b, void* stream, float* kernel_ms) {
  if (!b) return bfail(D3D_E_INVALID, "NULL batch");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != b->device) return bfail(D3D_E_INVALID, "wrong device");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!b->exec) {
    if (!b->capture_stream)
      B_TRY(cudaStreamCreateWithFlags(&b->capture_stream,
                                      cudaStreamNonBlocking),
            "cudaStreamCreateWithFlags");
    B_TRY(cudaStreamBeginCapture(b->capture_stream,
                                 cudaStreamCaptureModeThreadLocal),
          "cudaStreamBeginCapture");
    // The cluster-resident launches (forked), strip-kind grids' inputs
    // into the pitched copies, the per-step launches, results back into
    // the caller's arena, the step counters; then the join.
    unsigned long long launched = 0;
    int rc = enqueue_all(b, b->capture_stream, &launched);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return bcuda(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->exec = nullptr;
      return bcuda(e, "cudaGraphInstantiate");
    }
    b->launches_per_run = launched;
  }
  B_TRY(cudaEventRecord(b->ev[0], s), "cudaEventRecord");
  B_TRY(cudaGraphLaunch(b->exec, s), "cudaGraphLaunch");
  B_TRY(cudaEventRecord(b->ev[1], s), "cudaEventRecord");
  d3d::note_launches(b->launches_per_run);
  if (kernel_ms) {
    B_TRY(cudaEventSynchronize(b->ev[1]), "cudaEventSynchronize");
    B_TRY(cudaEventElapsedTime(kernel_ms, b->ev[0], b->ev[1]), "elapsed");
  }
  return D3D_OK;
}

int d3d_batch_info(d3d_batch b, char* buf, size_t len) {
  if (!b || !buf) return bfail(D3D_E_INVALID, "NULL argument");
  int nres = 0;
  for (const ResidentClass& rc : b->rclasses)
    if (class_resident(b, rc)) nres += (int)rc.grids.size();
  int used = snprintf(buf, len,
                      "{\"grids\": %zu, \"max_steps\": %d, \"items\": %lld, "
                      "\"launches_per_run\": %llu, \"resident\": "
                      "{\"on\": %s, \"max_cluster\": %d, \"grids\": %d, "
                      "\"classes\": [",
                      b->grids.size(), b->max_steps, b->total_items,
                      b->launches_per_run,
                      b->resident_on ? "true" : "false", b->res_max_cluster,
                      nres);
  for (size_t ci = 0, shown = 0; ci < b->rclasses.size() && used < (int)len;
       ++ci) {
    const ResidentClass& rc = b->rclasses[ci];
    if (!class_resident(b, rc)) continue;
    used += snprintf(buf + used, len - used,
                     "%s{\"cluster\": %d, \"threads\": %d, \"grids\": "
                     "%zu, \"clusters\": %d, \"smem\": %zu}",
                     shown++ ? ", " : "", rc.cluster,
                     d3d::resident_variant(rc.variant).threads,
                     rc.grids.size(), rc.nclusters, rc.smem);
  }
  if (used < (int)len)
    used += snprintf(buf + used, len - used, "]}, \"classes\": [");
  for (int ci = 0; ci < kNumClasses && used < (int)len; ++ci) {
    const ClassPlan& c = b->cls[ci];
    const int nr = kind_nr(c.kind);
    if (nr)
      used += snprintf(buf + used, len - used,
                       "%s{\"grids\": %zu, \"kernel\": \"%s\", "
                       "\"segments_per_thread\": %d, \"items\": %d}",
                       ci ? ", " : "", c.grids.size(),
                       kind_two(c.kind) ? "strip2" : "strip", nr, c.nitems);
    else
      used += snprintf(buf + used, len - used,
                       "%s{\"grids\": %zu, \"kernel\": \"march\", "
                       "\"tile\": [%d, %d], \"items\": %d}",
                       ci ? ", " : "", c.grids.size(), kBShapes[c.kind].bx,
                       kBShapes[c.kind].by, c.nitems);
  }
  if (used < (int)len) snprintf(buf + used, len - used, "]}");
  return D3D_OK;
}

int d3d_batch_progress(d3d_batch b, int* steps_done, int n) {
  if (!b || !steps_done) return bfail(D3D_E_INVALID, "NULL argument");
  if (n != (int)b->grids.size())
    return bfail(D3D_E_INVALID, "n must be the batch's grid count");
  B_TRY(cudaMemcpy(steps_done, b->d_counters, (size_t)n * sizeof(int),
                   cudaMemcpyDeviceToHost),
        "D2H step counters");
  return D3D_OK;
}

int d3d_batch_destroy(d3d_batch b) {
  if (!b) return D3D_OK;
  drop_graph(b);
  free_resident(b);
  if (b->d_counters) cudaFree(b->d_counters);
  if (b->d_classic_steps) cudaFree(b->d_classic_steps);
  for (int k = 0; k < kSideStreams; ++k) {
    if (b->side[k]) cudaStreamDestroy(b->side[k]);
    if (b->join[k]) cudaEventDestroy(b->join[k]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  for (auto& c : b->cls) free_class(c);
  if (b->d_rep_in) cudaFree(b->d_rep_in);
  if (b->d_rep_out) cudaFree(b->d_rep_out);
  if (b->pitched) cudaFree(b->pitched);
  if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  if (b->ev[0]) cudaEventDestroy(b->ev[0]);
  if (b->ev[1]) cudaEventDestroy(b->ev[1]);
  delete b;
  return D3D_OK;
}

}  // extern "C"
