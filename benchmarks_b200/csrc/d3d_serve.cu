// Continuous-batching solve server (d3d_server_* in include/d3d_b200.h).
//
// State of a request: queued -> active (its two buffers live in the device
// arena; input copied in on the copy stream) -> retiring (its result is
// being copied to the caller's host buffer) -> done.  A tick advances every
// active solve by up to `chunk` steps with one multi-grid step launch per
// sub-step: within a tick, solves are ordered by steps remaining so the
// ones still stepping at sub-step j are a prefix of the work list, and
// large grids are cut into z slabs so a few big solves still fill the GPU.
// At most two ticks are in flight; their descriptor/work lists use
// alternating staging buffers.
//
// Small solves.  A solve that the cluster-resident kernel fits (its whole
// grid in the shared memory of one cluster of at most 16 CTAs,
// d3d_resident.cu) skips the ticks: it is admitted into one dense buffer,
// and the next tick launches every such solve admitted since the last one
// in one persistent launch per cluster size, which runs all of their steps;
// each result is copied out as soon as that launch ends.
//
// Step kernel.  By default the strip form of the pitched TMA kernel
// (d3d_pitched.cu): each solve is stored with rows padded to a 16-byte
// pitch and read through two tensor maps encoded at admission, whose box
// is the solve's strip (whole rows of up to 248 columns).  Host copies
// stay dense and contiguous (one transfer each way); a device pass spreads
// an input into the pitched layout (filling the pads) and packs a result
// back.  d3d_server_set_kernel picks the tile form instead (0..4) or the
// unpadded march kernel of the batch API (-1).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <tuple>
#include <vector>

#include "d3d_b200.h"
#include "d3d_common.cuh"
#include "d3d_kernels.h"

namespace {

constexpr unsigned long long kAlign = 64;  // elements (256 bytes)
// Kernels 5 and 6: the strip form with 1 or 2 segments a thread.
constexpr int kStripBase = d3d::kNumPitchedVariants;
constexpr int kDefaultKernel = kStripBase + 1;  // strip, 2 segments
constexpr int kMaxKernel = kStripBase + 1;
int strip_nr(int kernel) {
  return kernel >= kStripBase ? kernel - kStripBase + 1 : 0;
}
constexpr int kMaxLanes = 8;               // compute streams
// Step-kernel geometry of a kernel id: strip segments a thread (0 for the
// tile forms and the march kernel) and, for the tile forms and the march
// kernel, the xy tile.
struct KernGeom {
  int nr, bx, by;
};
constexpr int kDefaultLanes = 4;

// First-fit allocator over the arena, in elements.
class ArenaAlloc {
 public:
  void reset(unsigned long long size) {
    free_.clear();
    free_[0] = size;
    used_ = 0;
  }
  bool alloc(unsigned long long n, unsigned long long* off) {
    n = (n + kAlign - 1) / kAlign * kAlign;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        *off = it->first;
        const unsigned long long rest = it->second - n;
        const unsigned long long start = it->first + n;
        free_.erase(it);
        if (rest) free_[start] = rest;
        used_ += n;
        return true;
      }
    }
    return false;
  }
  void release(unsigned long long off, unsigned long long n) {
    n = (n + kAlign - 1) / kAlign * kAlign;
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  unsigned long long used() const { return used_; }

 private:
  std::map<unsigned long long, unsigned long long> free_;
  unsigned long long used_ = 0;
};

struct Request {
  CUtensorMap map[2];  // pitched kernel: the fields at off_a and off_b
  long long id;
  // Cluster-resident solve: one dense buffer (off_a), its launch class
  // (cluster size, thread shape) and shared memory, planes per CTA.
  bool resident = false;
  int r_cluster = 0, r_variant = 0, r_pc = 0, r_yparts = 1, r_rows = 0;
  size_t r_smem = 0;
  int nx, ny, nz, steps, done;
  int px;  // row pitch in floats (nx, or nx rounded up to 4 when pitched)
  d3d::StripShape strip{};  // strip kernels: pieces, segments, rows
  int zc = 0, tiles = 0;  // this tick: planes per z slab, work items
  int n = 0;              // this tick: steps to run
  int lane = 0;           // compute stream that runs all its steps
  int kern = 0;           // step kernel (the server's, or its large one)
  float coeff[7];
  const float* host_in;
  float* host_out;
  unsigned long long off_a = 0, off_b = 0;
  bool cur_a = true;  // which buffer holds the current field
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  unsigned long long elems() const {
    return (unsigned long long)px * ny * nz;
  }
};

// Staging of one group of cluster-resident solves: descriptors (pinned and
// device), one work counter per launch, one step counter per solve, and
// the event that ends the group's launches.
struct ResStaging {
  d3d::ResidentDesc* h = nullptr;
  d3d::ResidentDesc* d = nullptr;
  int* d_steps = nullptr;
  size_t cap = 0;
  unsigned* d_queue = nullptr;  // kMaxResClasses counters
  cudaEvent_t done = nullptr;
  cudaStream_t stream = nullptr;  // descriptors in, launches joined
  bool in_flight = false;
};
constexpr int kMaxResClasses =
    d3d::kResidentMaxCluster * (d3d::kResidentParts + 3);
constexpr int kResStages = 16;         // group stagings in the ring
constexpr size_t kResGroupCap = 256;   // solves per group launch
constexpr int kResStreams = 16;        // streams the launches run on

// Staging for one tick's descriptors (BatchDesc or PitchedDesc, by the
// server's kernel) and work items, pinned + device.
struct Staging {
  void* h_desc = nullptr;
  int2* h_items = nullptr;
  void* d_desc = nullptr;
  int2* d_items = nullptr;
  size_t cap_desc = 0, cap_items = 0;  // bytes, items
  // Per lane: recorded before and after the lane's step launches.
  cudaEvent_t start[kMaxLanes] = {}, done[kMaxLanes] = {};
  bool used[kMaxLanes] = {};
  bool in_flight = false;
  bool timed = false;  // not yet added to the step time
};

}  // namespace

struct d3d_server_s {
  float* arena = nullptr;
  unsigned long long arena_elems = 0;
  ArenaAlloc alloc;
  int chunk = 8;
  int kernel = kDefaultKernel;  // pitched tile 0..4, strip 5..6, march -1
  // Solves whose pitched rows are at least large_px floats use
  // large_kernel (a pitched kernel) on the upper half of the lanes; the
  // others use `kernel` on the lower half.  large_kernel < 0: off.
  int large_kernel = -1, large_px = 0;
  std::deque<Request*> queued;
  std::vector<Request*> active;
  std::vector<Request*> retiring;
  // Solves are spread over `lanes` compute streams (each solve stays on
  // one), so one lane's launch tail overlaps another lane's work.
  cudaStream_t lane[kMaxLanes] = {};
  int lanes = kDefaultLanes;
  cudaStream_t copy = nullptr;
  Staging stage[2];
  int tick_index = 0;
  int device = 0;
  long long next_id = 0;
  long long submitted = 0, completed = 0, ticks = 0;
  double step_ms = 0.0;  // device time of the step launches
  unsigned long long launches = 0, peak_used = 0;
  // Cluster-resident solves: admitted and waiting for the next group
  // launch; the stream and stagings of those launches.
  bool resident = false;
  std::vector<Request*> res_pending;
  cudaStream_t res_pool[kResStreams] = {};
  cudaEvent_t res_join[kResStreams] = {};
  cudaEvent_t res_ready = nullptr;
  int res_rr = 0;
  // Group stagings: a fixed ring made when the resident path is switched
  // on.  Allocating while serving would serialise the lanes (a page-locked
  // or device allocation keeps work issued to different streams before and
  // after it from overlapping).  A staging is reused only once its launches
  // have ended (an event query, never a host wait), so a long small solve
  // does not hold up the ticks; with none free, the group waits a tick.
  std::vector<ResStaging*> rstage;
  long long res_solves = 0, res_launches = 0;
  std::map<std::tuple<int, int, size_t>, int> res_max_clusters;
};

namespace {

int sfail(int code, const char* msg) { return d3d::set_error(code, "%s", msg); }

#define S_TRY(call, what)                                             \
  do {                                                                \
    cudaError_t e__ = (call);                                         \
    if (e__ != cudaSuccess) return d3d::set_cuda_error(e__, what);    \
  } while (0)

void free_res_staging(ResStaging* st) {
  if (st->h) cudaFreeHost(st->h);
  if (st->d) cudaFree(st->d);
  if (st->d_steps) cudaFree(st->d_steps);
  if (st->d_queue) cudaFree(st->d_queue);
  if (st->done) cudaEventDestroy(st->done);
  if (st->stream) cudaStreamDestroy(st->stream);
  delete st;
}

// The resident path's stream pool, events and staging ring.  Streams and
// events missing after an earlier failure are made now; the ring is made
// whole or not at all, so a failed call leaves no half-built staging.
int make_resident_state(d3d_server s) {
  for (int i = 0; i < kResStreams; ++i) {
    if (!s->res_pool[i])
      S_TRY(cudaStreamCreateWithFlags(&s->res_pool[i],
                                      cudaStreamNonBlocking),
            "cudaStreamCreate");
    if (!s->res_join[i])
      S_TRY(cudaEventCreateWithFlags(&s->res_join[i],
                                     cudaEventDisableTiming),
            "cudaEventCreate");
  }
  if (!s->res_ready)
    S_TRY(cudaEventCreateWithFlags(&s->res_ready, cudaEventDisableTiming),
          "cudaEventCreate");
  if (!s->rstage.empty()) return D3D_OK;
  std::vector<ResStaging*> ring;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < kResStages && e == cudaSuccess; ++i) {
    ResStaging* st = new (std::nothrow) ResStaging();
    if (!st) {
      for (ResStaging* r : ring) free_res_staging(r);
      return sfail(D3D_E_OOM, "resident staging");
    }
    ring.push_back(st);
    st->cap = kResGroupCap;
    e = cudaMallocHost(&st->h, st->cap * sizeof(d3d::ResidentDesc));
    if (e == cudaSuccess)
      e = cudaMalloc(&st->d, st->cap * sizeof(d3d::ResidentDesc));
    if (e == cudaSuccess) e = cudaMalloc(&st->d_steps, st->cap * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMalloc(&st->d_queue, kMaxResClasses * sizeof(unsigned));
    if (e == cudaSuccess)
      e = cudaEventCreateWithFlags(&st->done, cudaEventDisableTiming);
    if (e == cudaSuccess)
      e = cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking);
  }
  if (e != cudaSuccess) {
    for (ResStaging* r : ring) free_res_staging(r);
    return d3d::set_cuda_error(e, "resident staging");
  }
  s->rstage.swap(ring);
  return D3D_OK;
}

int ensure_staging(Staging& st, size_t desc_bytes, size_t nitems) {
  if (desc_bytes > st.cap_desc) {
    if (st.h_desc) cudaFreeHost(st.h_desc);
    if (st.d_desc) cudaFree(st.d_desc);
    st.cap_desc = std::max(desc_bytes, 2 * st.cap_desc);
    S_TRY(cudaMallocHost(&st.h_desc, st.cap_desc),
          "cudaMallocHost (server staging)");
    S_TRY(cudaMalloc(&st.d_desc, st.cap_desc),
          "cudaMalloc (server staging)");
  }
  if (nitems > st.cap_items) {
    if (st.h_items) cudaFreeHost(st.h_items);
    if (st.d_items) cudaFree(st.d_items);
    st.cap_items = std::max(nitems, 2 * st.cap_items);
    S_TRY(cudaMallocHost(&st.h_items, st.cap_items * sizeof(int2)),
          "cudaMallocHost (server staging)");
    S_TRY(cudaMalloc(&st.d_items, st.cap_items * sizeof(int2)),
          "cudaMalloc (server staging)");
  }
  return D3D_OK;
}

void free_request(d3d_server s, Request* r) {
  if (r->ev_in) cudaEventDestroy(r->ev_in);
  if (r->ev_out) cudaEventDestroy(r->ev_out);
  s->alloc.release(r->off_a, r->elems());
  if (!r->resident) s->alloc.release(r->off_b, r->elems());
  delete r;
}

// Clusters of one resident launch class that fit the GPU at once (0: not
// schedulable), cached per (thread shape, cluster size, shared memory).
int res_max_clusters(d3d_server s, int variant, int cluster, size_t smem) {
  const auto key = std::make_tuple(variant, cluster, smem);
  auto it = s->res_max_clusters.find(key);
  if (it != s->res_max_clusters.end()) return it->second;
  int n = 0;
  if (d3d::resident_max_clusters(variant, cluster, smem, &n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  s->res_max_clusters[key] = n;
  return n;
}

// Whether a solve fits the cluster-resident kernel, and its class: the
// same rule as the batch API's (a thread shape covering its ceil(nx/4) * ny
// row segments a plane; at most 16 CTAs of pc planes plus one halo plane
// each), on a cluster the GPU can schedule.
void plan_resident_solve(d3d_server s, Request* r) {
  r->resident = false;
  if (!s->resident || r->steps < 1) return;
  if (d3d::resident_prepare() != cudaSuccess) {
    cudaGetLastError();
    s->resident = false;
    return;
  }
  d3d::ResidentFit fit;
  if (!d3d::resident_fit(r->nx, r->ny, r->nz, &fit)) return;
  const int cl = fit.cluster, v = fit.variant, pc = fit.pc;
  const size_t smem = fit.smem;
  if (res_max_clusters(s, v, cl, smem) < 1) return;
  r->resident = true;
  r->r_cluster = cl;
  r->r_variant = v;
  r->r_pc = pc;
  r->r_yparts = fit.yparts;
  r->r_rows = fit.rows;
  r->r_smem = smem;
  r->px = r->nx;  // one dense buffer
}

size_t dense_bytes(const Request* r) {
  return (size_t)r->nx * r->ny * r->nz * sizeof(float);
}

// Starts the device->host copy of a finished solve.  A pitched result is
// first made dense in the solve's other buffer (one device pass), so the
// copy to the host is one contiguous transfer.
// `in_a`: the result is in buffer a.  Called on the solve's lane right
// after its last step launch, so its copy-out does not wait for the rest
// of the lane's tick.
int start_retire(d3d_server s, Request* r, bool in_a) {
  const float* src = s->arena + (in_a ? r->off_a : r->off_b);
  if (r->px != r->nx) {
    float* dense = s->arena + (in_a ? r->off_b : r->off_a);
    S_TRY(d3d::launch_repitch(src, dense, r->nx, r->px,
                              (long long)r->ny * r->nz, false,
                              s->lane[r->lane]),
          "dense copy of a result");
    ++s->launches;
    d3d::note_launches(1);
    src = dense;
  }
  cudaEvent_t ready;
  S_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming),
        "cudaEventCreate");
  S_TRY(cudaEventRecord(ready, s->lane[r->lane]), "cudaEventRecord");
  S_TRY(cudaStreamWaitEvent(s->copy, ready, 0), "cudaStreamWaitEvent");
  cudaEventDestroy(ready);
  S_TRY(cudaMemcpyAsync(r->host_out, src, dense_bytes(r),
                        cudaMemcpyDeviceToHost, s->copy),
        "D2H copy (result)");
  S_TRY(cudaEventCreateWithFlags(&r->ev_out, cudaEventDisableTiming),
        "cudaEventCreate");
  S_TRY(cudaEventRecord(r->ev_out, s->copy), "cudaEventRecord");
  s->retiring.push_back(r);
  return D3D_OK;
}

int admit(d3d_server s) {
  // Outstanding point-steps per lane; a new solve joins the lightest.
  double work[kMaxLanes] = {};
  for (const Request* r : s->active)
    work[r->lane] += (double)r->elems() * (r->steps - r->done);
  for (auto it = s->queued.begin(); it != s->queued.end();) {
    Request* r = *it;
    unsigned long long a, b;
    if (r->resident) {
      if (!s->alloc.alloc(r->elems(), &a)) {
        ++it;
        continue;
      }
      r->off_a = a;
      S_TRY(cudaMemcpyAsync(s->arena + a, r->host_in, dense_bytes(r),
                            cudaMemcpyHostToDevice, s->copy),
            "H2D copy (input)");
      S_TRY(cudaEventCreateWithFlags(&r->ev_in, cudaEventDisableTiming),
            "cudaEventCreate");
      S_TRY(cudaEventRecord(r->ev_in, s->copy), "cudaEventRecord");
      it = s->queued.erase(it);
      s->res_pending.push_back(r);
      continue;
    }
    if (!s->alloc.alloc(r->elems(), &a)) {
      ++it;
      continue;
    }
    if (!s->alloc.alloc(r->elems(), &b)) {
      s->alloc.release(a, r->elems());
      ++it;
      continue;
    }
    r->off_a = a;
    r->off_b = b;
    // (One lane runs one kernel: with a single lane there is no split.)
    const bool large = s->kernel >= 0 && s->large_kernel >= 0 &&
                       s->lanes > 1 && r->px >= s->large_px;
    r->kern = large ? s->large_kernel : s->kernel;
    if (r->kern >= 0) {
      int bxm, bym;
      if (strip_nr(r->kern)) {
        r->strip = d3d::strip_shape(r->px, r->ny, strip_nr(r->kern));
        bxm = 4 * r->strip.segs + 8;
        bym = r->strip.rows + 2;
      } else {
        bxm = d3d::pitched_box_x(r->kern);
        bym = d3d::pitched_box_y(r->kern);
      }
      for (int m = 0; m < 2; ++m) {
        cudaError_t e = d3d::encode_field_map(
            &r->map[m], s->arena + (m ? b : a), r->px, r->ny, r->nz,
            d3d::kF32, bxm, bym);
        if (e != cudaSuccess) {
          s->alloc.release(a, r->elems());
          s->alloc.release(b, r->elems());
          return d3d::set_cuda_error(e, "tensor map of a served solve");
        }
      }
    }
    // The input lands dense; a pitched solve lands in its b buffer and is
    // spread into a (pads filled) by one device pass on the copy stream.
    float* land = s->arena + (r->px != r->nx ? b : a);
    S_TRY(cudaMemcpyAsync(land, r->host_in, dense_bytes(r),
                          cudaMemcpyHostToDevice, s->copy),
          "H2D copy (input)");
    if (r->px != r->nx) {
      S_TRY(d3d::launch_repitch(land, s->arena + a, r->nx, r->px,
                                (long long)r->ny * r->nz, true, s->copy),
            "pitched copy of an input");
      ++s->launches;
      d3d::note_launches(1);
    }
    S_TRY(cudaEventCreateWithFlags(&r->ev_in, cudaEventDisableTiming),
          "cudaEventCreate");
    S_TRY(cudaEventRecord(r->ev_in, s->copy), "cudaEventRecord");
    // With a large kernel, the two kernels keep to their own lanes.
    int l0 = 0, l1 = s->lanes;
    if (s->kernel >= 0 && s->large_kernel >= 0 && s->lanes > 1 &&
        s->large_kernel != s->kernel) {
      const int half = s->lanes / 2;
      if (large) l0 = half;
      else l1 = half;
    }
    r->lane = l0;
    for (int l = l0 + 1; l < l1; ++l)
      if (work[l] < work[r->lane]) r->lane = l;
    work[r->lane] += (double)r->elems() * r->steps;
    S_TRY(cudaStreamWaitEvent(s->lane[r->lane], r->ev_in, 0),
          "cudaStreamWaitEvent");
    it = s->queued.erase(it);
    if (r->steps == 0) {
      int rc = start_retire(s, r, true);
      if (rc) return rc;
    } else {
      s->active.push_back(r);
    }
  }
  s->peak_used = std::max(s->peak_used, s->alloc.used());
  return D3D_OK;
}

// Launches every cluster-resident solve admitted since the last group:
// one persistent launch per (cluster size, thread shape), largest work
// first.  A launch lasts as long as its longest solve (its steps run one
// after another), so each goes on an idle stream of the resident pool,
// after its solves' input copies, and groups overlap; each result is
// copied out on the same stream once its launch ends.  The group's
// descriptors travel on its staging's own stream, which joins the
// launches' streams to mark the staging free again.
int launch_resident_group(d3d_server s) {
  if (s->res_pending.empty()) return D3D_OK;
  ResStaging* free_st = nullptr;
  for (ResStaging* c : s->rstage) {
    if (c->in_flight) {
      const cudaError_t q = cudaEventQuery(c->done);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) return d3d::set_cuda_error(q, "resident group");
      c->in_flight = false;
    }
    free_st = c;
    break;
  }
  if (!free_st) return D3D_OK;  // every staging busy: a later tick launches
  ResStaging& st = *free_st;
  std::vector<Request*>& list = s->res_pending;
  std::stable_sort(list.begin(), list.end(), [](const Request* x,
                                                const Request* y) {
    if (x->r_cluster != y->r_cluster) return x->r_cluster > y->r_cluster;
    if (x->r_variant != y->r_variant) return x->r_variant < y->r_variant;
    return (double)x->nx * x->ny * x->nz * x->steps >
           (double)y->nx * y->ny * y->nz * y->steps;
  });
  // At most one staging's worth; the rest wait for the next group.  The
  // first `n` of the sorted list are still grouped by class.
  const size_t n = std::min(list.size(), st.cap);
  for (size_t i = 0; i < n; ++i) {
    const Request* r = list[i];
    d3d::ResidentDesc& d = st.h[i];
    d.in = s->arena + r->off_a;
    d.out = s->arena + r->off_a;  // each CTA writes only the planes it read
    d.nx = r->nx;
    d.ny = r->ny;
    d.nz = r->nz;
    d.steps = r->steps;
    d.px = (r->nx + 3) / 4 * 4;
    d.segs = d.px / 4;
    d.pc = r->r_pc;
    d.grid_id = (int)i;
    d.yparts = r->r_yparts;
    d.rows = r->r_rows;
    for (int j = 0; j < 7; ++j) d.k[j] = r->coeff[j];
    d.k[7] = -0.0f;
  }
  const cudaStream_t gs = st.stream;
  S_TRY(cudaMemcpyAsync(st.d, st.h, n * sizeof(d3d::ResidentDesc),
                        cudaMemcpyHostToDevice, gs),
        "H2D resident descriptors");
  S_TRY(cudaMemsetAsync(st.d_queue, 0, kMaxResClasses * sizeof(unsigned),
                        gs),
        "work counter reset");
  S_TRY(cudaEventRecord(s->res_ready, gs), "cudaEventRecord");
  int ci = 0;
  for (size_t b = 0; b < n; ++ci) {
    size_t e = b;
    size_t smem = 0;
    while (e < n && list[e]->r_cluster == list[b]->r_cluster &&
           list[e]->r_variant == list[b]->r_variant) {
      smem = std::max(smem, list[e]->r_smem);
      ++e;
    }
    // The first idle stream of the pool, else the next one in turn.
    int p = -1;
    for (int k = 0; k < kResStreams && p < 0; ++k) {
      const int c = (s->res_rr + k) % kResStreams;
      if (cudaStreamQuery(s->res_pool[c]) == cudaSuccess) p = c;
    }
    if (p < 0) p = s->res_rr % kResStreams;
    s->res_rr = p + 1;
    const cudaStream_t ps = s->res_pool[p];
    S_TRY(cudaStreamWaitEvent(ps, s->res_ready, 0), "cudaStreamWaitEvent");
    for (size_t i = b; i < e; ++i)
      S_TRY(cudaStreamWaitEvent(ps, list[i]->ev_in, 0),
            "cudaStreamWaitEvent");
    const int cl = list[b]->r_cluster, v = list[b]->r_variant;
    const int nclusters =
        std::min<int>((int)(e - b), res_max_clusters(s, v, cl, smem));
    S_TRY(d3d::launch_resident(v, st.d + b, (int)(e - b), st.d_queue + ci,
                               st.d_steps, cl, nclusters, smem, ps),
          "resident launch");
    ++s->res_launches;
    ++s->launches;
    d3d::note_launches(1);
    // The results go out on the launch's own stream: the shared copy
    // stream carries the inputs of later admissions, which must not wait
    // for these launches.
    for (size_t i = b; i < e; ++i) {
      Request* r = list[i];
      S_TRY(cudaMemcpyAsync(r->host_out, s->arena + r->off_a,
                            dense_bytes(r), cudaMemcpyDeviceToHost, ps),
            "D2H copy (result)");
      S_TRY(cudaEventCreateWithFlags(&r->ev_out, cudaEventDisableTiming),
            "cudaEventCreate");
      S_TRY(cudaEventRecord(r->ev_out, ps), "cudaEventRecord");
      s->retiring.push_back(r);
      ++s->res_solves;
    }
    S_TRY(cudaEventRecord(s->res_join[p], ps), "cudaEventRecord");
    S_TRY(cudaStreamWaitEvent(gs, s->res_join[p], 0), "cudaStreamWaitEvent");
    b = e;
  }
  S_TRY(cudaEventRecord(st.done, gs), "cudaEventRecord");
  st.in_flight = true;
  list.erase(list.begin(), list.begin() + n);
  return D3D_OK;
}

// z slabs: planes per work item are capped at kMaxSlab (long marches make
// one launch wait for its slowest CTAs); while a tick's launch would have
// fewer than kSlabTarget work items the cap halves, down to kMinSlab
// planes (each slab re-reads the plane above and below it).
constexpr long kSlabTarget = 8 * 148;
constexpr int kMaxSlab = 32, kMinSlab = 16;
// Steps per tick: chunk * clamp(ceil(remaining / (chunk * kStepHorizon)),
// 1, kMaxStepMult).
constexpr int kStepHorizon = 4, kMaxStepMult = 4;
int slab_planes(int nz, int cap) {
  const int ns = (nz + cap - 1) / cap;
  return (nz + ns - 1) / ns;  // balanced slabs of at most `cap` planes
}

// Adds a finished tick's step time to the counters (once): the span from
// its first lane's start to its last lane's end.
void harvest(d3d_server s, Staging& st) {
  if (!st.timed) return;
  int first = -1, last = -1;
  for (int l = 0; l < kMaxLanes; ++l) {
    if (!st.used[l]) continue;
    if (cudaEventQuery(st.done[l]) != cudaSuccess) return;
    float ms = 0.0f;
    if (first < 0 ||
        (cudaEventElapsedTime(&ms, st.start[l], st.start[first]) ==
             cudaSuccess &&
         ms > 0.0f))
      first = l;
    if (last < 0 ||
        (cudaEventElapsedTime(&ms, st.done[last], st.done[l]) ==
             cudaSuccess &&
         ms > 0.0f))
      last = l;
  }
  float ms = 0.0f;
  if (first >= 0 &&
      cudaEventElapsedTime(&ms, st.start[first], st.done[last]) ==
          cudaSuccess)
    s->step_ms += ms;
  st.timed = false;
}

// Waits for every lane of a staging's tick.
int wait_staging(d3d_server s, Staging& st) {
  for (int l = 0; l < kMaxLanes; ++l)
    if (st.used[l])
      S_TRY(cudaEventSynchronize(st.done[l]), "cudaEventSynchronize");
  harvest(s, st);
  for (bool& u : st.used) u = false;
  st.in_flight = false;
  return D3D_OK;
}

int advance(d3d_server s) {
  if (s->active.empty()) return D3D_OK;
  Staging& st = s->stage[s->tick_index & 1];
  if (st.in_flight) {
    int rc = wait_staging(s, st);
    if (rc) return rc;
  }
  std::vector<Request*>& act = s->active;
  const bool pitched = s->kernel >= 0;
  auto geom = [](int kern) {
    KernGeom g{strip_nr(kern), d3d::kBShapes[0].bx, d3d::kBShapes[0].by};
    if (kern >= 0 && !g.nr) {
      g.bx = 4 * d3d::pitched_variant(kern).lanes;
      g.by = d3d::pitched_variant(kern).by;
    }
    return g;
  };
  // xy work items of a solve: tiles_x across, tiles_xy in all.
  auto xy_tiles = [&](const Request* r, int* tx) {
    const KernGeom g = geom(r->kern);
    if (g.nr) {
      *tx = r->strip.pieces;
      return r->strip.pieces * ((r->ny + r->strip.rows - 1) / r->strip.rows);
    }
    *tx = (r->nx + g.bx - 1) / g.bx;
    return *tx * ((r->ny + g.by - 1) / g.by);
  };
  size_t nitems = 0;
  for (int cap = kMaxSlab;; cap /= 2) {
    nitems = 0;
    for (Request* r : act) {
      int tx;
      const int txy = xy_tiles(r, &tx);
      r->zc = slab_planes(r->nz, cap);
      r->tiles = txy * ((r->nz + r->zc - 1) / r->zc);
      nitems += r->tiles;
    }
    if ((long)nitems >= kSlabTarget || cap / 2 < kMinSlab) break;
  }
  // Steps this tick: `chunk`, or a multiple of it for solves with many
  // steps left, so they do not set the makespan by needing more ticks than
  // anyone else; their extra launches hold few items and overlap other
  // lanes' work.
  const int chunk = s->chunk;
  int nj = 0;  // launches this tick (the most steps any solve runs)
  for (Request* r : act) {
    const int rem = r->steps - r->done;
    const int mult = std::min(kMaxStepMult,
                              std::max(1, (rem + chunk * kStepHorizon - 1) /
                                              (chunk * kStepHorizon)));
    r->n = std::min(rem, chunk * mult);
    nj = std::max(nj, r->n);
  }
  // Each lane's solves are contiguous.  Within a lane, the solves still
  // stepping at launch j must be a prefix: order by the steps this tick
  // runs, then by slab depth, longest first, so a launch starts its
  // longest CTAs first and its tail is short.
  std::sort(act.begin(), act.end(), [](const Request* x, const Request* y) {
    if (x->lane != y->lane) return x->lane < y->lane;
    if (x->n != y->n) return x->n > y->n;
    return x->zc > y->zc;
  });
  const size_t desc_size =
      pitched ? sizeof(d3d::PitchedDesc) : sizeof(d3d::BatchDesc);
  int rc = ensure_staging(st, act.size() * desc_size, nitems);
  if (rc) return rc;
  // Per lane: first descriptor, first item, items active at sub-step j.
  size_t desc0[kMaxLanes + 1] = {}, item0[kMaxLanes + 1] = {};
  std::vector<int> active_at((size_t)kMaxLanes * nj, 0);
  size_t k = 0;
  for (size_t i = 0; i < act.size(); ++i) {
    Request* r = act[i];
    for (int l = r->lane + 1; l <= kMaxLanes; ++l) {
      desc0[l] = i + 1;
      item0[l] = k + r->tiles;
    }
    float* cur = s->arena + (r->cur_a ? r->off_a : r->off_b);
    float* nxt = s->arena + (r->cur_a ? r->off_b : r->off_a);
    int tiles_x;
    const int tiles_xy = xy_tiles(r, &tiles_x);
    if (pitched) {
      d3d::PitchedDesc& d = static_cast<d3d::PitchedDesc*>(st.h_desc)[i];
      d.map[0] = r->map[r->cur_a ? 0 : 1];
      d.map[1] = r->map[r->cur_a ? 1 : 0];
      d.a = cur;
      d.b = nxt;
      d.nx = r->nx;
      d.px = r->px;
      d.ny = r->ny;
      d.nz = r->nz;
      d.tiles_x = tiles_x;
      d.tiles_xy = tiles_xy;
      d.zc = r->zc;
      d.unused = 0;
      d.seg_w = r->strip.segs;
      d.rows = r->strip.rows;
      for (int j = 0; j < 7; ++j) d.k[j] = r->coeff[j];
      d.k[7] = -0.0f;
    } else {
      d3d::BatchDesc& d = static_cast<d3d::BatchDesc*>(st.h_desc)[i];
      d.a = cur;
      d.b = nxt;
      d.nx = r->nx;
      d.ny = r->ny;
      d.nz = r->nz;
      d.tiles_x = tiles_x;
      d.tiles_xy = tiles_xy;
      d.zc = r->zc;
      for (int j = 0; j < 7; ++j) d.k[j] = r->coeff[j];
      d.k[7] = -0.0f;
    }
    for (int t = 0; t < r->tiles; ++t) st.h_items[k++] = make_int2((int)i, t);
    for (int j = 0; j < r->n; ++j)
      active_at[(size_t)r->lane * nj + j] += r->tiles;
  }
  // Each lane copies its own descriptors and items and launches its
  // sub-steps on its stream; lanes never wait for one another.
  unsigned long long n_launch = 0;
  for (int l = 0; l < s->lanes; ++l) {
    const size_t nd = desc0[l + 1] - desc0[l], ni = item0[l + 1] - item0[l];
    if (nd == 0) continue;
    cudaStream_t ls = s->lane[l];
    char* hd = static_cast<char*>(st.h_desc) + desc0[l] * desc_size;
    char* dd = static_cast<char*>(st.d_desc) + desc0[l] * desc_size;
    S_TRY(cudaMemcpyAsync(dd, hd, nd * desc_size, cudaMemcpyHostToDevice, ls),
          "H2D descriptors");
    S_TRY(cudaMemcpyAsync(st.d_items + item0[l], st.h_items + item0[l],
                          ni * sizeof(int2), cudaMemcpyHostToDevice, ls),
          "H2D work items");
    if (!st.start[l]) {
      S_TRY(cudaEventCreate(&st.start[l]), "cudaEventCreate");
      S_TRY(cudaEventCreate(&st.done[l]), "cudaEventCreate");
    }
    S_TRY(cudaEventRecord(st.start[l], ls), "cudaEventRecord");
    const int* act_l = active_at.data() + (size_t)l * nj;
    // This lane's solves in launch order of their last step (they are
    // sorted by n, descending): retire each right after it.
    size_t fin = desc0[l + 1];
    const int lk = act[desc0[l]]->kern;  // one kernel a lane
    const int nr = strip_nr(lk);
    for (int j = 0; j < nj && act_l[j] > 0; ++j) {
      auto* pd = static_cast<d3d::PitchedDesc*>(st.d_desc);
      S_TRY(nr ? d3d::launch_pitched_strip(nr, pd, st.d_items + item0[l],
                                           act_l[j], j & 1, ls,
                                           d3d::device_error_word())
            : pitched
                ? d3d::launch_pitched_step(
                      lk, pd, st.d_items + item0[l], act_l[j], j & 1,
                      ls, d3d::device_error_word())
                : d3d::launch_batch_step(
                      0, static_cast<d3d::BatchDesc*>(st.d_desc),
                      st.d_items + item0[l], act_l[j], j & 1, ls),
            "server step launch");
      ++n_launch;
      while (fin > desc0[l] && act[fin - 1]->n == j + 1) {
        Request* r = act[--fin];
        if (r->done + r->n >= r->steps) {
          rc = start_retire(s, r, r->cur_a != (bool)(r->n & 1));
          if (rc) return rc;
        }
      }
    }
    S_TRY(cudaEventRecord(st.done[l], ls), "cudaEventRecord");
    st.used[l] = true;
  }
  s->launches += n_launch;
  d3d::note_launches(n_launch);
  st.in_flight = true;
  st.timed = true;
  ++s->tick_index;
  // Book-keeping (finished solves are already retiring).
  std::vector<Request*> still;
  for (Request* r : act) {
    r->done += r->n;
    if (r->n & 1) r->cur_a = !r->cur_a;
    if (r->done < r->steps) still.push_back(r);
  }
  act.swap(still);
  return D3D_OK;
}

}  // namespace

extern "C" {

int d3d_server_create(size_t arena_bytes, int chunk, d3d_server* out) {
  if (!out || arena_bytes < 256 || chunk < 1 || chunk > 256)
    return sfail(D3D_E_INVALID, "bad server arguments");
  *out = nullptr;
  d3d_server s = new (std::nothrow) d3d_server_s();
  if (!s) return sfail(D3D_E_OOM, "server allocation");
  cudaGetDevice(&s->device);
  s->chunk = chunk;
  s->arena_elems = arena_bytes / sizeof(float) / kAlign * kAlign;
  cudaError_t e = cudaMalloc(&s->arena, s->arena_elems * sizeof(float));
  for (int l = 0; l < kMaxLanes && e == cudaSuccess; ++l)
    e = cudaStreamCreateWithFlags(&s->lane[l], cudaStreamNonBlocking);
  if (e == cudaSuccess)
    e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    d3d_server_destroy(s);
    return d3d::set_cuda_error(e, "server setup");
  }
  s->alloc.reset(s->arena_elems);
  *out = s;
  return D3D_OK;
}

int d3d_server_submit(d3d_server s, int nx, int ny, int nz, int steps,
                      const float coeff[7], const float* host_in,
                      float* host_out, long long* id) {
  if (!s || !coeff || !host_in || !host_out)
    return sfail(D3D_E_INVALID, "NULL argument");
  if (nx < 1 || ny < 1 || nz < 1 || steps < 0 ||
      ((long long)nx + 3) / 4 * 4 * ny >= (1LL << 31))
    return sfail(D3D_E_INVALID, "bad grid dimensions or steps");
  const int px = s->kernel >= 0 ? (nx + 3) / 4 * 4 : nx;
  Request* r = new (std::nothrow) Request();
  if (!r) return sfail(D3D_E_OOM, "request allocation");
  r->px = px;
  r->nx = nx;
  r->ny = ny;
  r->nz = nz;
  r->steps = steps;
  r->done = 0;
  plan_resident_solve(s, r);  // may switch it to one dense buffer
  const unsigned long long pts = r->elems();
  const unsigned long long need = (r->resident ? 1 : 2) *
                                  ((pts + kAlign - 1) / kAlign * kAlign);
  if (need > s->arena_elems) {
    delete r;
    return sfail(D3D_E_BUSY, "solve larger than the server's arena");
  }
  r->id = s->next_id++;
  memcpy(r->coeff, coeff, sizeof r->coeff);
  r->host_in = host_in;
  r->host_out = host_out;
  s->queued.push_back(r);
  ++s->submitted;
  if (id) *id = r->id;
  return D3D_OK;
}

int d3d_server_tick(d3d_server s, long long* done_ids, int max_done,
                    int* n_done) {
  if (!s || !n_done || (max_done > 0 && !done_ids))
    return sfail(D3D_E_INVALID, "NULL argument");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != s->device) return sfail(D3D_E_INVALID, "wrong device");
  *n_done = 0;
  // 1. retire
  std::vector<Request*> keep;
  for (Request* r : s->retiring) {
    cudaError_t q = cudaEventQuery(r->ev_out);
    if (q == cudaSuccess && *n_done < max_done) {
      done_ids[(*n_done)++] = r->id;
      ++s->completed;
      free_request(s, r);
    } else if (q == cudaSuccess || q == cudaErrorNotReady) {
      keep.push_back(r);
    } else {
      return d3d::set_cuda_error(q, "result copy");
    }
  }
  s->retiring.swap(keep);
  // 2. admit, 3. advance (4. inside advance)
  int rc = admit(s);
  if (rc) return rc;
  rc = launch_resident_group(s);
  if (rc) return rc;
  rc = advance(s);
  if (rc) return rc;
  ++s->ticks;
  return D3D_OK;
}

int d3d_server_set_resident(d3d_server s, int on) {
  if (!s) return sfail(D3D_E_INVALID, "NULL server");
  if (!s->queued.empty() || !s->active.empty() || !s->retiring.empty() ||
      !s->res_pending.empty())
    return sfail(D3D_E_BUSY,
                 "the resident path changes only on an idle server");
  if (on) {
    const int rc = make_resident_state(s);
    if (rc) return rc;
  }
  s->resident = on != 0;
  return D3D_OK;
}

int d3d_server_set_kernel(d3d_server s, int kernel) {
  if (!s) return sfail(D3D_E_INVALID, "NULL server");
  if (kernel < -1 || kernel > kMaxKernel)
    return sfail(D3D_E_INVALID, "no such server kernel");
  if (!s->queued.empty() || !s->active.empty() || !s->retiring.empty() ||
      !s->res_pending.empty())
    return sfail(D3D_E_BUSY, "the step kernel changes only on an idle server");
  s->kernel = kernel;
  return D3D_OK;
}

int d3d_server_set_large_kernel(d3d_server s, int kernel, int min_px) {
  if (!s) return sfail(D3D_E_INVALID, "NULL server");
  if (kernel > kMaxKernel || (kernel >= 0 && min_px < 1))
    return sfail(D3D_E_INVALID, "no such large-solve kernel");
  if (!s->queued.empty() || !s->active.empty() || !s->retiring.empty() ||
      !s->res_pending.empty())
    return sfail(D3D_E_BUSY,
                 "the large-solve kernel changes only on an idle server");
  s->large_kernel = kernel < 0 ? -1 : kernel;
  s->large_px = min_px;
  return D3D_OK;
}

int d3d_server_set_lanes(d3d_server s, int lanes) {
  if (!s) return sfail(D3D_E_INVALID, "NULL server");
  if (lanes < 1 || lanes > kMaxLanes)
    return sfail(D3D_E_INVALID, "lanes must be 1 to 8");
  if (!s->queued.empty() || !s->active.empty() || !s->retiring.empty() ||
      !s->res_pending.empty())
    return sfail(D3D_E_BUSY, "lanes change only on an idle server");
  s->lanes = lanes;
  return D3D_OK;
}

int d3d_server_pending(d3d_server s, int* queued, int* active,
                       int* retiring) {
  if (!s) return sfail(D3D_E_INVALID, "NULL server");
  if (queued) *queued = (int)s->queued.size();
  if (active) *active = (int)(s->active.size() + s->res_pending.size());
  if (retiring) *retiring = (int)s->retiring.size();
  return D3D_OK;
}

int d3d_server_stats(d3d_server s, char* buf, size_t len) {
  if (!s || !buf) return sfail(D3D_E_INVALID, "NULL argument");
  for (auto& st : s->stage) harvest(s, st);
  snprintf(buf, len,
           "{\"submitted\": %lld, \"completed\": %lld, \"ticks\": %lld, "
           "\"launches\": %llu, \"chunk\": %d, \"kernel\": %d, "
           "\"lanes\": %d, "
           "\"step_ms\": %.4f, \"resident\": %s, "
           "\"resident_solves\": %lld, \"resident_launches\": %lld, "
           "\"arena_bytes\": %llu, \"peak_arena_bytes\": %llu}",
           s->submitted, s->completed, s->ticks, s->launches, s->chunk,
           s->kernel, s->lanes, s->step_ms, s->resident ? "true" : "false",
           s->res_solves, s->res_launches, s->arena_elems * 4ULL,
           s->peak_used * 4ULL);
  return D3D_OK;
}

int d3d_server_destroy(d3d_server s) {
  if (!s) return D3D_OK;
  for (cudaStream_t l : s->lane)
    if (l) cudaStreamSynchronize(l);
  for (cudaStream_t p : s->res_pool)
    if (p) cudaStreamSynchronize(p);
  for (ResStaging* st : s->rstage)
    if (st->stream) cudaStreamSynchronize(st->stream);
  if (s->copy) cudaStreamSynchronize(s->copy);
  for (Request* r : s->queued) delete r;
  for (Request* r : s->active) free_request(s, r);
  for (Request* r : s->res_pending) free_request(s, r);
  for (Request* r : s->retiring) free_request(s, r);
  for (ResStaging* st : s->rstage) free_res_staging(st);
  for (int i = 0; i < kResStreams; ++i) {
    if (s->res_pool[i]) cudaStreamDestroy(s->res_pool[i]);
    if (s->res_join[i]) cudaEventDestroy(s->res_join[i]);
  }
  if (s->res_ready) cudaEventDestroy(s->res_ready);
  for (auto& st : s->stage) {
    if (st.h_desc) cudaFreeHost(st.h_desc);
    if (st.h_items) cudaFreeHost(st.h_items);
    if (st.d_desc) cudaFree(st.d_desc);
    if (st.d_items) cudaFree(st.d_items);
    for (int l = 0; l < kMaxLanes; ++l) {
      if (st.start[l]) cudaEventDestroy(st.start[l]);
      if (st.done[l]) cudaEventDestroy(st.done[l]);
    }
  }
  if (s->arena) cudaFree(s->arena);
  for (cudaStream_t l : s->lane)
    if (l) cudaStreamDestroy(l);
  if (s->copy) cudaStreamDestroy(s->copy);
  delete s;
  return D3D_OK;
}

}  // extern "C"
