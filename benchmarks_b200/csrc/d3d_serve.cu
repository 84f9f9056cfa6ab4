// Continuous-batching solve server (d3d_server_* in include/d3d_b200.h).
//
// State of a request: queued -> active (its two buffers live in the device
// arena; input copied in on the copy stream) -> retiring (its result is
// being copied to the caller's host buffer) -> done.  A tick advances every
// active solve by up to `chunk` steps with the multi-grid step kernel, the
// same kernel the batch API uses: within a tick, solves are ordered by
// steps remaining so the ones still stepping at sub-step j are a prefix of
// the work list.  At most two ticks are in flight; their descriptor/work
// lists use alternating staging buffers.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "d3d_b200.h"
#include "d3d_common.cuh"
#include "d3d_kernels.h"

namespace {

constexpr unsigned long long kAlign = 64;  // elements (256 bytes)

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
  long long id;
  int nx, ny, nz, steps, done;
  float coeff[7];
  const float* host_in;
  float* host_out;
  unsigned long long off_a = 0, off_b = 0;
  bool cur_a = true;  // which buffer holds the current field
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  unsigned long long points() const {
    return (unsigned long long)nx * ny * nz;
  }
};

// Staging for one tick's descriptors and work items (pinned + device).
struct Staging {
  d3d::BatchDesc* h_desc = nullptr;
  int2* h_items = nullptr;
  d3d::BatchDesc* d_desc = nullptr;
  int2* d_items = nullptr;
  size_t cap_desc = 0, cap_items = 0;
  cudaEvent_t done = nullptr;  // recorded after the tick's kernels
  bool in_flight = false;
};

}  // namespace

struct d3d_server_s {
  float* arena = nullptr;
  unsigned long long arena_elems = 0;
  ArenaAlloc alloc;
  int chunk = 8;
  std::deque<Request*> queued;
  std::vector<Request*> active;
  std::vector<Request*> retiring;
  cudaStream_t compute = nullptr, copy = nullptr;
  Staging stage[2];
  int tick_index = 0;
  int device = 0;
  long long next_id = 0;
  long long submitted = 0, completed = 0, ticks = 0;
  unsigned long long launches = 0, peak_used = 0;
};

namespace {

int sfail(int code, const char* msg) { return d3d::set_error(code, "%s", msg); }

#define S_TRY(call, what)                                             \
  do {                                                                \
    cudaError_t e__ = (call);                                         \
    if (e__ != cudaSuccess) return d3d::set_cuda_error(e__, what);    \
  } while (0)

int ensure_staging(Staging& st, size_t ndesc, size_t nitems) {
  if (ndesc > st.cap_desc) {
    if (st.h_desc) cudaFreeHost(st.h_desc);
    if (st.d_desc) cudaFree(st.d_desc);
    st.cap_desc = std::max(ndesc, 2 * st.cap_desc);
    S_TRY(cudaMallocHost(&st.h_desc, st.cap_desc * sizeof(d3d::BatchDesc)),
          "cudaMallocHost (server staging)");
    S_TRY(cudaMalloc(&st.d_desc, st.cap_desc * sizeof(d3d::BatchDesc)),
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
  s->alloc.release(r->off_a, r->points());
  s->alloc.release(r->off_b, r->points());
  delete r;
}

// Starts the device->host copy of a finished solve.
int start_retire(d3d_server s, Request* r) {
  cudaEvent_t ready;
  S_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming),
        "cudaEventCreate");
  S_TRY(cudaEventRecord(ready, s->compute), "cudaEventRecord");
  S_TRY(cudaStreamWaitEvent(s->copy, ready, 0), "cudaStreamWaitEvent");
  cudaEventDestroy(ready);
  const float* src = s->arena + (r->cur_a ? r->off_a : r->off_b);
  S_TRY(cudaMemcpyAsync(r->host_out, src, r->points() * sizeof(float),
                        cudaMemcpyDeviceToHost, s->copy),
        "D2H copy (result)");
  S_TRY(cudaEventCreateWithFlags(&r->ev_out, cudaEventDisableTiming),
        "cudaEventCreate");
  S_TRY(cudaEventRecord(r->ev_out, s->copy), "cudaEventRecord");
  s->retiring.push_back(r);
  return D3D_OK;
}

int admit(d3d_server s) {
  for (auto it = s->queued.begin(); it != s->queued.end();) {
    Request* r = *it;
    unsigned long long a, b;
    if (!s->alloc.alloc(r->points(), &a)) {
      ++it;
      continue;
    }
    if (!s->alloc.alloc(r->points(), &b)) {
      s->alloc.release(a, r->points());
      ++it;
      continue;
    }
    r->off_a = a;
    r->off_b = b;
    S_TRY(cudaMemcpyAsync(s->arena + a, r->host_in,
                          r->points() * sizeof(float),
                          cudaMemcpyHostToDevice, s->copy),
          "H2D copy (input)");
    S_TRY(cudaEventCreateWithFlags(&r->ev_in, cudaEventDisableTiming),
          "cudaEventCreate");
    S_TRY(cudaEventRecord(r->ev_in, s->copy), "cudaEventRecord");
    S_TRY(cudaStreamWaitEvent(s->compute, r->ev_in, 0),
          "cudaStreamWaitEvent");
    it = s->queued.erase(it);
    if (r->steps == 0) {
      int rc = start_retire(s, r);
      if (rc) return rc;
    } else {
      s->active.push_back(r);
    }
  }
  s->peak_used = std::max(s->peak_used, s->alloc.used());
  return D3D_OK;
}

int advance(d3d_server s) {
  if (s->active.empty()) return D3D_OK;
  Staging& st = s->stage[s->tick_index & 1];
  if (st.in_flight) {
    S_TRY(cudaEventSynchronize(st.done), "cudaEventSynchronize");
    st.in_flight = false;
  }
  std::vector<Request*>& act = s->active;
  std::sort(act.begin(), act.end(), [](const Request* x, const Request* y) {
    return x->steps - x->done > y->steps - y->done;
  });
  const d3d::BShape sh = d3d::kBShapes[0];
  size_t nitems = 0;
  std::vector<int> tiles(act.size());
  for (size_t i = 0; i < act.size(); ++i) {
    const Request* r = act[i];
    tiles[i] = ((r->nx + sh.bx - 1) / sh.bx) * ((r->ny + sh.by - 1) / sh.by);
    nitems += tiles[i];
  }
  int rc = ensure_staging(st, act.size(), nitems);
  if (rc) return rc;
  std::vector<int> active_at(s->chunk, 0);
  size_t k = 0;
  for (size_t i = 0; i < act.size(); ++i) {
    Request* r = act[i];
    d3d::BatchDesc& d = st.h_desc[i];
    d.a = s->arena + (r->cur_a ? r->off_a : r->off_b);
    d.b = s->arena + (r->cur_a ? r->off_b : r->off_a);
    d.nx = r->nx;
    d.ny = r->ny;
    d.nz = r->nz;
    d.tiles_x = (r->nx + sh.bx - 1) / sh.bx;
    for (int j = 0; j < 7; ++j) d.k[j] = r->coeff[j];
    d.k[7] = -0.0f;
    for (int t = 0; t < tiles[i]; ++t) st.h_items[k++] = make_int2((int)i, t);
    const int n = std::min(s->chunk, r->steps - r->done);
    for (int j = 0; j < n; ++j) active_at[j] += tiles[i];
  }
  S_TRY(cudaMemcpyAsync(st.d_desc, st.h_desc,
                        act.size() * sizeof(d3d::BatchDesc),
                        cudaMemcpyHostToDevice, s->compute),
        "H2D descriptors");
  S_TRY(cudaMemcpyAsync(st.d_items, st.h_items, nitems * sizeof(int2),
                        cudaMemcpyHostToDevice, s->compute),
        "H2D work items");
  unsigned long long n_launch = 0;
  for (int j = 0; j < s->chunk && active_at[j] > 0; ++j) {
    S_TRY(d3d::launch_batch_step(0, st.d_desc, st.d_items, active_at[j],
                                 j & 1, s->compute),
          "server step launch");
    ++n_launch;
  }
  s->launches += n_launch;
  d3d::note_launches(n_launch);
  if (!st.done)
    S_TRY(cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming),
          "cudaEventCreate");
  S_TRY(cudaEventRecord(st.done, s->compute), "cudaEventRecord");
  st.in_flight = true;
  ++s->tick_index;
  // Book-keeping, then start the copies of the solves that finished.
  std::vector<Request*> still;
  for (Request* r : act) {
    const int n = std::min(s->chunk, r->steps - r->done);
    r->done += n;
    if (n & 1) r->cur_a = !r->cur_a;
    if (r->done >= r->steps) {
      rc = start_retire(s, r);
      if (rc) return rc;
    } else {
      still.push_back(r);
    }
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
  if (e == cudaSuccess)
    e = cudaStreamCreateWithFlags(&s->compute, cudaStreamNonBlocking);
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
      (long long)nx * ny >= (1LL << 31))
    return sfail(D3D_E_INVALID, "bad grid dimensions or steps");
  const unsigned long long pts = (unsigned long long)nx * ny * nz;
  const unsigned long long need = 2 * ((pts + kAlign - 1) / kAlign * kAlign);
  if (need > s->arena_elems)
    return sfail(D3D_E_BUSY, "solve larger than the server's arena");
  Request* r = new (std::nothrow) Request();
  if (!r) return sfail(D3D_E_OOM, "request allocation");
  r->id = s->next_id++;
  r->nx = nx;
  r->ny = ny;
  r->nz = nz;
  r->steps = steps;
  r->done = 0;
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
  rc = advance(s);
  if (rc) return rc;
  ++s->ticks;
  return D3D_OK;
}

int d3d_server_pending(d3d_server s, int* queued, int* active,
                       int* retiring) {
  if (!s) return sfail(D3D_E_INVALID, "NULL server");
  if (queued) *queued = (int)s->queued.size();
  if (active) *active = (int)s->active.size();
  if (retiring) *retiring = (int)s->retiring.size();
  return D3D_OK;
}

int d3d_server_stats(d3d_server s, char* buf, size_t len) {
  if (!s || !buf) return sfail(D3D_E_INVALID, "NULL argument");
  snprintf(buf, len,
           "{\"submitted\": %lld, \"completed\": %lld, \"ticks\": %lld, "
           "\"launches\": %llu, \"chunk\": %d, \"arena_bytes\": %llu, "
           "\"peak_arena_bytes\": %llu}",
           s->submitted, s->completed, s->ticks, s->launches, s->chunk,
           s->arena_elems * 4ULL, s->peak_used * 4ULL);
  return D3D_OK;
}

int d3d_server_destroy(d3d_server s) {
  if (!s) return D3D_OK;
  if (s->compute) cudaStreamSynchronize(s->compute);
  if (s->copy) cudaStreamSynchronize(s->copy);
  for (Request* r : s->queued) delete r;
  for (Request* r : s->active) free_request(s, r);
  for (Request* r : s->retiring) free_request(s, r);
  for (auto& st : s->stage) {
    if (st.h_desc) cudaFreeHost(st.h_desc);
    if (st.h_items) cudaFreeHost(st.h_items);
    if (st.d_desc) cudaFree(st.d_desc);
    if (st.d_items) cudaFree(st.d_items);
    if (st.done) cudaEventDestroy(st.done);
  }
  if (s->arena) cudaFree(s->arena);
  if (s->compute) cudaStreamDestroy(s->compute);
  if (s->copy) cudaStreamDestroy(s->copy);
  delete s;
  return D3D_OK;
}

}  // extern "C"
