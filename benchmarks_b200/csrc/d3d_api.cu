// The C ABI of libd3d_b200.so (declared in include/d3d_b200.h).
//
// Host-side runtime around the kernels: plans (shape, dtype, kernel and
// tile choice, cached TMA descriptors), the RunKernel-style step loops with
// the reference's pointer swap, host<->device staging, error reporting.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "d3d_b200.h"
#include "d3d_kernels.h"

using d3d::kF32;
using d3d::kF64;

static_assert(d3d::kNumTmaVariants == D3D_NUM_TILE_VARIANTS &&
                  d3d::kNumStep2dVariants == D3D_NUM_TILE_VARIANTS,
              "d3d_plan_set_tile takes one variant range for 2D and 3D");

namespace {

thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};

// Kernels record bounded-wait failures here instead of trapping.
__device__ unsigned g_dev_error_word;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky-free error so the next call is clean
  return fail(e == cudaErrorMemoryAllocation ? D3D_E_OOM : D3D_E_CUDA,
              "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
}

#define D3D_TRY(call, what)                         \
  do {                                              \
    cudaError_t e__ = (call);                       \
    if (e__ != cudaSuccess) return cuda_fail(e__, what); \
  } while (0)

// Device address of the error word in the current context, looked up once
// per context (a cudaDeviceReset replaces the device's primary context, and
// with it this address).
unsigned* dev_error_ptr() {
  struct Slot {
    void* ctx = nullptr;
    unsigned* ptr = nullptr;
  };
  static Slot slots[64];
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return nullptr;
  void* ctx = nullptr;
  if (d3d::current_context(&ctx) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  Slot& slot = slots[dev];
  if (!ctx || !slot.ptr || slot.ctx != ctx) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_dev_error_word) != cudaSuccess)
      return nullptr;
    if (d3d::current_context(&ctx) != cudaSuccess) return nullptr;
    slot.ptr = static_cast<unsigned*>(p);
    slot.ctx = ctx;
  }
  return slot.ptr;
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

bool valid_dims(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) return false;
  // TMA coordinates and the generic kernel's grid are 32-bit; planes of up
  // to 2^31 points and fields of up to 2^40 points are addressable.
  if ((long long)nx * ny >= (1LL << 31)) return false;
  if ((long long)nx * ny * nz >= (1LL << 40)) return false;
  return true;
}

// Diffusion3D::Diffusion3D (diffusion3d.h:54-66): the same expressions,
// evaluated with the same intermediate precisions as the reference when T
// is float (double literals 0.1, 1.0, 2.0*pi promote, then narrow).
template <typename T>
void reference_coefficients(int nx, int ny, int nz, T* coeff, T* geom) {
  const T kappa = (T)0.1;
  const T l = (T)1.0;
  const T dx = l / nx, dy = l / ny, dz = l / nz;
  const T k = (T)(2.0 * 3.14159265358979323846);
  const T dt = (T)(0.1 * dx * dx / kappa);
  const T ce = kappa * dt / (dx * dx);
  const T cn = kappa * dt / (dy * dy);
  const T ct = kappa * dt / (dz * dz);
  const T cc = (T)(1.0 - (ce + ce + cn + cn + ct + ct));
  if (coeff) {
    const T c[7] = {ce, ce, cn, cn, ct, ct, cc};
    memcpy(coeff, c, sizeof c);
  }
  if (geom) {
    const T g[8] = {kappa, dx, dy, dz, k, k, k, dt};
    memcpy(geom, g, sizeof g);
  }
}

// diffusion::Diffusion::Diffusion(nd, dims) (diffusion.h:93-108): the
// geometry and ce..cb of the diffusion3d constructor (ny = 1 below 2D,
// nz = 1 below 3D), but cc adds the z pair as a unit, and only in 3D:
// cc = 1.0 - (ce + cw + cn + cs + (nd == 3 ? ct + cb : 0)).
template <typename T>
void diffusion_coefficients(int nd, int nx, int ny, int nz, T* coeff,
                            T* geom) {
  T c[7];
  reference_coefficients<T>(nx, ny, nz, c, geom);
  const T xy = c[0] + c[1] + c[2] + c[3];
  const T zpair = nd == 3 ? (T)(c[4] + c[5]) : (T)0;
  c[6] = (T)(1.0 - (double)(xy + zpair));
  if (coeff) memcpy(coeff, c, sizeof c);
}

}  // namespace

namespace d3d {
int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}
int set_cuda_error(cudaError_t e, const char* what) {
  return cuda_fail(e, what);
}
void note_launches(unsigned long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
}
unsigned* device_error_word() { return dev_error_ptr(); }
}  // namespace d3d

struct d3d_plan_s {
  int nx, ny, nz, dtype, kernel, tb_depth;
  // 3 for 3D grids, 2 for the 2D grids of the diffusion::Diffusion surface.
  int ndim;
  // Sum the y-1 neighbour before y+1 (diffusion::Diffusion) instead of
  // after it (diffusion3d).
  int flip_y;
  int variant;  // TMA tile variant
  int zchunk;   // 0 = automatic
  int device;
  size_t n;
  // Small cache of TMA descriptors keyed by (pointer, box rows).
  struct MapEntry {
    const void* ptr;
    int box_x, box_y;
    CUtensorMap map;
  } maps[4];
  int map_next;
  double* cmp_scratch;  // device scratch for d3d_compare
  cudaEvent_t ev[2];
  // Step loops captured once into CUDA graphs and replayed, keyed by
  // buffers, step count, tile choice and coefficient bytes.
  struct GraphEntry {
    const void* f1;
    const void* f2;
    int count, variant, zchunk;
    unsigned char coeff[7 * 8];
    cudaGraphExec_t exec;
    void* result;
    void* other;
    unsigned long long launches;
  } graphs[4];
  int graph_next;
  int use_graphs;
  cudaStream_t capture_stream;
  d3d::LaunchInfo last;
  const char* last_kernel;
};

namespace {

int get_map(d3d_plan p, const void* ptr, int box_x, int box_y,
            const CUtensorMap** out) {
  for (auto& m : p->maps)
    if (m.ptr == ptr && m.box_x == box_x && m.box_y == box_y) {
      *out = &m.map;
      return D3D_OK;
    }
  auto& m = p->maps[p->map_next];
  p->map_next = (p->map_next + 1) % 4;
  cudaError_t e = d3d::encode_field_map(&m.map, ptr, p->nx, p->ny, p->nz,
                                        p->dtype, box_x, box_y);
  if (e != cudaSuccess) {
    m.ptr = nullptr;
    return fail(D3D_E_CUDA, "cuTensorMapEncodeTiled failed for %p", ptr);
  }
  m.ptr = ptr;
  m.box_x = box_x;
  m.box_y = box_y;
  *out = &m.map;
  return D3D_OK;
}

int check_device(d3d_plan p) {
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device)
    return fail(D3D_E_INVALID, "plan bound to device %d, current is %d",
                p->device, dev);
  return D3D_OK;
}

// One single-step launch, choosing the TMA path when the buffer allows it.
int step_once(d3d_plan p, const void* f1, void* f2, const void* coeff,
              cudaStream_t s, int zb = 0, int ze = -1) {
  if (p->ndim == 2) {
    D3D_TRY(d3d::launch_step2d(f1, f2, p->nx, p->ny, coeff, p->dtype,
                               p->variant, p->zchunk, s, &p->last),
            "step2d launch");
    p->last_kernel = "step2d";
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return D3D_OK;
  }
  const bool use_tma = p->kernel != D3D_KERNEL_GENERIC &&
                       d3d::tma_eligible(f1, p->nx, p->ny, p->dtype);
  if (p->kernel == D3D_KERNEL_TMA && !use_tma)
    return fail(D3D_E_UNSUPPORTED,
                "TMA kernel needs a 16-byte aligned buffer and nx*%d %% 16 == 0",
                (int)d3d::dtype_size(p->dtype));
  if (use_tma) {
    const CUtensorMap* map = nullptr;
    int rc = get_map(p, f1, d3d::tma_box_x(p->dtype),
                     d3d::tma_box_y(p->variant), &map);
    if (rc) return rc;
    D3D_TRY(d3d::launch_step_tma(*map, f2, p->nx, p->ny, p->nz, coeff,
                                 p->dtype, p->variant, p->zchunk, p->flip_y,
                                 s, dev_error_ptr(), &p->last, zb, ze),
            "step_tma launch");
    p->last_kernel = "step_tma";
  } else {
    D3D_TRY(d3d::launch_step_generic(f1, f2, p->nx, p->ny, p->nz, coeff,
                                     p->dtype, p->flip_y, s, &p->last, zb,
                                     ze),
            "step_generic launch");
    p->last_kernel = "step_generic";
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return D3D_OK;
}

// Temporal-blocking kernel choice: variant 0 of a K = 2 FP32 plan is the
// warp-row kernel, anything else the generic-K kernel.
bool use_tb2w(d3d_plan p) {
  return p->tb_depth == 2 && p->dtype == kF32 && p->variant == 0;
}

// Whether D3D_KERNEL_AUTO runs pairs of steps as fused two-step passes:
// FP32 3D grids of 2^27 points (512^3) or more, where the warp-row
// two-step kernel measured 12-14 % faster than single steps on B200
// (512^3: 837 against 732 Gpt/s; 768^3: 849 against 757); smaller grids
// keep the single-step kernel (384^3: 747 against 752).
bool auto_two_step(d3d_plan p, const void* f1, const void* f2) {
  return p->kernel == D3D_KERNEL_AUTO && p->dtype == kF32 && p->ndim == 3 &&
         p->n >= (size_t(1) << 27) &&
         d3d::tma_eligible(f1, p->nx, p->ny, p->dtype) &&
         d3d::tma_eligible(f2, p->nx, p->ny, p->dtype);
}

int tb2w_pass(d3d_plan p, const void* f1, void* f2, const void* coeff,
              int zchunk, cudaStream_t s) {
  const CUtensorMap* map = nullptr;
  int rc = get_map(p, f1, d3d::tb2w_box_x(), d3d::tb2w_box_y(), &map);
  if (rc) return rc;
  D3D_TRY(d3d::launch_steps_tb2w(*map, f2, p->nx, p->ny, p->nz, coeff,
                                 zchunk, p->flip_y, s, dev_error_ptr(),
                                 &p->last),
          "temporal-blocking launch");
  p->last_kernel = "steps_tb2w";
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return D3D_OK;
}

int tb_pass(d3d_plan p, const void* f1, void* f2, const void* coeff,
            cudaStream_t s) {
  if (use_tb2w(p)) return tb2w_pass(p, f1, f2, coeff, p->zchunk, s);
  const CUtensorMap* map = nullptr;
  int rc = get_map(p, f1, d3d::tb_box_x(p->dtype, p->tb_depth),
                   d3d::tb_box_y(p->tb_depth), &map);
  if (rc) return rc;
  D3D_TRY(d3d::launch_steps_tb(*map, f2, p->nx, p->ny, p->nz, coeff,
                               p->dtype, p->tb_depth, p->zchunk, p->flip_y, s,
                               dev_error_ptr(), &p->last),
          "temporal-blocking launch");
  p->last_kernel = "steps_tb";
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return D3D_OK;
}

int run_loop(d3d_plan p, void** f1, void** f2, const void* coeff, int count,
             cudaStream_t s) {
  int done = 0;
  if (count >= 2 && auto_two_step(p, *f1, *f2)) {
    for (; done + 2 <= count; done += 2) {
      int rc = tb2w_pass(p, *f1, *f2, coeff, 0, s);
      if (rc) return rc;
      std::swap(*f1, *f2);
    }
  }
  if (p->kernel == D3D_KERNEL_TB && p->tb_depth > 1 &&
      d3d::tma_eligible(*f1, p->nx, p->ny, p->dtype) &&
      d3d::tma_eligible(*f2, p->nx, p->ny, p->dtype)) {
    for (; done + p->tb_depth <= count; done += p->tb_depth) {
      int rc = tb_pass(p, *f1, *f2, coeff, s);
      if (rc) return rc;
      std::swap(*f1, *f2);
    }
  }
  for (; done < count; ++done) {
    int rc = step_once(p, *f1, *f2, coeff, s);
    if (rc) return rc;
    std::swap(*f1, *f2);
  }
  return D3D_OK;
}

void drop_graphs(d3d_plan p) {
  for (auto& g : p->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
  }
}

// The CUDA graph of a `count`-step run_loop on (f1, f2): found in the cache
// or captured once (on the plan's own stream, so nothing runs) and
// instantiated.  *out is null when graphs do not apply: disabled, fewer
// than two steps, or `s` itself being captured (the launches then land in
// the caller's graph).  Capture is host work only, so callers that time
// the loop call this before their start event.
int prepare_graph(d3d_plan p, void* f1, void* f2, const void* coeff,
                  int count, cudaStream_t s, d3d_plan_s::GraphEntry** out) {
  *out = nullptr;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (!p->use_graphs || count < 2 ||
      cudaStreamIsCapturing(s, &cap) != cudaSuccess ||
      cap != cudaStreamCaptureStatusNone)
    return D3D_OK;
  const size_t cb = 7 * d3d::dtype_size(p->dtype);
  for (auto& g : p->graphs)
    if (g.exec && g.f1 == f1 && g.f2 == f2 && g.count == count &&
        g.variant == p->variant && g.zchunk == p->zchunk &&
        memcmp(g.coeff, coeff, cb) == 0) {
      *out = &g;
      return D3D_OK;
    }
  if (!p->capture_stream)
    D3D_TRY(cudaStreamCreateWithFlags(&p->capture_stream,
                                      cudaStreamNonBlocking),
            "cudaStreamCreateWithFlags");
  auto& g = p->graphs[p->graph_next];
  p->graph_next = (p->graph_next + 1) % 4;
  if (g.exec) cudaGraphExecDestroy(g.exec);
  g.exec = nullptr;
  void* a = f1;
  void* b = f2;
  const unsigned long long l0 = g_launches.load();
  D3D_TRY(cudaStreamBeginCapture(p->capture_stream,
                                 cudaStreamCaptureModeThreadLocal),
          "cudaStreamBeginCapture");
  int rc = run_loop(p, &a, &b, coeff, count, p->capture_stream);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(p->capture_stream, &graph);
  const unsigned long long captured = g_launches.load() - l0;
  g_launches.fetch_sub(captured);  // counted when the graph runs
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    g.exec = nullptr;
    return cuda_fail(e, "cudaGraphInstantiate");
  }
  g.f1 = f1;
  g.f2 = f2;
  g.count = count;
  g.variant = p->variant;
  g.zchunk = p->zchunk;
  memcpy(g.coeff, coeff, cb);
  g.result = a;
  g.other = b;
  g.launches = captured;
  *out = &g;
  return D3D_OK;
}

int launch_graph(const d3d_plan_s::GraphEntry* g, void** f1, void** f2,
                 cudaStream_t s) {
  D3D_TRY(cudaGraphLaunch(g->exec, s), "cudaGraphLaunch");
  g_launches.fetch_add(g->launches, std::memory_order_relaxed);
  *f1 = g->result;
  *f2 = g->other;
  return D3D_OK;
}

// run_loop through a cached CUDA graph: the `count` launches of a
// RunKernel-style loop are captured once and replayed as one graph launch,
// which removes the per-launch host overhead and the gaps between steps.
int run_graphed(d3d_plan p, void** f1, void** f2, const void* coeff,
                int count, cudaStream_t s) {
  d3d_plan_s::GraphEntry* g = nullptr;
  int rc = prepare_graph(p, *f1, *f2, coeff, count, s, &g);
  if (rc) return rc;
  if (!g) return run_loop(p, f1, f2, coeff, count, s);
  return launch_graph(g, f1, f2, s);
}

}  // namespace

extern "C" {

const char* d3d_version(void) { return "d3d_b200 1.0 (sm_100a)"; }

const char* d3d_last_error(void) { return g_last_error.c_str(); }

unsigned long long d3d_launch_count(void) { return g_launches.load(); }

int d3d_coefficients(int nx, int ny, int nz, int dtype, void* coeff7,
                     void* geom8) {
  if (!valid_dims(nx, ny, nz))
    return fail(D3D_E_INVALID, "bad dims %dx%dx%d", nx, ny, nz);
  if (dtype == kF64)
    reference_coefficients<double>(nx, ny, nz, static_cast<double*>(coeff7),
                                   static_cast<double*>(geom8));
  else if (dtype == kF32)
    reference_coefficients<float>(nx, ny, nz, static_cast<float*>(coeff7),
                                  static_cast<float*>(geom8));
  else
    return fail(D3D_E_INVALID, "bad dtype %d", dtype);
  return D3D_OK;
}

}  // extern "C"

namespace {

int plan_new(int ndim, int flip_y, int nx, int ny, int nz, int dtype,
             int kernel, int tb_depth, d3d_plan* out) {
  if (!out) return fail(D3D_E_INVALID, "out is NULL");
  *out = nullptr;
  if (!valid_dims(nx, ny, nz))
    return fail(D3D_E_INVALID, "bad dims %dx%dx%d", nx, ny, nz);
  if (dtype != kF32 && dtype != kF64)
    return fail(D3D_E_INVALID, "bad dtype %d", dtype);
  if (kernel < D3D_KERNEL_AUTO || kernel > D3D_KERNEL_TB)
    return fail(D3D_E_INVALID, "bad kernel %d", kernel);
  if (ndim == 2 && (kernel == D3D_KERNEL_TMA || kernel == D3D_KERNEL_TB))
    return fail(D3D_E_UNSUPPORTED,
                "2D grids run the register-march kernel (AUTO or GENERIC); "
                "the TMA and temporal-blocking kernels are 3D");
  if (kernel == D3D_KERNEL_TB && !d3d::tb_supported(tb_depth, dtype))
    return fail(D3D_E_UNSUPPORTED, "temporal blocking depth %d unsupported",
                tb_depth);
  int dev = 0;
  D3D_TRY(cudaGetDevice(&dev), "cudaGetDevice");
  d3d_plan p = new (std::nothrow) d3d_plan_s();
  if (!p) return fail(D3D_E_OOM, "plan allocation");
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->ndim = ndim;
  p->flip_y = flip_y;
  p->dtype = dtype;
  p->kernel = kernel;
  p->tb_depth = kernel == D3D_KERNEL_TB ? tb_depth : 1;
  p->variant = kernel == D3D_KERNEL_TB ? 0
               : ndim == 2        ? d3d::default_step2d_variant()
                                  : d3d::default_tma_variant(nx, ny, nz, dtype);
  p->zchunk = 0;
  p->device = dev;
  p->n = (size_t)nx * ny * nz;
  p->last_kernel = "";
  p->use_graphs = 1;
  for (auto& m : p->maps) m.ptr = nullptr;
  cudaError_t e = cudaEventCreate(&p->ev[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&p->ev[1]);
  if (e != cudaSuccess) {
    delete p;
    return cuda_fail(e, "cudaEventCreate");
  }
  *out = p;
  return D3D_OK;
}

// nd and dims as diffusion::Diffusion takes them (main.cc builds dims as
// nd copies of --size); 0 on success with nx, ny, nz filled.
int diffusion_dims(int nd, const int* dims, int* nx, int* ny, int* nz) {
  if (!dims) return fail(D3D_E_INVALID, "dims is NULL");
  if (nd != 2 && nd != 3)
    return fail(D3D_E_INVALID, "nd must be 2 or 3, got %d", nd);
  *nx = dims[0];
  *ny = dims[1];
  *nz = nd == 3 ? dims[2] : 1;
  if (!valid_dims(*nx, *ny, *nz))
    return fail(D3D_E_INVALID, "bad dims %dx%dx%d", *nx, *ny, *nz);
  return D3D_OK;
}

}  // namespace

extern "C" {

int d3d_plan_create(int nx, int ny, int nz, int dtype, int kernel,
                    int tb_depth, d3d_plan* out) {
  return plan_new(3, 0, nx, ny, nz, dtype, kernel, tb_depth, out);
}

int d3d_diffusion_coefficients(int nd, const int* dims, int dtype,
                               void* coeff7, void* geom8) {
  int nx = 0, ny = 0, nz = 0;
  int rc = diffusion_dims(nd, dims, &nx, &ny, &nz);
  if (rc) return rc;
  if (dtype == kF64)
    diffusion_coefficients<double>(nd, nx, ny, nz,
                                   static_cast<double*>(coeff7),
                                   static_cast<double*>(geom8));
  else if (dtype == kF32)
    diffusion_coefficients<float>(nd, nx, ny, nz, static_cast<float*>(coeff7),
                                  static_cast<float*>(geom8));
  else
    return fail(D3D_E_INVALID, "bad dtype %d", dtype);
  return D3D_OK;
}

int d3d_diffusion_plan_create(int nd, const int* dims, int dtype, int kernel,
                              int tb_depth, d3d_plan* out) {
  if (out) *out = nullptr;
  int nx = 0, ny = 0, nz = 0;
  int rc = diffusion_dims(nd, dims, &nx, &ny, &nz);
  if (rc) return rc;
  return plan_new(nd, 1, nx, ny, nz, dtype, kernel, tb_depth, out);
}

int d3d_plan_set_tile(d3d_plan p, int variant, int zchunk) {
  if (!p) return fail(D3D_E_INVALID, "plan is NULL");
  if (variant < 0 || variant >= d3d::kNumTmaVariants || zchunk < 0)
    return fail(D3D_E_INVALID, "bad tile variant %d / zchunk %d", variant,
                zchunk);
  p->variant = variant;
  p->zchunk = zchunk;
  for (auto& m : p->maps) m.ptr = nullptr;  // box height may change
  return D3D_OK;
}

int d3d_plan_autotune(d3d_plan p, void* f1, void* f2, const void* coeff,
                      int steps, void* stream, double* best_ms) {
  if (!p || !f1 || !f2 || !coeff) return fail(D3D_E_INVALID, "NULL argument");
  if (f1 == f2) return fail(D3D_E_INVALID, "f1 and f2 alias");
  if (steps < 1) return fail(D3D_E_INVALID, "steps must be >= 1");
  int rc = check_device(p);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  const bool tb = p->kernel == D3D_KERNEL_TB;
  if (tb) steps = std::max(steps / p->tb_depth, 1) * p->tb_depth;
  const int zchunks3[] = {0, 16, 32, 64, 128, 256};
  const int zchunks2[] = {0, 2, 4, 6, 8, 12, 16, 32};  // rows per warp task
  const int* zchunks = p->ndim == 2 ? zchunks2 : zchunks3;
  const int nzc = p->ndim == 2 ? 8 : 6;
  // TB plans: variant 0 / 1 pick the K = 2 FP32 warp-row kernel or the
  // generic-K kernel (other depths and FP64 have only the latter).
  const int nvariants = tb ? ((p->tb_depth == 2 && p->dtype == kF32) ? 2 : 1)
                        : p->ndim == 2 ? d3d::kNumStep2dVariants
                                       : d3d::kNumTmaVariants;
  const int zext = p->ndim == 2 ? p->ny : p->nz;  // marched extent
  const int old_variant = p->variant, old_zchunk = p->zchunk;
  float best = -1.0f;
  int best_v = old_variant, best_z = old_zchunk;
  for (int v = 0; v < nvariants; ++v) {
    for (int zi = 0; zi < nzc; ++zi) {
      const int zc = zchunks[zi];
      if (zc != 0 && zc >= zext) continue;
      p->variant = (tb && nvariants == 1) ? p->variant : v;
      p->zchunk = zc;
      for (auto& m : p->maps) m.ptr = nullptr;
      void* a = f1;
      void* b = f2;
      // one untimed step (attributes, descriptors, caches), then timed
      rc = run_loop(p, &a, &b, coeff, tb ? p->tb_depth : 1, s);
      if (rc) break;
      D3D_TRY(cudaEventRecord(p->ev[0], s), "cudaEventRecord");
      rc = run_loop(p, &a, &b, coeff, steps, s);
      if (rc) break;
      D3D_TRY(cudaEventRecord(p->ev[1], s), "cudaEventRecord");
      D3D_TRY(cudaEventSynchronize(p->ev[1]), "cudaEventSynchronize");
      float ms = 0.0f;
      D3D_TRY(cudaEventElapsedTime(&ms, p->ev[0], p->ev[1]), "elapsed");
      if (best < 0.0f || ms < best) {
        best = ms;
        best_v = p->variant;
        best_z = zc;
      }
    }
    if (rc) break;
  }
  p->variant = rc ? old_variant : best_v;
  p->zchunk = rc ? old_zchunk : best_z;
  for (auto& m : p->maps) m.ptr = nullptr;
  drop_graphs(p);
  if (rc) return rc;
  if (best_ms) *best_ms = best / steps;
  return D3D_OK;
}

int d3d_plan_set_graphs(d3d_plan p, int enable) {
  if (!p) return fail(D3D_E_INVALID, "plan is NULL");
  p->use_graphs = enable ? 1 : 0;
  if (!enable) drop_graphs(p);
  return D3D_OK;
}

int d3d_plan_destroy(d3d_plan p) {
  if (!p) return D3D_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != p->device) cudaSetDevice(p->device);
  if (p->cmp_scratch) cudaFree(p->cmp_scratch);
  drop_graphs(p);
  if (p->capture_stream) cudaStreamDestroy(p->capture_stream);
  cudaEventDestroy(p->ev[0]);
  cudaEventDestroy(p->ev[1]);
  if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
  delete p;
  return D3D_OK;
}

int d3d_plan_info(d3d_plan p, char* buf, size_t len) {
  if (!p || !buf) return fail(D3D_E_INVALID, "NULL argument");
  const auto& L = p->last;
  snprintf(buf, len,
           "{\"nx\": %d, \"ny\": %d, \"nz\": %d, \"ndim\": %d, "
           "\"surface\": \"%s\", \"dtype\": \"%s\", "
           "\"kernel\": %d, \"tb_depth\": %d, \"variant\": %d, "
           "\"zchunk\": %d, \"device\": %d, \"last_kernel\": \"%s\", "
           "\"grid\": [%d, %d, %d], \"block\": %d, \"smem\": %d, "
           "\"launch_zchunk\": %d, \"ctas_per_sm\": %d, \"graphs\": %d}",
           p->nx, p->ny, p->nz, p->ndim,
           p->flip_y ? "diffusion" : "diffusion3d",
           p->dtype == kF64 ? "f64" : "f32", p->kernel,
           p->tb_depth, p->variant, p->zchunk, p->device, p->last_kernel,
           L.grid_x, L.grid_y, L.grid_z, L.block, L.smem_bytes, L.zchunk,
           L.ctas_per_sm, p->use_graphs);
  return D3D_OK;
}

int d3d_device_alloc(size_t bytes, void** ptr) {
  if (!ptr) return fail(D3D_E_INVALID, "ptr is NULL");
  D3D_TRY(cudaMalloc(ptr, bytes), "cudaMalloc");
  return D3D_OK;
}

int d3d_device_free(void* ptr) {
  D3D_TRY(cudaFree(ptr), "cudaFree");
  return D3D_OK;
}

int d3d_host_alloc(size_t bytes, void** ptr) {
  if (!ptr) return fail(D3D_E_INVALID, "ptr is NULL");
  D3D_TRY(cudaMallocHost(ptr, bytes), "cudaMallocHost");
  return D3D_OK;
}

int d3d_host_free(void* ptr) {
  D3D_TRY(cudaFreeHost(ptr), "cudaFreeHost");
  return D3D_OK;
}

int d3d_memcpy(void* dst, const void* src, size_t bytes, void* stream) {
  D3D_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault,
                          as_stream(stream)),
          "cudaMemcpyAsync");
  return D3D_OK;
}

int d3d_stream_sync(void* stream) {
  D3D_TRY(cudaStreamSynchronize(as_stream(stream)), "cudaStreamSynchronize");
  return D3D_OK;
}

int d3d_step(d3d_plan p, const void* f1, void* f2, const void* coeff,
             void* stream) {
  if (!p || !f1 || !f2 || !coeff) return fail(D3D_E_INVALID, "NULL argument");
  if (f1 == f2) return fail(D3D_E_INVALID, "f1 and f2 alias");
  int rc = check_device(p);
  if (rc) return rc;
  return step_once(p, f1, f2, coeff, as_stream(stream));
}

int d3d_step_planes(d3d_plan p, const void* f1, void* f2, int z_begin,
                    int z_end, const void* coeff, void* stream) {
  if (!p || !f1 || !f2 || !coeff) return fail(D3D_E_INVALID, "NULL argument");
  if (f1 == f2) return fail(D3D_E_INVALID, "f1 and f2 alias");
  if (p->ndim != 3)
    return fail(D3D_E_UNSUPPORTED, "plane ranges are for 3D plans");
  if (z_begin < 0 || z_begin >= z_end || z_end > p->nz)
    return fail(D3D_E_INVALID, "planes [%d, %d) outside [0, %d)", z_begin,
                z_end, p->nz);
  int rc = check_device(p);
  if (rc) return rc;
  return step_once(p, f1, f2, coeff, as_stream(stream), z_begin, z_end);
}

int d3d_run(d3d_plan p, void** f1, void** f2, const void* coeff, int count,
            void* stream) {
  if (!p || !f1 || !f2 || !*f1 || !*f2 || !coeff)
    return fail(D3D_E_INVALID, "NULL argument");
  if (*f1 == *f2) return fail(D3D_E_INVALID, "f1 and f2 alias");
  if (count < 0) return fail(D3D_E_INVALID, "negative count %d", count);
  int rc = check_device(p);
  if (rc) return rc;
  return run_graphed(p, f1, f2, coeff, count, as_stream(stream));
}

int d3d_run_host(d3d_plan p, void* host_f1, void* dev_f1, void* dev_f2,
                 const void* coeff, int count, void* stream,
                 float* kernel_ms) {
  if (!p || !host_f1 || !dev_f1 || !dev_f2 || !coeff)
    return fail(D3D_E_INVALID, "NULL argument");
  if (dev_f1 == dev_f2) return fail(D3D_E_INVALID, "f1 and f2 alias");
  if (count < 0) return fail(D3D_E_INVALID, "negative count %d", count);
  int rc = check_device(p);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  const size_t bytes = p->n * d3d::dtype_size(p->dtype);
  // Graph capture is one-off host setup; keep it out of the timed loop.
  d3d_plan_s::GraphEntry* g = nullptr;
  rc = prepare_graph(p, dev_f1, dev_f2, coeff, count, s, &g);
  if (rc) return rc;
  D3D_TRY(cudaMemcpyAsync(dev_f1, host_f1, bytes, cudaMemcpyHostToDevice, s),
          "H2D copy");
  D3D_TRY(cudaEventRecord(p->ev[0], s), "cudaEventRecord");
  void* a = dev_f1;
  void* b = dev_f2;
  rc = g ? launch_graph(g, &a, &b, s) : run_loop(p, &a, &b, coeff, count, s);
  if (rc) return rc;
  D3D_TRY(cudaEventRecord(p->ev[1], s), "cudaEventRecord");
  D3D_TRY(cudaMemcpyAsync(host_f1, a, bytes, cudaMemcpyDeviceToHost, s),
          "D2H copy");
  D3D_TRY(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  if (kernel_ms)
    D3D_TRY(cudaEventElapsedTime(kernel_ms, p->ev[0], p->ev[1]),
            "cudaEventElapsedTime");
  return D3D_OK;
}

int d3d_analytic(d3d_plan p, void* out, double time, void* stream) {
  if (!p || !out) return fail(D3D_E_INVALID, "NULL argument");
  int rc = check_device(p);
  if (rc) return rc;
  double g[8];
  reference_coefficients<double>(p->nx, p->ny, p->nz, nullptr, g);
  D3D_TRY(d3d::launch_analytic(out, p->dtype, p->ndim, p->nx, p->ny, p->nz,
                               g[4], g[5], g[6], g[1], g[2], g[3], g[0], time,
                               as_stream(stream)),
          "analytic launch");
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return D3D_OK;
}

int d3d_copy_calibrate(const float* f1, float* f2, size_t n, float cc,
                       int passes, void* stream, float* ms) {
  if (!f1 || !f2 || passes < 1) return fail(D3D_E_INVALID, "bad arguments");
  const uintptr_t a = reinterpret_cast<uintptr_t>(f1);
  const uintptr_t b = reinterpret_cast<uintptr_t>(f2);
  if (a < b + n * sizeof(float) && b < a + n * sizeof(float))
    return fail(D3D_E_INVALID, "the two buffers overlap");
  cudaStream_t s = as_stream(stream);
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaError_t e = cudaEventCreate(&ev[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
  if (e == cudaSuccess) e = cudaEventRecord(ev[0], s);
  const float* in = f1;
  float* out = f2;
  for (int i = 0; i < passes && e == cudaSuccess; ++i) {
    e = d3d::launch_scale_copy(in, out, n, cc, s);
    const float* t = in;
    in = out;
    out = const_cast<float*>(t);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ev[1], s);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
  float t_ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t_ms, ev[0], ev[1]);
  if (ev[0]) cudaEventDestroy(ev[0]);
  if (ev[1]) cudaEventDestroy(ev[1]);
  if (e != cudaSuccess) return cuda_fail(e, "copy calibration");
  g_launches.fetch_add((unsigned long long)passes, std::memory_order_relaxed);
  if (ms) *ms = t_ms;
  return D3D_OK;
}

int d3d_compare(d3d_plan p, const void* a, int a_dtype, const void* b,
                int b_dtype, size_t n, double out[4], void* stream) {
  if (!p || !a || !b || !out) return fail(D3D_E_INVALID, "NULL argument");
  if ((a_dtype != kF32 && a_dtype != kF64) ||
      (b_dtype != kF32 && b_dtype != kF64))
    return fail(D3D_E_INVALID, "bad dtype");
  int rc = check_device(p);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  if (!p->cmp_scratch)
    D3D_TRY(cudaMalloc(&p->cmp_scratch, d3d::compare_scratch_bytes()),
            "cudaMalloc (compare scratch)");
  D3D_TRY(d3d::launch_compare(a, a_dtype, b, b_dtype, n, p->cmp_scratch, s),
          "compare launch");
  g_launches.fetch_add(2, std::memory_order_relaxed);
  D3D_TRY(cudaMemcpyAsync(out, p->cmp_scratch, 4 * sizeof(double),
                          cudaMemcpyDeviceToHost, s),
          "D2H copy");
  D3D_TRY(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return D3D_OK;
}

}  // extern "C"

namespace {

d3d::PlanShape shape_of(d3d_plan p) {
  return d3d::PlanShape{p->nx, p->ny, p->nz, p->ndim, p->flip_y, p->dtype,
                        p->n};
}

int ensure_scratch(d3d_plan p) {
  if (!p->cmp_scratch)
    D3D_TRY(cudaMalloc(&p->cmp_scratch, d3d::compare_scratch_bytes()),
            "cudaMalloc (compare scratch)");
  return D3D_OK;
}

}  // namespace

extern "C" {

int d3d_checkpoint_save(d3d_plan p, const void* field, long long step,
                        const char* path, void* stream) {
  if (!p || !field || !path) return fail(D3D_E_INVALID, "NULL argument");
  int rc = check_device(p);
  if (!rc) rc = ensure_scratch(p);
  if (rc) return rc;
  return d3d::checkpoint_save(shape_of(p), p->cmp_scratch, field, step, path,
                              as_stream(stream));
}

int d3d_checkpoint_load(d3d_plan p, const char* path, void* field,
                        long long* step, void* stream) {
  if (!p || !field || !path) return fail(D3D_E_INVALID, "NULL argument");
  int rc = check_device(p);
  if (!rc) rc = ensure_scratch(p);
  if (rc) return rc;
  return d3d::checkpoint_load(shape_of(p), p->cmp_scratch, path, field, step,
                              as_stream(stream));
}

int d3d_checkpoint_save_host(d3d_plan p, const void* host_field,
                             long long step, const char* path) {
  if (!p || !host_field || !path) return fail(D3D_E_INVALID, "NULL argument");
  return d3d::checkpoint_save_host(shape_of(p), host_field, step, path);
}

int d3d_compare_noalloc(const void* a, int a_dtype, const void* b,
                        int b_dtype, size_t n, double out[4], void* stream) {
  if (!a || !b || !out) return fail(D3D_E_INVALID, "NULL argument");
  if ((a_dtype != kF32 && a_dtype != kF64) ||
      (b_dtype != kF32 && b_dtype != kF64))
    return fail(D3D_E_INVALID, "bad dtype");
  const size_t max_n = d3d::compare_noalloc_max_elements();
  if (n > max_n)
    return fail(D3D_E_INVALID,
                "n = %zu exceeds the allocation-free limit of %zu elements "
                "(use d3d_compare for larger fields)",
                n, max_n);
  cudaStream_t s = as_stream(stream);
  // The report comes back to the host, so the call waits for its stream;
  // a stream that is being captured cannot be waited for.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  D3D_TRY(cudaStreamIsCapturing(s, &cap), "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return fail(D3D_E_INVALID,
                "d3d_compare_noalloc waits for its stream and cannot be "
                "called on a stream that is being captured");
  double* scratch = nullptr;
  D3D_TRY(d3d::noalloc_scratch(&scratch),
          "cudaGetSymbolAddress (allocation-free scratch)");
  D3D_TRY(d3d::launch_compare_noalloc(a, a_dtype, b, b_dtype, n, scratch, s),
          "compare launch");
  g_launches.fetch_add(n ? 2 : 1, std::memory_order_relaxed);
  D3D_TRY(cudaMemcpyAsync(out, scratch, 4 * sizeof(double),
                          cudaMemcpyDeviceToHost, s),
          "D2H copy");
  D3D_TRY(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return D3D_OK;
}

int d3d_accuracy(d3d_plan p, const void* field, int count, double out[4],
                 void* stream) {
  if (!p || !field || !out) return fail(D3D_E_INVALID, "NULL argument");
  if (count < 0) return fail(D3D_E_INVALID, "negative count %d", count);
  int rc = check_device(p);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  if (!p->cmp_scratch)
    D3D_TRY(cudaMalloc(&p->cmp_scratch, d3d::compare_scratch_bytes()),
            "cudaMalloc (compare scratch)");
  // time = count * dt in the plan's precision, as GetCorrectAnswer forms it
  // (diffusion3d.h:113-120); the closed form itself in double.
  double time;
  if (p->dtype == kF64) {
    double g[8];
    reference_coefficients<double>(p->nx, p->ny, p->nz, nullptr, g);
    time = (double)count * g[7];
  } else {
    float g[8];
    reference_coefficients<float>(p->nx, p->ny, p->nz, nullptr, g);
    time = (double)((float)count * g[7]);
  }
  double g64[8];
  reference_coefficients<double>(p->nx, p->ny, p->nz, nullptr, g64);
  D3D_TRY(d3d::launch_accuracy(field, p->dtype, p->ndim, p->nx, p->ny,
                               p->nz, g64[4], g64[5], g64[6], g64[1], g64[2],
                               g64[3], g64[0], time, p->cmp_scratch, s),
          "accuracy launch");
  g_launches.fetch_add(2, std::memory_order_relaxed);
  D3D_TRY(cudaMemcpyAsync(out, p->cmp_scratch, 4 * sizeof(double),
                          cudaMemcpyDeviceToHost, s),
          "D2H copy");
  D3D_TRY(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return D3D_OK;
}

int d3d_selftest_wait_timeout(unsigned iterations, unsigned* flags_out) {
  unsigned* err = dev_error_ptr();
  if (!err) return fail(D3D_E_CUDA, "cannot resolve device error word");
  D3D_TRY(d3d::launch_selftest_wait(iterations, err, nullptr),
          "self-test launch");
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return d3d_check_device_errors(flags_out);
}

int d3d_check_device_errors(unsigned* flags_out) {
  D3D_TRY(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  unsigned* p = dev_error_ptr();
  if (!p) return fail(D3D_E_CUDA, "cannot resolve device error word");
  unsigned v = 0;
  D3D_TRY(cudaMemcpy(&v, p, sizeof v, cudaMemcpyDeviceToHost), "D2H copy");
  if (v) D3D_TRY(cudaMemset(p, 0, sizeof v), "cudaMemset");
  if (flags_out) *flags_out = v;
  if (v) return fail(D3D_E_TIMEOUT, "device error flags 0x%x", v);
  return D3D_OK;
}

}  // extern "C"
