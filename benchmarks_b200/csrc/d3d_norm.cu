// Device-side error norms and the analytic field.
//
// The reference reports accuracy on the host: GetCorrectAnswer rebuilds the
// analytic field with Initialize(t = count*dt) (diffusion3d.h:113-120) and
// Baseline::GetAccuracy sums the squared error in float (baseline.cc:51-60).
// These kernels provide the FP64 error report beside it, on the device:
//   * analytic_kernel -- the same closed form, evaluated in double;
//   * compare kernels  -- rms, max-abs, max-rel and a checksum accumulated
//     in double over two device fields of any dtype pair, in a fixed
//     reduction order (deterministic for a given device).
#include <cfloat>
#include <mutex>

#include "d3d_common.cuh"
#include "d3d_kernels.h"

namespace d3d {

namespace {

constexpr int kCmpThreads = 256;
constexpr int kCmpBlocks = 1024;  // partials in scratch: 4 doubles each

template <typename T>
__device__ __forceinline__ double ld_as_double(const void* p, size_t i) {
  return (double)static_cast<const T*>(p)[i];
}

struct Acc {
  double ss, mx, mr, sa;
};

// max that keeps a NaN: fmax returns the other operand when one is NaN,
// which would report a finite max_abs / max_rel for a field holding NaNs
// (its rms and checksum are NaN already).
__device__ __forceinline__ double nan_max(double a, double b) {
  return (isnan(a) || isnan(b)) ? a + b : fmax(a, b);
}

__device__ __forceinline__ void acc_merge(Acc& a, const Acc& b) {
  a.ss += b.ss;
  a.mx = nan_max(a.mx, b.mx);
  a.mr = nan_max(a.mr, b.mr);
  a.sa += b.sa;
}

__device__ Acc block_reduce(Acc v) {
  __shared__ Acc sh[kCmpThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Acc u;
    u.ss = __shfl_down_sync(0xffffffffu, v.ss, o);
    u.mx = __shfl_down_sync(0xffffffffu, v.mx, o);
    u.mr = __shfl_down_sync(0xffffffffu, v.mr, o);
    u.sa = __shfl_down_sync(0xffffffffu, v.sa, o);
    acc_merge(v, u);
  }
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  Acc r = {0, 0, 0, 0};
  if (threadIdx.x == 0) {
    for (int w = 0; w < kCmpThreads / 32; ++w) acc_merge(r, sh[w]);
  }
  return r;
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(kCmpThreads)
    compare_partial_kernel(const void* a, const void* b, size_t n,
                           double* partial) {
  Acc v = {0, 0, 0, 0};
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += stride) {
    const double x = ld_as_double<TA>(a, i);
    const double y = ld_as_double<TB>(b, i);
    const double d = x - y;
    const double ad = fabs(d);
    const double den = fmax(fabs(y), 1e-300);
    v.ss += d * d;
    v.mx = nan_max(v.mx, ad);
    v.mr = nan_max(v.mr, ad / den);
    v.sa += x;
  }
  Acc r = block_reduce(v);
  if (threadIdx.x == 0) {
    double* p = partial + 4 * (size_t)blockIdx.x;
    p[0] = r.ss;
    p[1] = r.mx;
    p[2] = r.mr;
    p[3] = r.sa;
  }
}

__global__ void __launch_bounds__(kCmpThreads)
    compare_final_kernel(const double* partial, int nparts, size_t n,
                         double* out) {
  Acc v = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    const double* p = partial + 4 * (size_t)i;
    Acc u = {p[0], p[1], p[2], p[3]};
    acc_merge(v, u);
  }
  Acc r = block_reduce(v);
  if (threadIdx.x == 0) {
    out[0] = n ? sqrt(r.ss / (double)n) : 0.0;
    out[1] = r.mx;
    out[2] = r.mr;
    out[3] = r.sa;
  }
}

template <typename T>
__global__ void analytic_kernel(T* out, int nx, int ny, int nz, double kx,
                                double ky, double kz, double dx, double dy,
                                double dz, double ax, double ay, double az) {
  const size_t n = (size_t)nx * ny * nz;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += stride) {
    const int jx = (int)(i % nx);
    const int jy = (int)((i / nx) % ny);
    const int jz = (int)(i / ((size_t)nx * ny));
    const double x = dx * (jx + 0.5), y = dy * (jy + 0.5), z = dz * (jz + 0.5);
    out[i] = (T)(0.125 * (1.0 - ax * cos(kx * x)) * (1.0 - ay * cos(ky * y)) *
                 (1.0 - az * cos(kz * z)));
  }
}

// Field against the analytic solution, the analytic value evaluated per
// point in double (no analytic buffer): one read of the field.
template <typename T>
__global__ void __launch_bounds__(kCmpThreads)
    accuracy_partial_kernel(const T* f, int nx, int ny, int nz, double kx,
                            double ky, double kz, double dx, double dy,
                            double dz, double ax, double ay, double az,
                            double* partial) {
  Acc v = {0, 0, 0, 0};
  const size_t n = (size_t)nx * ny * nz;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += stride) {
    const int jx = (int)(i % nx);
    const int jy = (int)((i / nx) % ny);
    const int jz = (int)(i / ((size_t)nx * ny));
    const double y_ref = 0.125 * (1.0 - ax * cos(kx * (dx * (jx + 0.5)))) *
                         (1.0 - ay * cos(ky * (dy * (jy + 0.5)))) *
                         (1.0 - az * cos(kz * (dz * (jz + 0.5))));
    const double x = (double)f[i];
    const double d = x - y_ref;
    const double ad = fabs(d);
    v.ss += d * d;
    v.mx = nan_max(v.mx, ad);
    v.mr = nan_max(v.mr, ad / fmax(fabs(y_ref), 1e-300));
    v.sa += x;
  }
  Acc r = block_reduce(v);
  if (threadIdx.x == 0) {
    double* p = partial + 4 * (size_t)blockIdx.x;
    p[0] = r.ss;
    p[1] = r.mx;
    p[2] = r.mr;
    p[3] = r.sa;
  }
}

// One CTA waits, with a short bound, on an mbarrier phase that nothing
// completes (no thread ever arrives): the bounded-wait failure path every
// TMA kernel relies on, exercised without a fault.
__global__ void selftest_wait_kernel(unsigned limit, unsigned* dev_err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  bool done = false;
  for (unsigned i = 0; i < limit && !done; ++i) done = mbar_try_wait(&bar, 0);
  if (!__syncthreads_or(done) && threadIdx.x == 0)
    atomicOr(dev_err, kDevWaitTimeout);
}

template <typename TA>
cudaError_t launch_partial(const void* a, const void* b, int b_dtype, size_t n,
                           double* partial, int blocks, cudaStream_t s) {
  if (b_dtype == kF64)
    compare_partial_kernel<TA, double>
        <<<blocks, kCmpThreads, 0, s>>>(a, b, n, partial);
  else
    compare_partial_kernel<TA, float>
        <<<blocks, kCmpThreads, 0, s>>>(a, b, n, partial);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free comparison (d3d_compare_noalloc).
//
// Some callers cannot allocate device memory when they need the error
// report: a serving process that has already handed all free HBM to its
// solve arena, a host whose allocator policy forbids driver allocations
// behind its back, or a latency-sensitive loop in which a cudaMalloc would
// synchronise the whole device.  For them the partial sums live in this
// fixed file-scope array, which every GPU that loads the library holds
// until the process exits.
//
// Limits and sharing: one partial per kNoAllocChunk elements, at most
// kNoAllocMaxParts partials, so n <= 2^28 elements (1 GiB of FP32).  Every
// call uses the same array: a call writes every partial it later reads,
// so nothing has to start at zero, but two calls whose kernels overlap on
// the GPU (different streams, no ordering between them) race on it.
// ---------------------------------------------------------------------------
constexpr int kNoAllocChunk = 1 << 16;
constexpr int kNoAllocMaxParts = 1 << 12;
static __device__ __align__(256) double
    g_noalloc_scratch[4 * (kNoAllocMaxParts + 1)];  // 128 KiB + 32 B

template <typename TA, typename TB>
__global__ void __launch_bounds__(kCmpThreads)
    compare_chunk_kernel(const void* a, const void* b, size_t n,
                         double* partial) {
  Acc v = {0, 0, 0, 0};
  const size_t lo = (size_t)blockIdx.x * kNoAllocChunk;
  const size_t hi = min(n, lo + kNoAllocChunk);
  for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double x = ld_as_double<TA>(a, i);
    const double y = ld_as_double<TB>(b, i);
    const double d = x - y;
    const double ad = fabs(d);
    v.ss += d * d;
    v.mx = nan_max(v.mx, ad);
    v.mr = nan_max(v.mr, ad / fmax(fabs(y), 1e-300));
    v.sa += x;
  }
  Acc r = block_reduce(v);
  if (threadIdx.x == 0) {
    double* p = partial + 4 * (size_t)blockIdx.x;
    p[0] = r.ss;
    p[1] = r.mx;
    p[2] = r.mr;
    p[3] = r.sa;
  }
}

template <typename TA>
void launch_chunks(const void* a, const void* b, int b_dtype, size_t n,
                   double* partial, int parts, cudaStream_t s) {
  if (b_dtype == kF64)
    compare_chunk_kernel<TA, double>
        <<<parts, kCmpThreads, 0, s>>>(a, b, n, partial);
  else
    compare_chunk_kernel<TA, float>
        <<<parts, kCmpThreads, 0, s>>>(a, b, n, partial);
}

}  // namespace

size_t compare_noalloc_max_elements() {
  return (size_t)kNoAllocMaxParts * kNoAllocChunk;
}

// Device address of g_noalloc_scratch in the current device's context.
// In host code the array's name is only a host-side stand-in, never a
// device address, so the address is looked up with cudaGetSymbolAddress,
// with the device current, the first time a context of that device calls
// this (once per device, and once more after a cudaDeviceReset has
// replaced the device's primary context: the lookup is keyed on the
// context, so an address from a destroyed context is never reused).
cudaError_t noalloc_scratch(double** out) {
  struct Slot {
    void* ctx = nullptr;
    double* ptr = nullptr;
  };
  static Slot cache[64];
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  void* ctx = nullptr;
  e = current_context(&ctx);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  Slot& slot = cache[dev];
  if (!ctx || !slot.ptr || slot.ctx != ctx) {
    // (No context current yet: the lookup itself makes the device's
    // primary context current.)
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    e = current_context(&ctx);
    if (e != cudaSuccess) return e;
    slot.ptr = static_cast<double*>(addr);
    slot.ctx = ctx;
  }
  *out = slot.ptr;
  return cudaSuccess;
}

cudaError_t launch_compare_noalloc(const void* a, int a_dtype, const void* b,
                                   int b_dtype, size_t n, double* scratch,
                                   cudaStream_t stream) {
  const int parts = (int)((n + kNoAllocChunk - 1) / kNoAllocChunk);
  double* partial = scratch + 4;
  if (parts > 0) {
    if (a_dtype == kF64)
      launch_chunks<double>(a, b, b_dtype, n, partial, parts, stream);
    else
      launch_chunks<float>(a, b, b_dtype, n, partial, parts, stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  compare_final_kernel<<<1, kCmpThreads, 0, stream>>>(partial, parts, n,
                                                      scratch);
  return cudaGetLastError();
}

size_t compare_scratch_bytes() { return (size_t)(kCmpBlocks + 1) * 4 * 8; }

// Result lands in scratch[0..3] (the partials live after it).
cudaError_t launch_compare(const void* a, int a_dtype, const void* b,
                           int b_dtype, size_t n, double* scratch,
                           cudaStream_t stream) {
  const int blocks = kCmpBlocks;
  double* partial = scratch + 4;
  cudaError_t e = a_dtype == kF64
                      ? launch_partial<double>(a, b, b_dtype, n, partial,
                                               blocks, stream)
                      : launch_partial<float>(a, b, b_dtype, n, partial,
                                              blocks, stream);
  if (e != cudaSuccess) return e;
  compare_final_kernel<<<1, kCmpThreads, 0, stream>>>(partial, blocks, n,
                                                      scratch);
  return cudaGetLastError();
}

cudaError_t launch_accuracy(const void* f, int dtype, int ndim, int nx,
                            int ny, int nz, double kx, double ky, double kz,
                            double dx, double dy, double dz, double kappa,
                            double time, double* scratch,
                            cudaStream_t stream) {
  const double ax = exp(-kappa * time * (kx * kx));
  const double ay = exp(-kappa * time * (ky * ky));
  // A 2D field has no z factor: az = 0 makes it exactly 1.
  const double az = ndim == 2 ? 0.0 : exp(-kappa * time * (kz * kz));
  double* partial = scratch + 4;
  if (dtype == kF64)
    accuracy_partial_kernel<double><<<kCmpBlocks, kCmpThreads, 0, stream>>>(
        static_cast<const double*>(f), nx, ny, nz, kx, ky, kz, dx, dy, dz, ax,
        ay, az, partial);
  else
    accuracy_partial_kernel<float><<<kCmpBlocks, kCmpThreads, 0, stream>>>(
        static_cast<const float*>(f), nx, ny, nz, kx, ky, kz, dx, dy, dz, ax,
        ay, az, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  compare_final_kernel<<<1, kCmpThreads, 0, stream>>>(
      partial, kCmpBlocks, (size_t)nx * ny * nz, scratch);
  return cudaGetLastError();
}

cudaError_t launch_selftest_wait(unsigned limit, unsigned* dev_err,
                                 cudaStream_t stream) {
  selftest_wait_kernel<<<1, 32, 0, stream>>>(limit, dev_err);
  return cudaGetLastError();
}

cudaError_t launch_analytic(void* out, int dtype, int ndim, int nx, int ny,
                            int nz, double kx, double ky, double kz,
                            double dx, double dy, double dz, double kappa,
                            double time, cudaStream_t stream) {
  const double ax = exp(-kappa * time * (kx * kx));
  const double ay = exp(-kappa * time * (ky * ky));
  const double az = ndim == 2 ? 0.0 : exp(-kappa * time * (kz * kz));
  const int threads = 256, blocks = 148 * 8;
  if (dtype == kF64)
    analytic_kernel<double><<<blocks, threads, 0, stream>>>(
        static_cast<double*>(out), nx, ny, nz, kx, ky, kz, dx, dy, dz, ax, ay,
        az);
  else
    analytic_kernel<float><<<blocks, threads, 0, stream>>>(
        static_cast<float*>(out), nx, ny, nz, kx, ky, kz, dx, dy, dz, ax, ay,
        az);
  return cudaGetLastError();
}

}  // namespace d3d
