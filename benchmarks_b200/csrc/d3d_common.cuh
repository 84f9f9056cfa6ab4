// Shared device-side building blocks of the diffusion3d sm_100a kernels.
//
// Field layout (as the reference's OFFSET3D, diffusion3d.h:33-34): x fastest,
// offset(i, j, k) = i + j*nx + k*nx*ny, no padding, FP32 or FP64.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace d3d {

// The seven coefficients in the reference's member order (diffusion3d.h:52).
template <typename T>
struct Coef {
  T ce, cw, cn, cs, ct, cb, cc;
};

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// One point update, diffusion3d_openmp.cc:61-62:
//   cc*c + cw*w + ce*e + cs*s + cn*n + cb*b + ct*t
// summed left to right, every product and sum rounded separately (no FMA
// contraction), so the result is bit-identical to the reference's CPU build.
// n is y-1, s is y+1, b is z-1, t is z+1.
template <typename T>
__device__ __forceinline__ T point(const Coef<T>& k, T c, T w, T e, T s, T n,
                                   T b, T t) {
  T v = mul_rn(k.cc, c);
  v = add_rn(v, mul_rn(k.cw, w));
  v = add_rn(v, mul_rn(k.ce, e));
  v = add_rn(v, mul_rn(k.cs, s));
  v = add_rn(v, mul_rn(k.cn, n));
  v = add_rn(v, mul_rn(k.cb, b));
  v = add_rn(v, mul_rn(k.ct, t));
  return v;
}

// 16-byte vector of T (4 floats or 2 doubles).
template <typename T>
struct alignas(16) V16 {
  static constexpr int N = 16 / sizeof(T);
  T e[N];
};

template <typename T>
__device__ __forceinline__ V16<T> ld16_shared(const T* p) {
  V16<T> r;
  *reinterpret_cast<int4*>(&r) = *reinterpret_cast<const int4*>(p);
  return r;
}

template <typename T>
__device__ __forceinline__ void st16_global(T* p, const V16<T>& v) {
  *reinterpret_cast<int4*>(p) = *reinterpret_cast<const int4*>(&v);
}

// ----------------------------------------------------------------------
// Device error word.  Kernels never trap: a wait that exceeds its bound
// records a code here and the kernel returns; the host reads it after the
// launch (d3d_check_device_errors).
// ----------------------------------------------------------------------
enum DeviceError : unsigned {
  kDevOk = 0,
  kDevWaitTimeout = 1,
  kDevDrainTimeout = 2,
  kDevBadLaunch = 3,
  kDevPeerWaitTimeout = 4,
};

// ----------------------------------------------------------------------
// mbarrier + TMA (cp.async.bulk.tensor) helpers, sm_90+ PTX, used on sm_100a.
// No multicast form is used anywhere in this library.
// ----------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
                                                      unsigned bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase.  Each try_wait suspends for a
// hardware-chosen interval; the bound keeps the total far below any
// watchdog but far above any real TMA latency.
constexpr unsigned kMaxWaitIters = 1u << 22;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar,
                                                  unsigned parity) {
  for (unsigned i = 0; i < kMaxWaitIters; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* smem_dst,
                                            const CUtensorMap* map,
                                            uint64_t* bar, int x, int y,
                                            int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::"
      "complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
      "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

}  // namespace d3d
