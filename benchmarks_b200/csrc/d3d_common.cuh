// Shared device-side building blocks of the diffusion3d sm_100a kernels.
//
// Field layout (as the reference's OFFSET3D, diffusion3d.h:33-34): x fastest,
// offset(i, j, k) = i + j*nx + k*nx*ny, no padding, FP32 or FP64.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace d3d {

// The seven coefficients in the reference's member order (diffusion3d.h:52),
// plus `nz`, which the host always sets to -0.0: a runtime value the
// compiler cannot see, used to form exactly rounded packed products (see
// point2).
template <typename T>
struct Coef {
  T ce, cw, cn, cs, ct, cb, cc;
  T nz;
};

// Host: the kernel argument from a caller's 7-value coefficient array.
template <typename T>
inline Coef<T> coef_from(const void* c) {
  const T* p = static_cast<const T*>(c);
  return Coef<T>{p[0], p[1], p[2], p[3], p[4], p[5], p[6], (T)-0.0};
}

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

// ----------------------------------------------------------------------
// Packed FP32x2 arithmetic (sm_100: one instruction, two lanes).  Each lane
// is rounded to nearest-even on its own, exactly like the scalar .rn ops.
//
// ptxas contracts add.rn.f32x2(mul.rn.f32x2(a, b), c) into a fused
// multiply-add even under --fmad=false (measured on B200: the pair matched
// the fused result on every input, while each op alone and the scalar .rn
// pair were exact).  The product is therefore formed as
// fma.rn.f32x2(a, b, z) with z = -0.0 supplied at run time: a*b + (-0) is
// exactly round(a*b) for every a, b (including signed zeros), the compiler
// cannot drop an addend it does not know, and an FMA result cannot be
// fused into the following add.
// ----------------------------------------------------------------------
__device__ __forceinline__ uint64_t pack2(float lo, float hi) {
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
  return d;
}
__device__ __forceinline__ void unpack2(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
// round(a*b) per lane; z must hold -0.0 in both lanes.
__device__ __forceinline__ uint64_t mul2_rn(uint64_t a, uint64_t b,
                                            uint64_t z) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(z));
  return d;
}
__device__ __forceinline__ uint64_t add2_rn(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// Coefficients broadcast into both lanes of a packed pair.
struct Coef2 {
  uint64_t ce, cw, cn, cs, ct, cb, cc, nz;
};
__device__ __forceinline__ Coef2 coef2(const Coef<float>& k) {
  return Coef2{pack2(k.ce, k.ce), pack2(k.cw, k.cw), pack2(k.cn, k.cn),
               pack2(k.cs, k.cs), pack2(k.ct, k.ct), pack2(k.cb, k.cb),
               pack2(k.cc, k.cc), pack2(k.nz, k.nz)};
}

// `point` on two adjacent x positions at once (same order, same rounding).
__device__ __forceinline__ uint64_t point2(const Coef2& k, uint64_t c,
                                           uint64_t w, uint64_t e, uint64_t s,
                                           uint64_t n, uint64_t b,
                                           uint64_t t) {
  uint64_t v = mul2_rn(k.cc, c, k.nz);
  v = add2_rn(v, mul2_rn(k.cw, w, k.nz));
  v = add2_rn(v, mul2_rn(k.ce, e, k.nz));
  v = add2_rn(v, mul2_rn(k.cs, s, k.nz));
  v = add2_rn(v, mul2_rn(k.cn, n, k.nz));
  v = add2_rn(v, mul2_rn(k.cb, b, k.nz));
  v = add2_rn(v, mul2_rn(k.ct, t, k.nz));
  return v;
}

// The stencil on one 16-byte segment: c, n, s, b, t are the segment's own
// x positions in the centre/north/south/bottom/top planes; wl and er are
// the x neighbours just outside the segment (already clamped by the
// caller).  FP32 uses packed pairs, FP64 scalar ops; both follow `point`.
template <typename T, typename K>
__device__ __forceinline__ V16<T> point_seg(const K& k, const V16<T>& c,
                                            const V16<T>& n, const V16<T>& s,
                                            const V16<T>& b, const V16<T>& t,
                                            T wl, T er);

template <>
__device__ __forceinline__ V16<float> point_seg<float, Coef2>(
    const Coef2& k, const V16<float>& c, const V16<float>& n,
    const V16<float>& s, const V16<float>& b, const V16<float>& t, float wl,
    float er) {
  const uint64_t c01 = pack2(c.e[0], c.e[1]), c23 = pack2(c.e[2], c.e[3]);
  const uint64_t mid = pack2(c.e[1], c.e[2]);  // w of 2..3 and e of 0..1
  const uint64_t w01 = pack2(wl, c.e[0]);
  const uint64_t e23 = pack2(c.e[3], er);
  const uint64_t r01 =
      point2(k, c01, w01, mid, pack2(s.e[0], s.e[1]), pack2(n.e[0], n.e[1]),
             pack2(b.e[0], b.e[1]), pack2(t.e[0], t.e[1]));
  const uint64_t r23 =
      point2(k, c23, mid, e23, pack2(s.e[2], s.e[3]), pack2(n.e[2], n.e[3]),
             pack2(b.e[2], b.e[3]), pack2(t.e[2], t.e[3]));
  V16<float> o;
  unpack2(r01, o.e[0], o.e[1]);
  unpack2(r23, o.e[2], o.e[3]);
  return o;
}

template <>
__device__ __forceinline__ V16<double> point_seg<double, Coef<double>>(
    const Coef<double>& k, const V16<double>& c, const V16<double>& n,
    const V16<double>& s, const V16<double>& b, const V16<double>& t,
    double wl, double er) {
  V16<double> o;
  o.e[0] = point(k, c.e[0], wl, c.e[1], s.e[0], n.e[0], b.e[0], t.e[0]);
  o.e[1] = point(k, c.e[1], c.e[0], er, s.e[1], n.e[1], b.e[1], t.e[1]);
  return o;
}

// Coefficient form each precision's point_seg takes.
template <typename T> struct SegCoef;
template <> struct SegCoef<float> {
  using type = Coef2;
  __device__ static Coef2 make(const Coef<float>& k) { return coef2(k); }
};
template <> struct SegCoef<double> {
  using type = Coef<double>;
  __device__ static Coef<double> make(const Coef<double>& k) { return k; }
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

// `fallback`, or the shared-memory word at p where `pred` holds: a
// predicated load with no branch around it.
__device__ __forceinline__ float ld_shared_if(bool pred, const float* p,
                                              float fallback) {
  float r = fallback;
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %1, 0;\n\t"
      "@q ld.shared.f32 %0, [%2];\n\t}"
      : "+f"(r)
      : "r"((int)pred), "r"(smem_u32(p))
      : "memory");
  return r;
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

}  // namespace d3d
