// Single-step diffusion3d kernels for sm_100a.
//
// Replaces the reference's per-step kernels (diffusion3d_cuda.cu:13-45 and
// its optimised siblings, e.g. the b/c/t register queue of :129-170 and the
// halo'd shared tiles of diffusion3d_cuda_shared1.cu:10-80) with:
//
//  * step_tma_kernel  -- the HBM-roofline path.  Each CTA owns a BX x BY xy
//    tile and marches a z-chunk.  One thread issues a TMA 3-D box load per
//    z-plane (tile + 1-row y halo + a 16-byte x halo) into a ring of
//    shared-memory stages completed through mbarriers; the other planes of
//    the ring are in flight while the CTA computes.  b and c planes of each
//    thread's 16-byte column segment live in registers (the reference's
//    t1/t2/t3 queue), x neighbours come from warp shuffles, y neighbours
//    and the next plane from shared memory, and every output row segment
//    is a 128-bit coalesced store.
//
//  * step_generic_kernel -- any shape and alignment (TMA needs 16-byte row
//    pitches): d3d::march_tile over 32x8 tiles and z-chunks, clamped load
//    addresses implementing the replicated boundary.
//
// Both evaluate d3d::point (exact reference order, no FMA), so results are
// bit-identical to Diffusion3DOpenMP::RunKernel.
#include <algorithm>
#include <cstdio>

#include "d3d_common.cuh"
#include "d3d_kernels.h"
#include "d3d_march.cuh"

namespace d3d {

// ---------------------------------------------------------------------------
// TMA-staged z-march
// ---------------------------------------------------------------------------
template <typename T, int BY, int S>
struct StepTmaCfg {
  static constexpr int WARPS = 8;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int V = 16 / sizeof(T);  // elements per 16-byte segment
  static constexpr int BX = 32 * V;         // one warp spans the tile width
  static constexpr int HX = V;              // 16-byte x halo on each side
  static constexpr int P = BX + 2 * HX;     // smem row pitch (elements)
  static constexpr int R = BY + 2;          // rows per stage (1-row y halo)
  static constexpr int RPW = BY / WARPS;    // tile rows per warp
  static constexpr int STAGE_BYTES_RAW = P * R * (int)sizeof(T);
  static constexpr int STAGE_BYTES = (STAGE_BYTES_RAW + 127) / 128 * 128;
  static constexpr int STAGE_ELEMS = STAGE_BYTES / (int)sizeof(T);
  static constexpr int SMEM = S * STAGE_BYTES + S * 8 + 128;
  static_assert(BY % WARPS == 0, "BY must be a multiple of the warp count");
  static_assert(P <= 256 && R <= 256, "TMA box dimensions are at most 256");
  static_assert(S >= 4, "the ring keeps planes z, z+1, z+2 and one in flight");
};

// FLIP: sum the y-1 neighbour 4th and y+1 5th (diffusion::Diffusion)
// instead of y+1 4th and y-1 5th (diffusion3d).
template <typename T, int BY, int S, bool FLIP>
__global__ void __launch_bounds__(StepTmaCfg<T, BY, S>::THREADS)
    step_tma_kernel(const __grid_constant__ CUtensorMap src,
                    T* __restrict__ dst, int nx, int ny, int nz, Coef<T> k,
                    int zchunk, int zb, int ze,
                    unsigned* __restrict__ dev_err) {
  using C = StepTmaCfg<T, BY, S>;
  constexpr int V = C::V;
  constexpr int RPW = C::RPW;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  T* stages = reinterpret_cast<T*>(base);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * C::STAGE_BYTES);

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int x0 = blockIdx.x * C::BX;
  const int y0 = blockIdx.y * BY;
  // Output planes [zb, ze) of the field, zchunk a CTA (the clamps below
  // use the field's own ends, 0 and nz - 1).
  const int z0 = zb + blockIdx.z * zchunk;
  const int z1 = min(ze, z0 + zchunk);
  if (z0 >= z1) return;
  const int pbase = z0 > 0 ? z0 - 1 : 0;  // first plane loaded (b of z0)
  const int plast = min(z1, nz - 1);      // last plane needed (t of z1-1)

  // p >= pbase always: unsigned arithmetic keeps these a mask and a shift.
  auto stage_of = [&](int p) { return (int)((unsigned)(p - pbase) % S); };
  auto parity_of = [&](int p) { return ((unsigned)(p - pbase) / S) & 1u; };
  auto stage_ptr = [&](int p) { return stages + stage_of(p) * C::STAGE_ELEMS; };
  auto issue = [&](int p) {
    const int s = stage_of(p);
    mbar_arrive_expect_tx(&bars[s], C::STAGE_BYTES_RAW);
    tma_load_3d(stages + s * C::STAGE_ELEMS, &src, &bars[s], x0 - C::HX,
                y0 - 1, p);
  };

  if (threadIdx.x == 0) {
    tma_prefetch_desc(&src);
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int p = pbase; p <= plast && p < pbase + S; ++p) issue(p);
  }

  // Loop-invariant addressing.  Every replicated-boundary rule becomes an
  // address: at y = 0 the north load reads the centre row, at y = ny-1 the
  // south load does, at x = 0 lane 0 reads its own first element as w; at
  // z = nz-1 the top plane is the centre plane (stage_ptr(min(z+1, nz-1))).
  const int xg = x0 + V * lane;      // first x of this thread's segment
  const int col = C::HX + V * lane;  // its shared-memory column
  const bool x_hi = (xg + V - 1 == nx - 1);
  int c_off[RPW], n_off[RPW], s_off[RPW];
  size_t g_off[RPW];
  bool store_ok[RPW];
#pragma unroll
  for (int r = 0; r < RPW; ++r) {
    const int row = warp * RPW + r;
    const int yg = y0 + row;
    c_off[r] = (row + 1) * C::P + col;
    n_off[r] = (yg == 0) ? c_off[r] : row * C::P + col;
    s_off[r] = (yg >= ny - 1) ? c_off[r] : (row + 2) * C::P + col;
    g_off[r] = (size_t)yg * nx + xg;
    store_ok[r] = (yg < ny) && (xg < nx);
    if constexpr (FLIP) {
      const int t = n_off[r];
      n_off[r] = s_off[r];
      s_off[r] = t;
    }
  }
  const int wl_adj = (xg == 0) ? 0 : -1;  // lane 0's w load
  const size_t plane = (size_t)nx * ny;
  const typename SegCoef<T>::type kk = SegCoef<T>::make(k);

  // Register queue: three rotating sets of RPW segments (b, c, t roles),
  // unrolled three ways so no values are copied between iterations.
  V16<T> q0[RPW], q1[RPW], q2[RPW];
  int drain_lo = pbase, drain_hi = min(plast, pbase + S - 1);

  // Prologue: planes z0 (c) and z0-1 (b), and z0+1 (t of the first step).
  // (Every thread waits here: measured on B200, a single waiting thread
  // plus the barrier was no faster for this kernel and cost registers.)
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
    const T* sc = stage_ptr(z0);
    const T* sb = stage_ptr(pbase);  // == sc when z0 == 0 (b = c at z = 0)
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
      q1[r] = ld16_shared(sc + c_off[r]);
      q0[r] = ld16_shared(sb + c_off[r]);
    }
  }
  __syncthreads();
  if (z0 > 0 && threadIdx.x == 0 && pbase + S <= plast) issue(pbase + S);

  {
    // One z step: b, c in registers, t loaded into `vt`; then wait for the
    // next t plane and recycle plane z's stage.  Returns false on timeout.
    auto step = [&](int z, const V16<T>* vb, const V16<T>* vc,
                    V16<T>* vt) -> bool {
      const T* sc = stage_ptr(z);
      const T* st = stage_ptr(min(z + 1, nz - 1));
      T* out = dst + (size_t)z * plane;
#pragma unroll
      for (int r = 0; r < RPW; ++r) {
        vt[r] = ld16_shared(st + c_off[r]);
        const V16<T> n = ld16_shared(sc + n_off[r]);
        const V16<T> s = ld16_shared(sc + s_off[r]);
        T wl = __shfl_up_sync(0xffffffffu, vc[r].e[V - 1], 1);
        T er = __shfl_down_sync(0xffffffffu, vc[r].e[0], 1);
        if (lane == 0) wl = sc[c_off[r] + wl_adj];
        if (lane == 31) er = sc[c_off[r] + V];
        if (x_hi) er = vc[r].e[V - 1];
        const V16<T> o = point_seg<T>(kk, vc[r], n, s, vb[r], vt[r], wl, er);
        if (store_ok[r]) st16_global(out + g_off[r], o);
      }
      // Plane z+2 is the t plane of the next step; wait for it before the
      // barrier that releases plane z's stage to the producer.
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

    int zf = -1;  // the step whose wait ran out
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
  // A wait ran out: let every load this CTA issued and has not yet waited
  // for land before its shared memory is released.  Bounded as well.
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
// Generic kernel: any nx, ny, nz, any alignment -- d3d::march_tile over a
// 32 x 8 tile and a z-chunk (d3d_march.cuh).
// ---------------------------------------------------------------------------
// FP32: two cells per thread on 64 x 8 tiles (packed arithmetic);
// FP64: one cell per thread on 32 x 8 tiles.
template <typename T> struct GenTile;
template <> struct GenTile<float> { static constexpr int BX = 64, BY = 8; };
template <> struct GenTile<double> { static constexpr int BX = 32, BY = 8; };

template <typename T, bool FLIP>
__global__ void __launch_bounds__(256)
    step_generic_kernel(const T* __restrict__ src, T* __restrict__ dst,
                        int nx, int ny, int nz, Coef<T> k, int zchunk,
                        int zb, int ze) {
  constexpr int BX = GenTile<T>::BX, BY = GenTile<T>::BY;
  const int z0 = zb + blockIdx.z * zchunk;
  const int z1 = min(ze, z0 + zchunk);
  if (z0 >= z1) return;
  if constexpr (sizeof(T) == 4) {
    __shared__ __align__(16) float stage[2][MarchTile2<BX, BY>::E];
    march_tile2<BX, BY, FLIP>(src, dst, nx, ny, nz, blockIdx.x * BX,
                              blockIdx.y * BY, z0, z1, k, stage);
  } else {
    __shared__ double stage[2][MarchTile<BX, BY>::E];
    march_tile<double, BX, BY, FLIP>(src, dst, nx, ny, nz, blockIdx.x * BX,
                                     blockIdx.y * BY, z0, z1, k, stage);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

// (rows per tile, planes in the ring).  Variant 0 is the default for tall
// grids: at 512^3 FP32 it runs two 256-thread CTAs per SM and measured the
// fastest of these on B200.
const TmaVariant kTmaVariants[kNumTmaVariants] = {
    {32, 4}, {16, 4}, {8, 4}, {16, 6}, {32, 6}, {8, 8}};

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t,
                                  void*, const cuuint64_t*, const cuuint64_t*,
                                  const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p,
                                cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

}  // namespace

cudaError_t current_context(void** ctx) {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault,
                                &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<CtxGetCurrentFn>(p);
    return static_cast<CtxGetCurrentFn>(nullptr);
  }();
  *ctx = nullptr;
  if (!fn) return cudaErrorNotSupported;
  CUcontext c = nullptr;
  if (fn(&c) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  *ctx = c;
  return cudaSuccess;
}

namespace {

int num_sms() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

// z-chunk so that all CTAs of one step are resident at once (one wave),
// with chunks of at least `min_chunk` planes.
int pick_zchunk(int nz, long tiles, int ctas_per_sm, int min_chunk) {
  long capacity = (long)num_sms() * std::max(ctas_per_sm, 1);
  long zs = std::max(1L, capacity / std::max(tiles, 1L));
  zs = std::min<long>(zs, std::max(1, nz / min_chunk));
  return (int)((nz + zs - 1) / zs);
}

// z-chunk of the TMA z-march: short chunks (16 planes FP32, 12 FP64) when
// they make at least four waves of CTAs, else pick_zchunk's single wave.
// Many short chunks keep every SM busy to the end of the step; a single
// wave leaves the SMs it does not fill idle.  Measured on B200
// (Gpt-updates/s, one wave against short chunks, short runs): FP32 768^3
// 706-731 / 769-795, 1024 x 1024 x 130 758 / 757-768; FP64 512^3 303-315 /
// 347-357.  At 512^3 FP32, sustained over 0.8 s under the power cap, one
// wave and 16-plane chunks tie (720.1 / 719.5, five alternating rounds)
// while 12-plane chunks draw more power and run 1% slower (712.9).
int pick_tma_zchunk(int nz, long tiles, int ctas_per_sm, int fine) {
  const long capacity = (long)num_sms() * std::max(ctas_per_sm, 1);
  const long ctas = tiles * ((nz + fine - 1) / fine);
  if (ctas >= 4 * capacity) return fine;
  return pick_zchunk(nz, tiles, ctas_per_sm, 8);
}

template <typename T, int BY, int S, bool FLIP>
cudaError_t launch_tma_t(const CUtensorMap& src, void* f2, int nx, int ny,
                         int nz, const void* coef, int zchunk_override,
                         int zb, int ze,
                         cudaStream_t stream, unsigned* dev_err,
                         LaunchInfo* info) {
  using C = StepTmaCfg<T, BY, S>;
  auto kern = step_tma_kernel<T, BY, S, FLIP>;
  static bool attr_set = false;  // per instantiation; same on every device
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, C::THREADS,
                                                C::SMEM);
  const int gx = (nx + C::BX - 1) / C::BX;
  const int gy = (ny + BY - 1) / BY;
  const int nzr = ze - zb;
  const int zchunk = zchunk_override > 0
                         ? zchunk_override
                         : pick_tma_zchunk(nzr, (long)gx * gy, occ,
                                           sizeof(T) == 8 ? 12 : 16);
  const int gz = (nzr + zchunk - 1) / zchunk;
  if (info) *info = LaunchInfo{gx, gy, gz, C::THREADS, C::SMEM, zchunk, occ};
  kern<<<dim3(gx, gy, gz), C::THREADS, C::SMEM, stream>>>(
      src, static_cast<T*>(f2), nx, ny, nz, coef_from<T>(coef), zchunk, zb,
      ze, dev_err);
  return cudaGetLastError();
}

template <typename T, bool F>
cudaError_t launch_tma_dtype(const CUtensorMap& src, void* f2, int nx, int ny,
                             int nz, const void* coef, int variant,
                             int zchunk_override, int zb, int ze,
                             cudaStream_t stream, unsigned* dev_err,
                             LaunchInfo* info) {
  switch (variant) {
    case 0: return launch_tma_t<T, 32, 4, F>(src, f2, nx, ny, nz, coef, zchunk_override, zb, ze, stream, dev_err, info);
    case 1: return launch_tma_t<T, 16, 4, F>(src, f2, nx, ny, nz, coef, zchunk_override, zb, ze, stream, dev_err, info);
    case 2: return launch_tma_t<T, 8, 4, F>(src, f2, nx, ny, nz, coef, zchunk_override, zb, ze, stream, dev_err, info);
    case 3: return launch_tma_t<T, 16, 6, F>(src, f2, nx, ny, nz, coef, zchunk_override, zb, ze, stream, dev_err, info);
    case 4: return launch_tma_t<T, 32, 6, F>(src, f2, nx, ny, nz, coef, zchunk_override, zb, ze, stream, dev_err, info);
    case 5: return launch_tma_t<T, 8, 8, F>(src, f2, nx, ny, nz, coef, zchunk_override, zb, ze, stream, dev_err, info);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

const TmaVariant& tma_variant(int i) { return kTmaVariants[i]; }

int default_tma_variant(int nx, int ny, int nz, int dtype) {
  // The tallest tile (32, 16 or 8 rows) that still gives two resident CTAs
  // per SM with z-chunks of 8 planes or more: at 256^3 and up that is the
  // 32-row tile (the fastest measured); small grids need shorter tiles to
  // fill the GPU (128^3: 8-row tiles, 355 against 216 Gpt/s).
  // FP64 starts at 16 rows: its 32-row tiles measured slower on B200 at
  // every size from 256^3 to 512^3 (512^3: 341 against 357 Gpt/s, both at
  // 12-plane chunks).
  const long bx = 32L * (16 / (long)dtype_size(dtype));
  const long cap = 2L * num_sms();
  const long zslabs = std::max(1, nz / 8);
  const int order[3] = {0, 1, 2};  // by = 32, 16, 8
  for (int v : order) {
    if (v == 0 && dtype_size(dtype) == 8) continue;
    const long by = kTmaVariants[v].by;
    const long tiles = ((nx + bx - 1) / bx) * ((ny + by - 1) / by) * zslabs;
    if (tiles >= cap) return v;
  }
  return 2;
}

int tma_box_x(int dtype) {
  const int v = 16 / (int)dtype_size(dtype);
  return 32 * v + 2 * v;
}
int tma_box_y(int variant) { return kTmaVariants[variant].by + 2; }

bool tma_eligible(const void* ptr, int nx, int ny, int dtype) {
  const size_t es = dtype_size(dtype);
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) != 0) return false;
  if (((size_t)nx * es) % 16 != 0) return false;  // row pitch, 16-byte rule
  (void)ny;
  return encode_fn() != nullptr;
}

cudaError_t encode_field_map(CUtensorMap* map, const void* ptr, int nx, int ny,
                             int nz, int dtype, int box_x, int box_y) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  const size_t es = dtype_size(dtype);
  cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  cuuint64_t strides[2] = {(cuuint64_t)nx * es, (cuuint64_t)nx * ny * es};
  cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map,
                  dtype == kF64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  3, const_cast<void*>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_step_tma(const CUtensorMap& src, void* f2, int nx, int ny,
                            int nz, const void* coef, int dtype, int variant,
                            int zchunk_override, int flip_y,
                            cudaStream_t stream, unsigned* dev_err,
                            LaunchInfo* info, int zb, int ze) {
  if (ze < 0) ze = nz;
  if (zb < 0 || zb >= ze || ze > nz) return cudaErrorInvalidValue;
  auto run = [&](auto fn) {
    return fn(src, f2, nx, ny, nz, coef, variant, zchunk_override, zb, ze,
              stream, dev_err, info);
  };
  if (dtype == kF64)
    return flip_y ? run(launch_tma_dtype<double, true>)
                  : run(launch_tma_dtype<double, false>);
  return flip_y ? run(launch_tma_dtype<float, true>)
                : run(launch_tma_dtype<float, false>);
}

cudaError_t launch_step_generic(const void* f1, void* f2, int nx, int ny,
                                int nz, const void* coef, int dtype,
                                int flip_y, cudaStream_t stream,
                                LaunchInfo* info, int zb, int ze) {
  if (ze < 0) ze = nz;
  if (zb < 0 || zb >= ze || ze > nz) return cudaErrorInvalidValue;
  const int bx = dtype == kF64 ? GenTile<double>::BX : GenTile<float>::BX;
  const int by = dtype == kF64 ? GenTile<double>::BY : GenTile<float>::BY;
  const int gx = (nx + bx - 1) / bx;
  const int gy = (ny + by - 1) / by;
  // 24-plane chunks when they make four or more waves (8 CTAs an SM),
  // else one wave of chunks of 32 planes or more.  Measured on B200
  // (Gpt-updates/s, one wave against 24-plane chunks): FP32 511^3 551 /
  // 622, 767^3 566 / 618; FP64 511^3 290 / 354.
  constexpr int kFine = 24;
  const long tiles = (long)gx * gy;
  const int zchunk =
      tiles * ((ze - zb + kFine - 1) / kFine) >= 4L * num_sms() * 8
          ? kFine
          : pick_zchunk(ze - zb, tiles, 8, 32);
  const int gz = (ze - zb + zchunk - 1) / zchunk;
  if (info) *info = LaunchInfo{gx, gy, gz, 256, 0, zchunk, 8};
  dim3 grid(gx, gy, gz), block(256);
  auto go = [&](auto kern, auto* a, auto* b, auto k) {
    kern<<<grid, block, 0, stream>>>(a, b, nx, ny, nz, k, zchunk, zb, ze);
  };
  const double* d1 = static_cast<const double*>(f1);
  const float* s1 = static_cast<const float*>(f1);
  if (dtype == kF64) {
    double* d2 = static_cast<double*>(f2);
    if (flip_y)
      go(step_generic_kernel<double, true>, d1, d2, coef_from<double>(coef));
    else
      go(step_generic_kernel<double, false>, d1, d2, coef_from<double>(coef));
  } else {
    float* s2 = static_cast<float*>(f2);
    if (flip_y)
      go(step_generic_kernel<float, true>, s1, s2, coef_from<float>(coef));
    else
      go(step_generic_kernel<float, false>, s1, s2, coef_from<float>(coef));
  }
  return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// HBM calibration: out = cc * in, the stencil's own traffic (4 bytes read,
// 4 written per point) with no neighbours -- the measured ceiling the step
// kernels are compared against.  The reference's DiffusionCUDACopy
// (diffusion/diffusion_cuda_copy.cu:8-24) plays this role there.  16-byte
// loads and stores in a grid-stride loop when both pointers are 16-byte
// aligned, a scalar tail after them (or scalar throughout otherwise).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    scale_copy_kernel(const float* __restrict__ in, float* __restrict__ out,
                      size_t n, float cc, bool vec) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t done = 0;
  if (vec) {
    const size_t nq = n / 4;
    const float4* qi = reinterpret_cast<const float4*>(in);
    float4* qo = reinterpret_cast<float4*>(out);
    for (size_t q = i; q < nq; q += stride) {
      const float4 v = qi[q];
      qo[q] = make_float4(__fmul_rn(cc, v.x), __fmul_rn(cc, v.y),
                          __fmul_rn(cc, v.z), __fmul_rn(cc, v.w));
    }
    done = nq * 4;
  }
  for (size_t j = done + i; j < n; j += stride) out[j] = __fmul_rn(cc, in[j]);
}

cudaError_t launch_scale_copy(const float* in, float* out, size_t n, float cc,
                              cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const bool vec = ((reinterpret_cast<uintptr_t>(in) |
                     reinterpret_cast<uintptr_t>(out)) & 15) == 0;
  // Eight 256-thread CTAs per SM, each thread a few 16-byte loads in flight.
  const int blocks = num_sms() * 8;
  scale_copy_kernel<<<blocks, 256, 0, s>>>(in, out, n, cc, vec);
  return cudaGetLastError();
}

}  // namespace d3d
