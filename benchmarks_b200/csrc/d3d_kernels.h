// Host-side declarations of the kernel launchers inside libd3d_b200.so.
// Not part of the public C ABI (include/d3d_b200.h is).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>

namespace d3d {

// Error and launch bookkeeping shared by every C-ABI translation unit
// (defined in d3d_api.cu): the calling thread's last-error text and the
// process-wide count of kernel launches.
int set_error(int code, const char* fmt, ...);
int set_cuda_error(cudaError_t e, const char* what);
void note_launches(unsigned long long n);

enum Dtype { kF32 = 0, kF64 = 1 };

inline size_t dtype_size(int dtype) { return dtype == kF64 ? 8 : 4; }

// Tile configurations of the TMA-staged single-step kernel.
struct TmaVariant {
  int by;      // rows of the xy tile
  int stages;  // planes in the shared-memory ring
};
constexpr int kNumTmaVariants = 6;
// Default tile variant for an nx*ny*nz grid of `dtype`.
int default_tma_variant(int nx, int ny, int nz, int dtype);
const TmaVariant& tma_variant(int i);

// Launch geometry actually used (for reporting and for the autotuner).
struct LaunchInfo {
  int grid_x, grid_y, grid_z;
  int block;
  int smem_bytes;
  int zchunk;
  int ctas_per_sm;
};

bool tma_eligible(const void* ptr, int nx, int ny, int dtype);

// Encodes a 3-D tiled tensor map over a field for the TMA kernels.
// box = (tile_x + 2*halo_x) x (tile_y + 2*halo_y) x 1.
cudaError_t encode_field_map(CUtensorMap* map, const void* ptr, int nx, int ny,
                             int nz, int dtype, int box_x, int box_y);

// Every 3D launcher takes `flip_y`: 0 sums the y+1 neighbour 4th and y-1
// 5th (diffusion3d, diffusion3d_openmp.cc:57-62); 1 sums y-1 4th and y+1
// 5th (the diffusion::Diffusion surface, diffusion_openmp.cc:98-103).

// out = cc * in over n floats (HBM calibration at the stencil's 8 bytes
// per point).
cudaError_t launch_scale_copy(const float* in, float* out, size_t n, float cc,
                              cudaStream_t s);

// One time step, f2 = stencil(f1), with the TMA-staged z-march.  Only
// output planes [zb, ze) are written (ze < 0: nz); the boundary clamps
// stay at the field's own ends.
cudaError_t launch_step_tma(const CUtensorMap& src, void* f2, int nx, int ny,
                            int nz, const void* coef, int dtype, int variant,
                            int zchunk_override, int flip_y,
                            cudaStream_t stream, unsigned* dev_err,
                            LaunchInfo* info, int zb = 0, int ze = -1);
int tma_box_x(int dtype);
int tma_box_y(int variant);

// One time step with the generic kernel (any shape, any alignment).
cudaError_t launch_step_generic(const void* f1, void* f2, int nx, int ny,
                                int nz, const void* coef, int dtype,
                                int flip_y, cudaStream_t stream,
                                LaunchInfo* info, int zb = 0, int ze = -1);

// One 2D 5-point time step (diffusion::Diffusion with nd = 2), any shape
// and alignment; ychunk_override = rows per warp task (0 = automatic).
struct Step2dVariant {
  int ring;  // rows in each lane's register ring
};
constexpr int kNumStep2dVariants = 6;
extern const Step2dVariant kStep2dVariants[kNumStep2dVariants];
int default_step2d_variant();
cudaError_t launch_step2d(const void* f1, void* f2, int nx, int ny,
                          const void* coef, int dtype, int variant,
                          int ychunk_override, cudaStream_t stream,
                          LaunchInfo* info);
// The widest access (in values, 16 bytes at most) that nx and the buffers'
// alignment allow; the 2D kernel uses vector accesses when it is 16 bytes.
int step2d_vector_width(const void* f1, const void* f2, int nx, int dtype);

// k fused time steps (temporal blocking), f2 = stencil^k(f1).
cudaError_t launch_steps_tb(const CUtensorMap& src, void* f2, int nx, int ny,
                            int nz, const void* coef, int dtype, int k,
                            int zchunk_override, int flip_y,
                            cudaStream_t stream, unsigned* dev_err,
                            LaunchInfo* info);
int tb_box_x(int dtype, int k);
int tb_box_y(int k);
bool tb_supported(int k, int dtype);

// Two fused steps, FP32, warp-row tiles (d3d_tb2.cu): the default TB
// kernel for K = 2 in FP32; the generic-K kernel stays selectable.
cudaError_t launch_steps_tb2w(const CUtensorMap& src, void* f2, int nx,
                              int ny, int nz, const void* coef,
                              int zchunk_override, int flip_y,
                              cudaStream_t stream, unsigned* dev_err,
                              LaunchInfo* info);
int tb2w_box_x();
int tb2w_box_y();

// FP64-accumulated comparison of two device fields (any dtype pair):
// out[0] = rms(a-b), out[1] = max|a-b|, out[2] = max|a-b|/|b|, out[3] = sum(a).
// `scratch` holds `compare_scratch_bytes()` bytes of device memory.
size_t compare_scratch_bytes();
cudaError_t launch_compare(const void* a, int a_dtype, const void* b,
                           int b_dtype, size_t n, double* scratch,
                           cudaStream_t stream);

// The allocation-free comparison: same outputs as launch_compare, partial
// sums in a fixed file-scope device array (n <= compare_noalloc_max_elements).
size_t compare_noalloc_max_elements();
cudaError_t noalloc_scratch(double** out);
cudaError_t launch_compare_noalloc(const void* a, int a_dtype, const void* b,
                                   int b_dtype, size_t n, double* scratch,
                                   cudaStream_t stream);

// One grid of a multi-grid step launch: step `parity` reads a (parity 0)
// or b (parity 1) and writes the other.  A work item (grid, tile) names
// xy tile `tile % tiles_xy` (x fastest, tiles_x per row) and z slab
// `tile / tiles_xy` of `zc` planes.
struct BatchDesc {
  float* a;
  float* b;
  int nx, ny, nz, tiles_x;
  int tiles_xy, zc;
  float k[8];  // ce, cw, cn, cs, ct, cb, cc, and -0.0
};

// One grid of a pitched multi-grid TMA launch (the solve server's layout):
// rows of px >= nx floats (px a multiple of 4), pads x in [nx, px) holding
// copies of column nx-1; map[0] / map[1] cover a / b as px x ny x nz
// fields.  Items as for BatchDesc.
struct alignas(64) PitchedDesc {
  CUtensorMap map[2];
  float* a;
  float* b;
  int nx, px, ny, nz, tiles_x, tiles_xy, zc, unused;
  int seg_w, rows;  // strip form: segments per piece, rows per strip
  float k[8];       // ce, cw, cn, cs, ct, cb, cc, and -0.0
};

// Tile shapes of the pitched kernel: `lanes` per tile row (tile width
// 4 * lanes), `by` rows, `stages` planes in the TMA ring.
struct PitchedVariant {
  int lanes, by, stages;
};
constexpr int kNumPitchedVariants = 5;
const PitchedVariant& pitched_variant(int v);
int pitched_box_x(int v);
int pitched_box_y(int v);

// One time step for `nitems` (grid, tile) work items of pitched grids.
cudaError_t launch_pitched_step(int variant, const PitchedDesc* descs,
                                const int2* items, int nitems, int parity,
                                cudaStream_t s, unsigned* dev_err);

// Strip form of the pitched kernel (NR = 1 or 2 segments a thread): a CTA
// covers `rows` whole rows of one of `pieces` near-equal pieces of the
// pitch (segs 16-byte segments each) and a z slab; items as for the tile
// form, with tiles_x = pieces and tiles_xy = pieces * ceil(ny / rows).
// Tensor-map box: (4 * segs + 8) x (rows + 2).
constexpr int kStripMaxW = 248;  // columns per piece: box width <= 256
__host__ __device__ constexpr int strip_stage_bytes(int nr) {
  return nr * 6656;
}
struct StripShape {
  int pieces, segs, rows;
};
StripShape strip_shape(int px, int ny, int nr);
cudaError_t launch_pitched_strip(int nr, const PitchedDesc* descs,
                                 const int2* items, int nitems, int parity,
                                 cudaStream_t s, unsigned* dev_err);

// Two fused steps per pass, strip form (NR = 1 or 2 level-2 segments a
// thread), for grids whose pitch is one piece (px <= kStripMaxW; pieces = 0
// from strip2_shape otherwise).  Items: tiles_x = 1, tiles_xy = strips,
// zc = z slab.  Tensor-map box: (px + 8) x (rows + 4), from y0 - 2.  A
// pass reads map[parity] and writes the other buffer two steps later.
__host__ __device__ constexpr int strip2_slot_bytes(int nr) {
  return nr * 6656;
}
StripShape strip2_shape(int px, int ny, int nr);
cudaError_t launch_pitched_strip2(int nr, const PitchedDesc* descs,
                                  const int2* items, int nitems, int parity,
                                  cudaStream_t s, unsigned* dev_err);

// One grid of a multi-grid repitch: `rows` (= ny * nz) rows of nx floats
// at `dense`, px floats at `pitched`.
struct RepitchDesc {
  float* dense;
  float* pitched;
  int nx, px;
  long long rows;
};
// Dense -> pitched (pads filled from column nx-1) when to_pitched, else
// pitched -> dense, for n grids in one launch.
cudaError_t launch_repitch_multi(const RepitchDesc* d, int n,
                                 bool to_pitched, cudaStream_t s);

// Dense rows (nx floats) -> pitched rows (px floats, pads filled from
// column nx-1) when to_pitched, else pitched -> dense; rows = ny * nz.
// src and dst must not overlap.
cudaError_t launch_repitch(const float* src, float* dst, int nx, int px,
                           long long rows, bool to_pitched, cudaStream_t s);

// One grid of the cluster-resident multi-grid kernel (d3d_resident.cu):
// dense fields in and out (out may equal in), the pitch px = ceil4(nx) and
// segs = px / 4 of its shared-memory rows, pc planes per CTA of its
// cluster, and the index of its step counter.
struct ResidentDesc {
  const float* in;
  float* out;
  int nx, ny, nz, steps;
  int px, segs, pc, grid_id;
  int yparts, rows;  // row parts of a plane (1, 2 or 4), rows in a part
  float k[8];        // ce, cw, cn, cs, ct, cb, cc, and -0.0
};
// Thread shapes: `threads` a CTA, at most `units` 16-byte row segments of
// a plane a thread (a plane of segs * ny segments fits when
// segs * ny <= threads * units).
struct ResidentVariant {
  int threads, units;
};
constexpr int kNumResidentVariants = 5;
// Launch variant ids: the shape index, plus kResidentParts for the build
// with row parts (shapes 0..2 only).
constexpr int kResidentParts = kNumResidentVariants;
constexpr int kResidentMaxCluster = 16;
// Dynamic shared memory a CTA may hold: its pc planes and a halo plane.
constexpr size_t kResidentSmemMax = 232448 - 1024;
const ResidentVariant& resident_variant(int v);
// Launch class of one grid on the resident kernel: a thread shape and a
// cut of each plane into 1, 2 or 4 row parts (`rows` rows each) such that
// a CTA's ceil(nx/4) * rows row segments are covered and the grid fits in
// at most 16 CTAs (yparts row parts times z slabs of pc planes, plus a halo
// plane each) within the shared memory a CTA of that shape may take -- a
// share of the SM for the 128- and 256-thread shapes, so that 512 threads
// run on an SM.  Narrow shapes and whole planes are preferred.  False: no
// shape fits the grid.
struct ResidentFit {
  int cluster, variant, pc, px, yparts, rows;
  size_t smem;
};
bool resident_fit(int nx, int ny, int nz, ResidentFit* fit);
// Opts the kernels into the full shared memory and 16-CTA clusters on the
// current device (once per device).
cudaError_t resident_prepare();
// Clusters of `cluster` CTAs with `smem` bytes each that fit on the GPU at
// once (0: not schedulable).
cudaError_t resident_max_clusters(int variant, int cluster, size_t smem,
                                  int* out);
// A persistent launch of `nclusters` clusters walking descs[0, ngrids)
// through the work counter *queue (zero it before the launch).
cudaError_t launch_resident(int variant, const ResidentDesc* descs,
                            int ngrids, unsigned* queue, int* steps_done,
                            int cluster, int nclusters, size_t smem,
                            cudaStream_t s);

// counters[id_steps[i].x] = id_steps[i].y for i < n: the step counters
// of grids that ran on the per-step path, set after its last launch.
cudaError_t launch_set_counters(const int2* id_steps, int n, int* counters,
                                cudaStream_t s);

// This device's kernel error word (bounded-wait failures).
unsigned* device_error_word();

// The driver context current on the calling thread (null when the runtime
// has not made one current yet).  Device addresses of file-scope
// __device__ variables are cached per context with it.
cudaError_t current_context(void** ctx);

// Tile shapes of the multi-grid step kernel (256 threads each).
struct BShape {
  int bx, by;
};
constexpr int kNumBShapes = 4;
extern const BShape kBShapes[kNumBShapes];

// One time step for `nitems` (grid, tile) work items.
cudaError_t launch_batch_step(int shape, const BatchDesc* descs,
                              const int2* items, int nitems, int parity,
                              cudaStream_t s);

// FP64 error norms of a field against the analytic solution at `time`,
// evaluated per point (no analytic buffer); result in scratch[0..3].
// ndim = 2 drops the z factor (the 2D field of diffusion::Diffusion).
cudaError_t launch_accuracy(const void* f, int dtype, int ndim, int nx,
                            int ny, int nz, double kx, double ky, double kz,
                            double dx, double dy, double dz, double kappa,
                            double time, double* scratch,
                            cudaStream_t stream);

// What the checkpoint code needs of a plan.
struct PlanShape {
  int nx, ny, nz, ndim, flip_y, dtype;
  size_t n;
};
// Binary checkpoints (d3d_io.cu).  `scratch` is compare_scratch_bytes() of
// device memory; the device forms synchronise `s`.
int checkpoint_save(const PlanShape& ps, double* scratch, const void* field,
                    long long step, const char* path, cudaStream_t s);
int checkpoint_load(const PlanShape& ps, double* scratch, const char* path,
                    void* field, long long* step, cudaStream_t s);
int checkpoint_save_host(const PlanShape& ps, const void* host_field,
                         long long step, const char* path);

// A one-CTA kernel whose bounded mbarrier wait is bound to run out.
cudaError_t launch_selftest_wait(unsigned limit, unsigned* dev_err,
                                 cudaStream_t stream);

// Analytic solution (the reference's Initialize, computed in FP64 on the
// device) written in `dtype` at `time`.
cudaError_t launch_analytic(void* out, int dtype, int ndim, int nx, int ny,
                            int nz, double kx, double ky, double kz,
                            double dx, double dy, double dz, double kappa,
                            double time, cudaStream_t stream);

}  // namespace d3d
