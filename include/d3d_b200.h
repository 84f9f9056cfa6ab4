/*
 * d3d_b200.h -- C ABI of libd3d_b200.so, the B200 (sm_100a) backend of the
 * diffusion3d 7-point stencil.
 *
 * This is the boundary a Diffusion3DB200 subclass of the reference's
 * diffusion3d::Baseline (src/diffusion3d/baseline.h:8-22) binds: plain C,
 * plain pointers and sizes, no CUDA or C++ types in any signature
 * (streams are passed as `void*` holding a cudaStream_t; NULL = default
 * stream).  Each entry point names the reference code it replaces.
 *
 * Conventions
 *  - Fields are x-fastest, offset(i,j,k) = i + j*nx + k*nx*ny, no padding
 *    (the reference's OFFSET3D, src/diffusion3d/diffusion3d.h:33-34).
 *  - `coeff` points at 7 values of the plan's dtype in the reference's
 *    member order ce, cw, cn, cs, ct, cb, cc (diffusion3d.h:52).
 *  - Every entry returns an int status: D3D_OK (0) or a negative D3D_E_*.
 *    d3d_last_error() gives the text of the calling thread's last failure.
 *    The reference's own convention is assert/exit (diffusion3d_cuda.cu:6-9);
 *    nothing here aborts the process.
 *  - Results are bit-identical to the reference's Diffusion3DOpenMP for
 *    FP32 (same operation order, no FMA contraction).
 *  - A plan is not thread-safe; use one plan per host thread.
 */
#ifndef D3D_B200_H_
#define D3D_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  D3D_OK = 0,
  D3D_E_INVALID = -1,     /* bad dimensions, pointer or argument */
  D3D_E_CUDA = -2,        /* a CUDA runtime call failed */
  D3D_E_OOM = -3,         /* device or pinned allocation failed */
  D3D_E_TIMEOUT = -4,     /* a bounded device wait ran out */
  D3D_E_UNSUPPORTED = -5, /* shape/dtype/kernel combination not supported */
  D3D_E_BUSY = -6,        /* admission refused (serving) */
  D3D_E_IO = -7,          /* a checkpoint file could not be written or read,
                             or failed its checksum */
  D3D_E_TRANSPORT = -8    /* a z-slab transport callback reported failure */
};

enum { D3D_F32 = 0, D3D_F64 = 1 };

enum {
  D3D_KERNEL_AUTO = 0,    /* TMA z-march when eligible, else generic;
                             FP32 3D grids of 2^27+ points run pairs of
                             steps as fused two-step passes (faster there
                             on B200, same bits) */
  D3D_KERNEL_GENERIC = 1, /* any shape / alignment */
  D3D_KERNEL_TMA = 2,     /* TMA-staged z-march (row pitch % 16 B == 0) */
  D3D_KERNEL_TB = 3       /* temporal blocking: tb_depth fused steps/pass */
};

typedef struct d3d_plan_s* d3d_plan;

/* Library version string. */
const char* d3d_version(void);

/* Text of the calling thread's most recent failure ("" if none). */
const char* d3d_last_error(void);

/* Number of kernels this library has launched in this process. */
unsigned long long d3d_launch_count(void);

/* The coefficients and geometry the reference constructor derives for an
 * nx*ny*nz grid (Diffusion3D::Diffusion3D, diffusion3d.h:54-66), in the
 * plan dtype: coeff7 = ce,cw,cn,cs,ct,cb,cc; geom8 = kappa,dx,dy,dz,kx,ky,kz,dt.
 * Either output may be NULL. */
int d3d_coefficients(int nx, int ny, int nz, int dtype, void* coeff7,
                     void* geom8);

/* Creates a plan for one grid shape and precision: the launch
 * configuration the reference keeps in Diffusion3DCUDA (block_x_, block_y_,
 * grid_z_; diffusion3d_cuda.h:44-47).  kernel = D3D_KERNEL_*; tb_depth is
 * the fused step count for D3D_KERNEL_TB (2..4), ignored otherwise.
 * The plan binds to the CUDA device current at creation. */
int d3d_plan_create(int nx, int ny, int nz, int dtype, int kernel,
                    int tb_depth, d3d_plan* out);

/* ---------------------------------------------------------------------
 * The reference's second plugin surface, diffusion::Diffusion
 * (src/diffusion/diffusion.h:80-180): nd = 2 (5-point, nx*ny) or nd = 3
 * (7-point) grids, dims = {nx, ny[, nz]} as its constructor
 * Diffusion(int ndim, const int* dims) takes them (diffusion.h:93-108).
 * Two arithmetic differences from diffusion3d, both reproduced:
 *   - cc = 1.0 - (ce + cw + cn + cs + (nd == 3 ? ct + cb : 0))
 *     (diffusion.h:107), which can round differently from diffusion3d's;
 *   - the y-1 neighbour is summed before y+1: f = cc*c + cw*w + ce*e +
 *     cs*s + cn*n [+ cb*b + ct*t] with s = y-1, n = y+1
 *     (diffusion_openmp.cc:71-74, 98-103).
 * ------------------------------------------------------------------- */

/* The coefficients and geometry diffusion::Diffusion derives for an nd-D
 * grid (ct, cb and dz are those of a one-plane z axis when nd = 2 and go
 * unused).  Same output layout as d3d_coefficients. */
int d3d_diffusion_coefficients(int nd, const int* dims, int dtype,
                               void* coeff7, void* geom8);

/* A plan for a diffusion::Diffusion grid: the launch state
 * DiffusionCUDA keeps (diffusion_cuda.h:30-61).  Every d3d_plan entry point
 * below works on it (step, run, run_host, autotune, analytic, compare,
 * accuracy).  nd = 3 runs the 3D kernels in this surface's order and takes
 * any kernel; nd = 2 runs the 2D register-march kernel and takes
 * D3D_KERNEL_AUTO or D3D_KERNEL_GENERIC (D3D_E_UNSUPPORTED otherwise). */
int d3d_diffusion_plan_create(int nd, const int* dims, int dtype, int kernel,
                              int tb_depth, d3d_plan* out);

/* Overrides the tile variant (0..D3D_NUM_TILE_VARIANTS-1) and z-chunk
 * (planes per CTA, 0 = automatic) of a plan; used by the autotuner.  On a
 * 2D plan the variant picks the 2D kernel's register-ring depth and zchunk
 * is the rows per warp task. */
#define D3D_NUM_TILE_VARIANTS 6
int d3d_plan_set_tile(d3d_plan plan, int variant, int zchunk);

/* Enables (default) or disables CUDA-graph replay of d3d_run step loops.
 * Enabled, the `count` launches of a loop are captured once per (buffers,
 * count, tile, coefficients) and replayed as one graph launch -- the
 * replacement for the reference's per-step host launches
 * (diffusion3d_cuda.cu:361-367).  Loops issued on a stream that is itself
 * being captured are launched directly into the caller's graph. */
int d3d_plan_set_graphs(d3d_plan plan, int enable);

/* Autotuner (the reference's tile sweep, src/diffusion3d/build.py:9-44,
 * done at run time instead of by rebuilding): times every tile variant and
 * a set of z-chunk lengths over `steps` time steps on the caller's buffers
 * f1/f2 (their contents are overwritten) with CUDA events on `stream`, and
 * keeps the fastest in the plan.  For D3D_KERNEL_TB plans it tunes the
 * z-chunk of the fused passes, for 2D plans the rows per warp task.
 * *best_ms (may be NULL) receives the best time per step. */
int d3d_plan_autotune(d3d_plan plan, void* f1, void* f2, const void* coeff,
                      int steps, void* stream, double* best_ms);

int d3d_plan_destroy(d3d_plan plan);

/* JSON description of the plan and its last launch geometry. */
int d3d_plan_info(d3d_plan plan, char* buf, size_t len);

/* Device / pinned-host memory, as Diffusion3DCUDA::InitializeBenchmark and
 * FinalizeBenchmark use cudaMalloc / cudaMallocHost / cudaFree
 * (diffusion3d_cuda.cu:329-350). */
int d3d_device_alloc(size_t bytes, void** ptr);
int d3d_device_free(void* ptr);
int d3d_host_alloc(size_t bytes, void** ptr);
int d3d_host_free(void* ptr);
int d3d_memcpy(void* dst, const void* src, size_t bytes, void* stream);
int d3d_stream_sync(void* stream);

/* One time step f2 = stencil(f1) on device buffers: one launch of
 * diffusion_kernel (diffusion3d_cuda.cu:13-45, launched at :362-363).
 * f1 and f2 must not overlap. */
int d3d_step(d3d_plan plan, const void* f1, void* f2, const void* coeff,
             void* stream);

/* d3d_step restricted to output planes [z_begin, z_end) of a 3D plan
 * (0 <= z_begin < z_end <= nz): those planes of f2 get one step of f1, the
 * rest of f2 is not touched; neighbours and the replicated boundary are
 * the whole field's.  No counterpart in the reference (its RunKernel steps
 * whole fields); the z-slab solver runs the planes its neighbours need
 * first, hands them to the exchange, and steps the interior meanwhile. */
int d3d_step_planes(d3d_plan plan, const void* f1, void* f2, int z_begin,
                    int z_end, const void* coeff, void* stream);

/* `count` time steps ping-ponging between two device buffers: the launch
 * loop of Diffusion3DCUDA::RunKernel (diffusion3d_cuda.cu:361-367).  Like
 * the reference, the buffer pointers are swapped after every step, so on
 * return *f1 points at the result and *f2 at the other buffer.  With
 * D3D_KERNEL_TB, count/tb_depth fused passes run first and count%tb_depth
 * single steps finish the job (exactly `count` steps for any count). */
int d3d_run(d3d_plan plan, void** f1, void** f2, const void* coeff, int count,
            void* stream);

/* ---------------------------------------------------------------------
 * One rank's z slab of a global nx*ny*nz grid split across processes (no
 * counterpart in the reference, whose only multi-node path is the external
 * Physis MPI runtime, src/diffusion3d/Makefile:253-268).  The rank owns
 * planes [z0, z1) and holds `halo` ghost planes on each side that has a
 * neighbour: a local buffer of planes [max(z0-halo, 0), min(z1+halo, nz)).
 * d3d_slab_run advances it in passes of k <= halo steps:
 *   1. for each neighbour, k steps of a 3*halo-plane piece around the rank
 *      boundary (copied out of the field), whose middle halo planes are
 *      then exact (a step clamped at a false edge is wrong only next to
 *      it, one more plane per step);
 *   2. transport.post hands those planes to the neighbours and names where
 *      theirs land;
 *   3. k steps of the owned planes in one d3d_run (fused two-step passes
 *      where the plan uses them), exact except the halo planes at each
 *      rank boundary, which step 1's planes overwrite;
 *   4. transport.wait, then the received planes become the ghosts.
 * The owned planes stay bit-identical to a one-GPU run of the whole grid.
 * ------------------------------------------------------------------- */
typedef struct d3d_slab_s* d3d_slab;

typedef struct d3d_slab_transport {
  /* Starts this pass's exchange: send[i] -> the neighbour on side i (0: the
   * rank below, owning lower z; 1: the rank above) and that neighbour's
   * planes into recv[i]; `bytes` each, device memory; NULL entries for a
   * side without a neighbour.  send[i] is ready once the work queued on
   * `stream` so far has run and stays untouched until wait() returns;
   * recv[i] is not read before wait() returns.  Nonzero: failure. */
  int (*post)(void* user, void* const send[2], void* const recv[2],
              size_t bytes, void* stream);
  /* Returns once work queued on `stream` after it is ordered after the
   * receives (or once they have landed).  Nonzero: failure. */
  int (*wait)(void* user, void* stream);
  void* user;
} d3d_slab_transport;

/* Creates the slab state for owned planes [z0, z1) of an nx*ny*nz grid
 * (0 <= z0 < z1 <= nz, halo >= 1; with a neighbour, z1 - z0 >= 2*halo and
 * halo planes beyond that side).  It owns two plans and, per neighbour,
 * two 3*halo-plane piece buffers and one halo-plane landing buffer; the
 * field's buffers are the caller's.  *local_nz (may be NULL) receives the
 * planes of the caller's buffers. */
int d3d_slab_create(int nx, int ny, int nz, int z0, int z1, int halo,
                    int dtype, d3d_slab* out, int* local_nz);

/* `count` steps of the slab held in *f1 (local_nz planes, ghost planes
 * current), ping-ponging with *f2; on return *f1 holds the result, its
 * ghost planes current, like d3d_run.  `transport` may be NULL only
 * without neighbours.  A callback's failure ends the run with
 * D3D_E_TRANSPORT after its queued work. */
int d3d_slab_run(d3d_slab slab, void** f1, void** f2, const void* coeff,
                 int count, const d3d_slab_transport* transport,
                 void* stream);

int d3d_slab_destroy(d3d_slab slab);

/* Diffusion3DCUDA::RunKernel(count) as a whole (diffusion3d_cuda.cu:353-371):
 * copies host_f1 to dev_f1, runs `count` steps between dev_f1 and dev_f2,
 * copies the result back into host_f1 and synchronises.  *kernel_ms (may be
 * NULL) receives the device time of the step loop alone (the reference's
 * "Kernel-only performance", :373-384); the loop's CUDA graph, captured on
 * the first call for a given (buffers, count), is built before that timing
 * starts. */
int d3d_run_host(d3d_plan plan, void* host_f1, void* dev_f1, void* dev_f2,
                 const void* coeff, int count, void* stream, float* kernel_ms);

/* The analytic solution at `time` (GetCorrectAnswer, diffusion3d.h:113-120,
 * with Initialize, diffusion3d.cc:14-39) written to a device buffer of the
 * plan dtype, evaluated in double precision on the device. */
int d3d_analytic(d3d_plan plan, void* out, double time, void* stream);

/* Binary checkpoints of a field of the plan's shape and dtype: the
 * replacement for the reference's text dump (Baseline::Dump,
 * baseline.cc:62-70, one "%.7E" line per value).  The file is a 64-byte
 * header (magic "D3DCKPT1", dtype, ndim, nx, ny, nz, `step`, the sum of the
 * payload's 32-bit words modulo 2^64, payload bytes, surface flag) and the
 * raw field, x fastest (benchmarks_b200.read_checkpoint reads one on a
 * host).  Device copies go through pinned staging that overlaps PCIe and
 * file I/O.  Load checks the shape, dtype and surface flag against the
 * plan (D3D_E_INVALID, before the field is touched) and the stored checksum
 * against the loaded field (D3D_E_IO); *step (may be NULL) receives the
 * saved step.  A load that fails after the header checks (a truncated or
 * corrupt payload, D3D_E_IO) leaves `field` partly overwritten: its
 * contents are then undefined.  The device
 * forms synchronise `stream`; d3d_checkpoint_save_host writes the same file
 * from a field in host memory (what a plugin's Dump holds in f1_). */
int d3d_checkpoint_save(d3d_plan plan, const void* field, long long step,
                        const char* path, void* stream);
int d3d_checkpoint_load(d3d_plan plan, const char* path, void* field,
                        long long* step, void* stream);
int d3d_checkpoint_save_host(d3d_plan plan, const void* host_field,
                             long long step, const char* path);

/* Error norms of device field a against device field b (n elements, any
 * dtype pair), accumulated in double on the device: out[0] = rms(a-b),
 * out[1] = max|a-b|, out[2] = max|a-b|/|b|, out[3] = sum(a).  The FP64
 * counterpart of Baseline::GetAccuracy (baseline.cc:51-60).  Synchronises
 * `stream`.  Uses plan-owned device scratch. */
int d3d_compare(d3d_plan plan, const void* a, int a_dtype, const void* b,
                int b_dtype, size_t n, double out[4], void* stream);

/* HBM calibration: `passes` ping-pong passes of f2 = cc * f1 over n floats
 * (then f1 = cc * f2, ...), 16-byte vectorised when both buffers are
 * 16-byte aligned.  It moves the stencil's 8 bytes per point with no
 * neighbours, so 8 * n * passes / time is the ceiling the step kernels
 * are held to.  The counterpart of the reference's DiffusionCUDACopy
 * (diffusion/diffusion_cuda_copy.cu:8-24).  *ms receives the device time
 * (CUDA events on `stream`); synchronises `stream`.  The buffers must not
 * overlap. */
int d3d_copy_calibrate(const float* f1, float* f2, size_t n, float cc,
                       int passes, void* stream, float* ms);

/* ---------------------------------------------------------------------
 * Batched solves: many independent FP32 grids of different shapes,
 * coefficients and step counts advanced together -- one multi-grid step
 * launch per size class and time step, the whole run captured once into a
 * CUDA graph and replayed as one graph launch.  Each size class runs the
 * kernel its autotuner picked: a shared-memory march over the caller's
 * fields, or a TMA strip kernel over pitched copies the batch keeps (and
 * fills and writes back inside the same graph).  No counterpart in the
 * reference (which runs one grid per
 * process); each grid's arithmetic is still RunKernel's, so every grid's
 * result is bit-identical to running it alone (with the reference or with
 * d3d_run).
 *
 * Fields live in one caller-owned device arena.  Grid i uses two buffers
 * of nx*ny*nz floats at element offsets offset_a and offset_b; its input
 * is in buffer a, and after the run its result is in buffer a when steps
 * is even and in buffer b when steps is odd (the reference's ping-pong).
 * --------------------------------------------------------------------- */
typedef struct {
  int nx, ny, nz, steps;
  float coeff[7];              /* ce, cw, cn, cs, ct, cb, cc */
  unsigned long long offset_a; /* element offsets into the arena */
  unsigned long long offset_b;
} d3d_batch_grid;

typedef struct d3d_batch_s* d3d_batch;

/* Coefficients for a grid of any shape: like the reference constructor
 * (diffusion3d.h:54-66) but with dt = 0.1*h^2/kappa for h = min(dx, dy, dz),
 * which keeps cc >= 0.4 (the reference derives dt from dx alone, which
 * makes non-cubic grids with ny or nz > nx unstable). */
int d3d_batch_coefficients(int nx, int ny, int nz, float kappa,
                           float coeff7[7]);

/* Packs grids back to back (two buffers each, 256-byte aligned) and sets
 * their offsets; *arena_bytes receives the arena size needed. */
int d3d_batch_layout(d3d_batch_grid* grids, int n, size_t* arena_bytes);

/* Builds the batch: size classes by nx, each class's grids ordered by step
 * count, their descriptors and work items, and device memory for pitched
 * copies of every grid (two buffers of ceil4(nx)*ny*nz floats each; if
 * that allocation fails the batch runs the march kinds only, on the
 * caller's fields, and d3d_batch_set_kind refuses the others with
 * D3D_E_UNSUPPORTED).  `arena` must stay valid for the batch's lifetime. */
int d3d_batch_create(const d3d_batch_grid* grids, int n, void* arena,
                     size_t arena_bytes, d3d_batch* out);

/* Times each kernel kind (4 march tile shapes, 2 strip forms, and 2
 * two-step strip forms where the class's grids allow) per size class on
 * the batch's own grids (their fields are overwritten) and keeps the
 * fastest per class: tile shape and temporal-block depth per class. */
int d3d_batch_autotune(d3d_batch batch, void* stream);

/* Sets every size class to one kernel kind: 0..3 the march kernel with
 * tile 32x16 (x pairs), 64x8 (x pairs), 32x8, 16x16; 4 and 5 the strip
 * kernel with 1 or 2 segments a thread (4 is the default before
 * d3d_batch_autotune); 6 and 7 its two-step form (temporal-block depth 2:
 * fused step pairs, and one strip step to finish an odd step count),
 * D3D_E_UNSUPPORTED if a grid is wider than 248 floats.  Kind 8
 * (D3D_BATCH_KIND_RESIDENT) runs every grid that fits on the cluster-
 * resident kernel: a cluster of up to 16 CTAs holds the whole grid in
 * shared memory for all of its steps (one persistent launch per cluster
 * size and thread shape, walking its grids through a work counter); the
 * grids it does not fit take kind 4.  d3d_batch_autotune also times the
 * whole run without kind 8 and with it for the grids that fit clusters of
 * at most 4, 8, 12 or 16 CTAs, and keeps the fastest. */
#define D3D_BATCH_NUM_KINDS 9
#define D3D_BATCH_KIND_RESIDENT 8
int d3d_batch_set_kind(d3d_batch batch, int kind);

/* With the cluster-resident kernel in use (kind 8 or the autotuner's
 * pick): only grids that fit clusters of at most max_cluster CTAs
 * (1..16) run on it, the others keep their size class's kind.
 * max_cluster = 0 turns the resident kernel off. */
int d3d_batch_set_resident_max_cluster(d3d_batch batch, int max_cluster);

/* Per-grid step counters of the last run (n = the batch's grid count):
 * the cluster-resident kernel advances a grid's counter after each of its
 * steps; grids on the per-step kinds get their step count once their last
 * launch has run.  A counter below the grid's steps after a run has
 * returned names a grid whose steps did not all complete.  Synchronous. */
int d3d_batch_progress(d3d_batch batch, int* steps_done, int n);

/* Runs every grid for its step count: the first call captures the run
 * into a CUDA graph, every call replays it as one graph launch.
 * *kernel_ms (may be NULL) receives the device time.  A bounded wait that
 * ran out in the TMA kernel is reported by d3d_check_device_errors. */
int d3d_batch_run(d3d_batch batch, void* stream, float* kernel_ms);

/* JSON summary: grids, steps, work items, launches per run, and per size
 * class its kernel (march tile shape or strip form) and work items. */
int d3d_batch_info(d3d_batch batch, char* buf, size_t len);

int d3d_batch_destroy(d3d_batch batch);

/* ---------------------------------------------------------------------
 * Serving: a continuous-batching solve server.  No counterpart in the
 * reference (a served request is what one RunKernel call does there:
 * InitializeBenchmark -> RunKernel -> FinalizeBenchmark).
 *
 * Requests (grid shape, steps, coefficients, a host input field and a host
 * output buffer) are queued by d3d_server_submit.  Each d3d_server_tick
 *   1. retires solves whose result has reached host memory,
 *   2. admits queued solves whose two buffers fit in the free part of the
 *      server's device arena (its HBM budget), copying their inputs in on a
 *      copy stream,
 *   3. advances every active solve by up to `chunk` steps with the
 *      multi-grid step kernel (solves admitted this tick included; by
 *      default a TMA kernel over row-padded copies of the fields), and
 *   4. starts the device->host copy of every solve that just finished.
 * Requests that arrive while others run join at the next tick; their work
 * overlaps on the device.  Each solve's arithmetic is RunKernel's, so its
 * result is bit-identical whether it runs alone or in any mix.
 * Host buffers must stay valid until the request is reported done; pinned
 * buffers (d3d_host_alloc) make the copies asynchronous.
 * --------------------------------------------------------------------- */
typedef struct d3d_server_s* d3d_server;

/* arena_bytes: device memory reserved for solve state (allocated once). */
int d3d_server_create(size_t arena_bytes, int chunk, d3d_server* out);

/* Queues one solve; *id receives its request id.  D3D_E_BUSY if the solve
 * can never fit the arena (2 * ceil4(nx)*ny*nz floats > arena with the
 * default kernel; 2 * nx*ny*nz with the march kernel). */
int d3d_server_submit(d3d_server server, int nx, int ny, int nz, int steps,
                      const float coeff[7], const float* host_in,
                      float* host_out, long long* id);

/* One scheduling round (does not wait for the GPU except to keep at most
 * two rounds in flight).  Writes up to max_done finished request ids. */
int d3d_server_tick(d3d_server server, long long* done_ids, int max_done,
                    int* n_done);

/* The step kernel of an idle server (D3D_E_BUSY otherwise): 0..4 the
 * pitched TMA kernel's tile shapes (0: 64 x 16, 1: 128 x 16, 2: 128 x 32,
 * 3: 64 x 32, 4: 128 x 8); 5 and 6 its strip form, where a CTA covers
 * whole rows of up to 248 columns and a thread takes 1 or 2 16-byte
 * segments (6 is the default); -1 the batch API's march kernel.
 * With the TMA kernel each solve is stored with rows padded to a multiple
 * of 4 floats, so it takes 2 * ceil4(nx)*ny*nz floats of the arena. */
int d3d_server_set_kernel(d3d_server server, int kernel);

/* Compute streams of an idle server (1..8, default 4; D3D_E_BUSY when
 * not idle).  Each solve runs all its steps on one stream, picked at
 * admission as the one with the least outstanding work; streams never wait
 * for one another, so one stream's launch tail overlaps another's work. */
int d3d_server_set_lanes(d3d_server server, int lanes);

/* A second step kernel for large solves on an idle server (D3D_E_BUSY
 * otherwise): solves whose pitched rows (ceil4(nx) floats) are at least
 * min_px use `kernel` (0..6, the ids of d3d_server_set_kernel) on the
 * upper half of the compute streams, the others the server's kernel on the
 * lower half.  kernel < 0 turns it off (the default); it has no effect
 * with the march kernel or a single stream. */
int d3d_server_set_large_kernel(d3d_server server, int kernel, int min_px);

/* Whether an idle server (D3D_E_BUSY otherwise) runs the solves that fit
 * the cluster-resident kernel on it (default off: on the 32..256 serving
 * stream it measured slower, the resident launches taking whole SMs from
 * the ticks' larger solves): such a solve (its grid
 * within one cluster's shared memory, the rule of D3D_BATCH_KIND_RESIDENT)
 * takes one dense buffer of the arena instead of two, and all of its steps
 * run in one persistent launch per cluster size together with the other
 * such solves admitted in the same tick, each launch on an idle stream of
 * a pool of 16; the ticks' step launches carry only the larger solves.
 * The first switch to on allocates the path's streams and its ring of 16
 * group stagings (pinned and device, 256 solves each), so serving itself
 * allocates nothing; on failure nothing of the ring is kept. */
int d3d_server_set_resident(d3d_server server, int on);

/* Number of requests queued, active on the device and copying out. */
int d3d_server_pending(d3d_server server, int* queued, int* active,
                       int* retiring);

/* JSON counters: submitted, completed, ticks, launches, chunk, kernel,
 * lanes, step_ms (device time of the step launches from CUDA events: per
 * tick, first stream's start to last stream's end), arena size and peak
 * arena use. */
int d3d_server_stats(d3d_server server, char* buf, size_t len);

int d3d_server_destroy(d3d_server server);

/* d3d_compare without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory at
 * the moment they want an error report -- a serving loop that has already
 * given all free HBM to its solve arena, or a host whose allocator policy
 * forbids driver allocations behind its back (a cudaMalloc would also
 * synchronise the whole device in the middle of a latency-sensitive loop).
 * The caller still passes the two fields; the partial sums go to a fixed
 * 128 KiB array in the library's device image, which every GPU that loads
 * the library keeps until exit.
 *  - n may be at most D3D_NOALLOC_MAX_ELEMENTS (2^28 elements, 1 GiB of
 *    FP32); larger n returns D3D_E_INVALID without touching the GPU.
 *  - The first call in a device's context looks up the array's device
 *    address (once per device, that device current; again after a
 *    cudaDeviceReset).
 *  - All calls share the array.  Each call writes every slot it reads, so
 *    results never depend on an earlier call, but calls whose kernels
 *    overlap on the GPU (different streams with no ordering) race.
 *  - The report is copied back to `out` on the host, so the call waits for
 *    `stream`; on a stream that is being captured it returns D3D_E_INVALID
 *    before launching anything.
 * Same outputs as d3d_compare (summation order differs: sums agree to
 * rounding, maxima exactly; a NaN in either field makes every output NaN). */
#define D3D_NOALLOC_MAX_ELEMENTS ((size_t)1 << 28)
int d3d_compare_noalloc(const void* a, int a_dtype, const void* b,
                        int b_dtype, size_t n, double out[4], void* stream);

/* The reference's accuracy report computed on the device: the field (plan
 * shape and dtype) against the analytic solution after `count` steps
 * (GetCorrectAnswer, diffusion3d.h:113-120; GetAccuracy, baseline.cc:51-60),
 * with the closed form evaluated per point in double and the errors summed in
 * double -- one read of the field, no analytic buffer.  out = rms, max_abs,
 * max_rel, sum(field).  (The reference sums in float sequentially on the
 * host; its figure is reproduced there, this is the FP64 report.) */
int d3d_accuracy(d3d_plan plan, const void* field, int count, double out[4],
                 void* stream);

/* Failure-path self-test: launches one CTA whose mbarrier wait (bounded by
 * `iterations` tries) can never complete, and returns what
 * d3d_check_device_errors returns afterwards -- D3D_E_TIMEOUT with the
 * timeout flag set, and a context that stays usable.  No fault, no trap. */
int d3d_selftest_wait_timeout(unsigned iterations, unsigned* flags_out);

/* Reads and clears the device error word that kernels set instead of
 * trapping when a bounded wait runs out; returns D3D_E_TIMEOUT if any bit
 * was set.  Synchronises the current device. */
int d3d_check_device_errors(unsigned* flags_out);

#ifdef __cplusplus
}
#endif

#endif /* D3D_B200_H_ */
