/* Test infrastructure only: the oracle, never the product.
 *
 * CPU restatement of the reference's diffusion3d hot path
 * (naoyam/benchmarks, src/diffusion3d), used by tests/, by smoke() and by
 * bench.py's CPU-baseline leg as the checker.  The product (libd3d_b200.so)
 * neither links nor calls it.
 *
 * Restated functions (bodies in d3d_oracle_impl.h):
 *   d3do_params_{f32,f64}      Diffusion3D::Diffusion3D       diffusion3d.h:54-66
 *   d3do_initialize_{f32,f64}  Initialize                     diffusion3d.cc:14-39
 *   d3do_step_{f32,f64}        Diffusion3DOpenMP::RunKernel   diffusion3d_openmp.cc:43-71
 *   d3do_run_{f32,f64}         (same, `count` steps)
 *   d3do_accuracy_{f32,f64}    Baseline::GetAccuracy          baseline.cc:51-60
 * and of the second plugin surface, diffusion::Diffusion (src/diffusion;
 * bodies in dif_oracle_impl.h):
 *   difo_params_{f32,f64}      Diffusion::Diffusion           diffusion.h:93-108
 *   difo_initialize_{f32,f64}  Initialize                     diffusion.h:48-77
 *                              DiffusionOpenMP::Initialize2D/3D diffusion_openmp.cc:5-49
 *   difo_step_{f32,f64}        DiffusionOpenMP::RunKernel2D/3D diffusion_openmp.cc:59-112
 *   difo_run_{f32,f64}         (same, `count` steps)
 *   difo_accuracy_{f32,f64}    Baseline::GetAccuracy          baseline.h:86-95
 * plus FP64-accumulated error norms between two fields (no reference
 * counterpart: the FP64 error report the reference lacks).
 *
 * Pinning: tests/test_oracle.py checks every function bit-for-bit against
 * the reference's own objects (oracle/_ref, built from the reference sources
 * by `make -C oracle ref`) and against the committed golden fixtures in
 * tests/golden/ that tests/golden/make_golden.py generated from them.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define D3DO_PI 3.14159265358979323846

/* FP32: the reference's precision.  C++ overload resolution on float
 * arguments selects expf/cosf/sqrtf in the reference's <math.h>. */
#define REAL float
#define SFX f32
#define EXP_R expf
#define COS_R cosf
#define SQRT_R sqrtf
#include "d3d_oracle_impl.h"
#include "dif_oracle_impl.h"
#undef REAL
#undef SFX
#undef EXP_R
#undef COS_R
#undef SQRT_R

/* FP64: the same code with REAL = double. */
#define REAL double
#define SFX f64
#define EXP_R exp
#define COS_R cos
#define SQRT_R sqrt
#include "d3d_oracle_impl.h"
#include "dif_oracle_impl.h"
#undef REAL
#undef SFX
#undef EXP_R
#undef COS_R
#undef SQRT_R

int d3do_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* Error norms of `a` against `b` accumulated in double:
 * out[0] = sqrt(mean((a-b)^2)), out[1] = max|a-b|,
 * out[2] = max|a-b| / max(|b|, tiny), out[3] = sum(a) (a checksum). */
#define D3DO_NORMS(NAME, TA, TB)                                          \
  int NAME(const TA *a, const TB *b, long n, double *out) {               \
    double ss = 0.0, mx = 0.0, mr = 0.0, sa = 0.0;                        \
    for (long i = 0; i < n; ++i) {                                        \
      double d = (double)a[i] - (double)b[i];                             \
      double ad = fabs(d);                                                \
      double den = fabs((double)b[i]);                                    \
      ss += d * d;                                                        \
      if (ad > mx) mx = ad;                                               \
      if (den < 1e-300) den = 1e-300;                                     \
      if (ad / den > mr) mr = ad / den;                                   \
      sa += (double)a[i];                                                 \
    }                                                                     \
    out[0] = n > 0 ? sqrt(ss / (double)n) : 0.0;                          \
    out[1] = mx;                                                          \
    out[2] = mr;                                                          \
    out[3] = sa;                                                          \
    return 0;                                                             \
  }
D3DO_NORMS(d3do_norms_f32_f32, float, float)
D3DO_NORMS(d3do_norms_f32_f64, float, double)
D3DO_NORMS(d3do_norms_f64_f64, double, double)
