/* Test infrastructure only: the oracle, never the product.
 *
 * Type-generic body of the CPU restatement of the reference's second plugin
 * surface, diffusion::Diffusion (src/diffusion): the same explicit diffusion
 * update on 2D (5-point) or 3D (7-point) grids.  d3d_oracle.c includes this
 * file once per precision, like d3d_oracle_impl.h.
 *
 * What differs from the diffusion3d surface, and is restated here:
 *   - cc sums the 3D pair last, (ce+cw+cn+cs) + (ct+cb)  (diffusion.h:107);
 *   - the y-neighbour order: s is y-1 and is summed before n = y+1
 *     (diffusion_openmp.cc:71-74, 98-103; baseline.h:55-70);
 *   - Initialize rounds the xy product to REAL before the z factor
 *     (diffusion.h:60-73), while DiffusionOpenMP::Initialize3D forms the
 *     whole product before rounding (diffusion_openmp.cc:25-49).
 *
 * Expects: REAL, SFX, EXP_R, COS_R, SQRT_R (as d3d_oracle_impl.h).
 */

#define DIFO_CAT2(a, b) a##b
#define DIFO_CAT(a, b) DIFO_CAT2(a, b)
#define DIFO_FN(name) DIFO_CAT(name, SFX)

/* diffusion::Diffusion::Diffusion(nd, dims), diffusion.h:93-108, with
 * nx, ny, nz as the constructor sets them (ny = 1 when nd < 2, nz = 1 when
 * nd < 3).  coeff = ce, cw, cn, cs, ct, cb, cc; geom = kappa, dx, dy, dz,
 * kx, ky, kz, dt. */
int DIFO_FN(difo_params_)(int nd, int nx, int ny, int nz, REAL *coeff,
                          REAL *geom) {
  REAL kappa = (REAL)0.1;
  REAL l = (REAL)1.0;
  REAL dx = l / nx;
  REAL dy = l / ny;
  REAL dz = l / nz;
  REAL k = (REAL)(2.0 * D3DO_PI);
  REAL dt = (REAL)(0.1 * dx * dx / kappa);
  REAL ce = kappa * dt / (dx * dx);
  REAL cn = kappa * dt / (dy * dy);
  REAL ct = kappa * dt / (dz * dz);
  /* cc_ = 1.0 - (ce_ + cw_ + cn_ + cs_ + (ndim_ == 3 ? (ct_ + cb_) : 0)):
   * the conditional has type REAL, and the REAL sum is widened for 1.0 -. */
  REAL xy = ce + ce + cn + cn;
  REAL zpair = (nd == 3) ? (REAL)(ct + ct) : (REAL)0;
  REAL cc = (REAL)(1.0 - (double)(xy + zpair));
  if (coeff) {
    coeff[0] = ce; coeff[1] = ce; coeff[2] = cn; coeff[3] = cn;
    coeff[4] = ct; coeff[5] = ct; coeff[6] = cc;
  }
  if (geom) {
    geom[0] = kappa; geom[1] = dx; geom[2] = dy; geom[3] = dz;
    geom[4] = k; geom[5] = k; geom[6] = k; geom[7] = dt;
  }
  return 0;
}

/* The analytic field.  omp = 0: the header's Initialize, diffusion.h:48-77
 * (Baseline::InitializeInput, baseline.h:33-37, and GetCorrectAnswer,
 * diffusion.h:172-179): the xy product is rounded to REAL, then a 3D grid
 * multiplies in the z factor and rounds again.  omp = 1:
 * DiffusionOpenMP::Initialize2D / Initialize3D (diffusion_openmp.cc:5-49),
 * which form the whole product before the one rounding (identical to
 * omp = 0 in 2D). */
int DIFO_FN(difo_initialize_)(REAL *buff, int nx, int ny, int nz, REAL kx,
                              REAL ky, REAL kz, REAL dx, REAL dy, REAL dz,
                              REAL kappa, REAL time, int nd, int omp) {
  REAL ax = EXP_R(-kappa * time * (kx * kx));
  REAL ay = EXP_R(-kappa * time * (ky * ky));
  REAL az = EXP_R(-kappa * time * (kz * kz));
  int jz;
#pragma omp parallel for
  for (jz = 0; jz < nz; jz++) {
    for (int jy = 0; jy < ny; jy++) {
      for (int jx = 0; jx < nx; jx++) {
        size_t j = (size_t)jz * nx * ny + (size_t)jy * nx + jx;
        REAL x = dx * ((REAL)(jx + 0.5));
        REAL y = dy * ((REAL)(jy + 0.5));
        double px = 1.0 - (double)(ax * COS_R(kx * x));
        double py = 1.0 - (double)(ay * COS_R(ky * y));
        REAL f0;
        if (nd == 3) {
          REAL z = dz * ((REAL)(jz + 0.5));
          double pz = 1.0 - (double)(az * COS_R(kz * z));
          if (omp) {
            f0 = (REAL)((double)(REAL)0.125 * px * py * pz);
          } else {
            f0 = (REAL)((double)(REAL)0.125 * px * py);
            f0 = (REAL)((double)f0 * pz);
          }
        } else {
          f0 = (REAL)((double)(REAL)0.125 * px * py);
        }
        buff[j] = f0;
      }
    }
  }
  return 0;
}

/* One time step of DiffusionOpenMP::RunKernel2D / RunKernel3D
 * (diffusion_openmp.cc:59-112; Baseline::RunKernel, baseline.h:46-80, is
 * the same arithmetic).  Clamped neighbours w = x-1, e = x+1, s = y-1,
 * n = y+1, b = z-1, t = z+1; the sum runs left to right as written,
 * cc*c + cw*w + ce*e + cs*s + cn*n [+ cb*b + ct*t], no contraction.
 * c = {ce, cw, cn, cs, ct, cb, cc}.  nd = 2 uses nz = 1. */
int DIFO_FN(difo_step_)(const REAL *f1, REAL *f2, int nd, int nx, int ny,
                        int nz, const REAL *c) {
  const REAL ce = c[0], cw = c[1], cn = c[2], cs = c[3], ct = c[4],
             cb = c[5], cc = c[6];
  const long xy = (long)nx * ny;
  int z;
#pragma omp parallel for
  for (z = 0; z < nz; z++) {
    for (int y = 0; y < ny; y++) {
      for (int x = 0; x < nx; x++) {
        long ci = x + (long)y * nx + (long)z * xy;
        long w = (x == 0) ? ci : ci - 1;
        long e = (x == nx - 1) ? ci : ci + 1;
        long s = (y == 0) ? ci : ci - nx;
        long n = (y == ny - 1) ? ci : ci + nx;
        REAL v = cc * f1[ci];
        v = v + cw * f1[w];
        v = v + ce * f1[e];
        v = v + cs * f1[s];
        v = v + cn * f1[n];
        if (nd == 3) {
          long b = (z == 0) ? ci : ci - xy;
          long t = (z == nz - 1) ? ci : ci + xy;
          v = v + cb * f1[b];
          v = v + ct * f1[t];
        }
        f2[ci] = v;
      }
    }
  }
  return 0;
}

/* `count` steps with the reference's pointer swap (diffusion_openmp.cc:
 * 77-79, 107-109); the result is copied into `f1` when it ended in `f2`. */
int DIFO_FN(difo_run_)(REAL *f1, REAL *f2, int nd, int nx, int ny, int nz,
                       const REAL *c, int count) {
  REAL *a = f1, *b = f2;
  for (int i = 0; i < count; ++i) {
    DIFO_FN(difo_step_)(a, b, nd, nx, ny, nz, c);
    REAL *t = a;
    a = b;
    b = t;
  }
  if (a != f1) memcpy(f1, a, sizeof(REAL) * (size_t)nx * ny * nz);
  return 0;
}

/* Baseline::GetAccuracy(count), baseline.h:86-95, with GetCorrectAnswer
 * (diffusion.h:172-179): RMS of the header Initialize at time count*dt
 * minus f, accumulated sequentially in REAL. */
REAL DIFO_FN(difo_accuracy_)(const REAL *f, int nd, int nx, int ny, int nz,
                             int count) {
  REAL geom[8];
  DIFO_FN(difo_params_)(nd, nx, ny, nz, NULL, geom);
  size_t len = (size_t)nx * ny * nz;
  REAL *ref = (REAL *)malloc(sizeof(REAL) * len);
  if (!ref) return (REAL)-1;
  REAL time = (REAL)count * geom[7];
  DIFO_FN(difo_initialize_)(ref, nx, ny, nz, geom[4], geom[5], geom[6],
                            geom[1], geom[2], geom[3], geom[0], time, nd, 0);
  REAL err = (REAL)0.0;
  for (size_t i = 0; i < len; i++) {
    REAL diff = ref[i] - f[i];
    err += diff * diff;
  }
  free(ref);
  return (REAL)SQRT_R(err / (REAL)(long)len);
}

#undef DIFO_FN
#undef DIFO_CAT
#undef DIFO_CAT2
