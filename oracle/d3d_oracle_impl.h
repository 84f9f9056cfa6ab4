/* Test infrastructure only: the oracle, never the product.
 *
 * Type-generic body of the CPU restatement of the reference's diffusion3d
 * path.  d3d_oracle.c includes this file twice, once with REAL = float
 * (the reference's own precision, diffusion3d.h:13) and once with
 * REAL = double (the FP64 run the reference cannot build because REAL is
 * hard-wired).  Every function names the reference lines it restates.
 *
 * Expects: REAL, SFX (function-name suffix), EXP_R / COS_R (the libm
 * functions C++ overload resolution picks for a REAL argument: expf/cosf
 * for float, exp/cos for double).
 */

#define D3DO_CAT2(a, b) a##b
#define D3DO_CAT(a, b) D3DO_CAT2(a, b)
#define D3DO_FN(name) D3DO_CAT(name, SFX)

/* Diffusion3D::Diffusion3D(nx, ny, nz), diffusion3d.h:54-66.
 * coeff = ce, cw, cn, cs, ct, cb, cc; geom = kappa, dx, dy, dz, kx, ky, kz, dt.
 * The casts reproduce where the reference computes in double (literals 0.1,
 * 1.0, 2.0*M_PI) before storing into REAL members. */
int D3DO_FN(d3do_params_)(int nx, int ny, int nz, REAL *coeff, REAL *geom) {
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
  REAL cc = (REAL)(1.0 - (ce + ce + cn + cn + ct + ct));
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

/* Initialize(buff, ...), diffusion3d.cc:14-39 (and the identical
 * Diffusion3DOpenMP::InitializeOMP, diffusion3d_openmp.cc:5-31).
 * x = dx*(REAL)(jx + 0.5); f0 = (REAL)0.125 * (1.0 - ax*cos(kx*x)) * ...
 * where the 1.0 - ... terms and their product are evaluated in double. */
int D3DO_FN(d3do_initialize_)(REAL *buff, int nx, int ny, int nz, REAL kx,
                              REAL ky, REAL kz, REAL dx, REAL dy, REAL dz,
                              REAL kappa, REAL time) {
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
        REAL z = dz * ((REAL)(jz + 0.5));
        double px = 1.0 - (double)(ax * COS_R(kx * x));
        double py = 1.0 - (double)(ay * COS_R(ky * y));
        double pz = 1.0 - (double)(az * COS_R(kz * z));
        REAL f0 = (REAL)((double)(REAL)0.125 * px * py * pz);
        buff[j] = f0;
      }
    }
  }
  return 0;
}

/* One time step of Diffusion3DOpenMP::RunKernel, diffusion3d_openmp.cc:43-71
 * (same arithmetic as Baseline::RunKernel, baseline.cc:22-49).  Clamped
 * neighbours: w=x-1, e=x+1, n=y-1, s=y+1, b=z-1, t=z+1, each replaced by the
 * centre at the domain edge.  Summation order as written at
 * diffusion3d_openmp.cc:61-62, left to right, no contraction.
 * c = {ce, cw, cn, cs, ct, cb, cc}. */
int D3DO_FN(d3do_step_)(const REAL *f1, REAL *f2, int nx, int ny, int nz,
                        const REAL *c) {
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
        long n = (y == 0) ? ci : ci - nx;
        long s = (y == ny - 1) ? ci : ci + nx;
        long b = (z == 0) ? ci : ci - xy;
        long t = (z == nz - 1) ? ci : ci + xy;
        REAL v = cc * f1[ci];
        v = v + cw * f1[w];
        v = v + ce * f1[e];
        v = v + cs * f1[s];
        v = v + cn * f1[n];
        v = v + cb * f1[b];
        v = v + ct * f1[t];
        f2[ci] = v;
      }
    }
  }
  return 0;
}

/* `count` steps with the reference's ping-pong (diffusion3d_openmp.cc:44-69,
 * pointer swap at :67-69).  The reference leaves its f1_ pointing at the
 * result; this restatement copies the result into `f1` when it ended in `f2`
 * so that callers always read `f1`. */
int D3DO_FN(d3do_run_)(REAL *f1, REAL *f2, int nx, int ny, int nz,
                       const REAL *c, int count) {
  REAL *a = f1, *b = f2;
  for (int i = 0; i < count; ++i) {
    D3DO_FN(d3do_step_)(a, b, nx, ny, nz, c);
    REAL *t = a;
    a = b;
    b = t;
  }
  if (a != f1) memcpy(f1, a, sizeof(REAL) * (size_t)nx * ny * nz);
  return 0;
}

/* Baseline::GetAccuracy(count), baseline.cc:51-60, with GetCorrectAnswer,
 * diffusion3d.h:113-120: RMS of (analytic at time count*dt) - f, accumulated
 * sequentially in REAL. */
REAL D3DO_FN(d3do_accuracy_)(const REAL *f, int nx, int ny, int nz, int count) {
  REAL geom[8];
  D3DO_FN(d3do_params_)(nx, ny, nz, NULL, geom);
  size_t len = (size_t)nx * ny * nz;
  REAL *ref = (REAL *)malloc(sizeof(REAL) * len);
  if (!ref) return (REAL)-1;
  REAL time = (REAL)count * geom[7];
  D3DO_FN(d3do_initialize_)(ref, nx, ny, nz, geom[4], geom[5], geom[6],
                            geom[1], geom[2], geom[3], geom[0], time);
  REAL err = (REAL)0.0;
  for (size_t i = 0; i < len; i++) {
    REAL diff = ref[i] - f[i];
    err += diff * diff;
  }
  free(ref);
  return (REAL)SQRT_R(err / (REAL)(long)len);
}

#undef D3DO_FN
#undef D3DO_CAT
#undef D3DO_CAT2
