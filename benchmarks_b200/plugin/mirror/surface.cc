// Definitions of the restated diffusion3d plugin surface (mirror/).
#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "diffusion3d/baseline.h"

namespace diffusion3d {

// Cell-centred analytic field.  Precision follows the reference's
// Initialize (diffusion3d.cc:14-39): coordinates, exp and cos in REAL (the
// float overloads for REAL = float), the "1 - a*cos" factors and their
// product in double, the result narrowed to REAL.
void Initialize(REAL* buff, const int nx, const int ny, const int nz,
                const REAL kx, const REAL ky, const REAL kz, const REAL dx,
                const REAL dy, const REAL dz, const REAL kappa,
                const REAL time) {
  const REAL ax = std::exp(-kappa * time * (kx * kx));
  const REAL ay = std::exp(-kappa * time * (ky * ky));
  const REAL az = std::exp(-kappa * time * (kz * kz));
  for (int jz = 0; jz < nz; ++jz) {
    const REAL z = dz * ((REAL)(jz + 0.5));
    const double fz = 1.0 - az * std::cos(kz * z);
    for (int jy = 0; jy < ny; ++jy) {
      const REAL y = dy * ((REAL)(jy + 0.5));
      const double fy = 1.0 - ay * std::cos(ky * y);
      REAL* row = buff + (size_t)jz * nx * ny + (size_t)jy * nx;
      for (int jx = 0; jx < nx; ++jx) {
        const REAL x = dx * ((REAL)(jx + 0.5));
        const double fx = 1.0 - ax * std::cos(kx * x);
        row[jx] = (REAL)((REAL)0.125 * fx * fy * fz);
      }
    }
  }
}

void Baseline::InitializeBenchmark() {
  const size_t n = (size_t)nx_ * ny_ * nz_;
  f1_ = (REAL*)malloc(sizeof(REAL) * n);
  f2_ = (REAL*)malloc(sizeof(REAL) * n);
  assert(f1_ && f2_);
  Initialize(f1_, nx_, ny_, nz_, kx_, ky_, kz_, dx_, dy_, dz_, kappa_, 0.0);
}

void Baseline::FinalizeBenchmark() {
  free(f1_);
  free(f2_);
  f1_ = f2_ = NULL;
}

// This surface carries no stencil implementation of its own: the compute
// belongs to the backend (Diffusion3DB200 overrides RunKernel).
void Baseline::RunKernel(int) {
  fprintf(stderr,
          "diffusion3d: Baseline::RunKernel is not part of the restated "
          "surface; use a backend such as Diffusion3DB200\n");
  exit(EXIT_FAILURE);
}

// Root-mean-square difference to the analytic field, summed in REAL in
// index order (the reference's Baseline::GetAccuracy, baseline.cc:51-60).
REAL Baseline::GetAccuracy(int count) {
  REAL* ref = GetCorrectAnswer(count);
  const long len = (long)nx_ * ny_ * nz_;
  REAL sum = 0.0;
  for (long i = 0; i < len; ++i) {
    const REAL d = ref[i] - f1_[i];
    sum += d * d;
  }
  free(ref);
  return (REAL)std::sqrt(sum / len);
}

// One value per line, "%.7E" (the reference's Dump, baseline.cc:62-70).
void Baseline::Dump() const {
  FILE* out = fopen(GetDumpPath().c_str(), "w");
  assert(out);
  const long n = (long)nx_ * ny_ * nz_;
  for (long i = 0; i < n; ++i) fprintf(out, "%.7E\n", f1_[i]);
  fclose(out);
}

}  // namespace diffusion3d
