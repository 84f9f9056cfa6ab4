// Definitions of the restated diffusion plugin surface (mirror/diffusion).
#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "diffusion/baseline.h"

namespace diffusion {

void Baseline::Setup() {
  const size_t n = (size_t)nx_ * ny_ * nz_;
  f1_ = (REAL*)malloc(sizeof(REAL) * n);
  f2_ = (REAL*)malloc(sizeof(REAL) * n);
  assert(f1_ && f2_);
}

void Baseline::InitializeInput() {
  Initialize(f1_, nx_, ny_, nz_, kx_, ky_, kz_, dx_, dy_, dz_, kappa_, 0.0,
             ndim_);
}

void Baseline::FinalizeBenchmark() {
  free(f1_);
  free(f2_);
  f1_ = f2_ = NULL;
}

// This surface carries no stencil implementation of its own: the compute
// belongs to the backend (DiffusionB200 overrides RunKernel).
void Baseline::RunKernel(int) {
  fprintf(stderr,
          "diffusion: Baseline::RunKernel is not part of the restated "
          "surface; use a backend such as DiffusionB200\n");
  exit(EXIT_FAILURE);
}

// Root-mean-square difference to the analytic field, summed in REAL in
// index order.
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

// One value per line, "%.7E".
void Baseline::Dump() const {
  FILE* out = fopen(GetDumpPath().c_str(), "w");
  assert(out);
  const long n = (long)nx_ * ny_ * nz_;
  for (long i = 0; i < n; ++i) fprintf(out, "%.7E\n", f1_[i]);
  fclose(out);
}

}  // namespace diffusion
