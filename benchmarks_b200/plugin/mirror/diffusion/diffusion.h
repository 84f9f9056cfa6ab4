// The diffusion plugin surface (2D and 3D grids), restated for builds
// without the reference tree (the reference's is
// src/diffusion/diffusion.h:46-181).
//
// A backend written against the reference's header compiles against this
// one: same namespace, class names, protected members and virtuals.  The
// constructor, Initialize and the reported rates use the reference's
// arithmetic (REAL members, double literals promoting and narrowing where
// the reference's do), so a backend reports what it would report in the
// reference tree.
#ifndef DIFFUSION_DIFFUSION_H_
#define DIFFUSION_DIFFUSION_H_

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <iostream>
#include <string>

#include "common/stopwatch.h"

#ifndef REAL
#define REAL float
#endif

// x fastest, then y, then z; no padding.
#define OFFSET2D(i, j, nx) ((i) + (j) * (nx))
#define OFFSET3D(i, j, k, nx, ny) ((i) + (j) * (nx) + (k) * (nx) * (ny))

namespace diffusion {

// Analytic field at `time` on cell centres:
// 0.125 * (1 - ax cos(kx x)) * (1 - ay cos(ky y)), rounded to REAL, then
// for ndim == 3 times (1 - az cos(kz z)) and rounded again.  exp/cos take
// REAL arguments (the float overloads when REAL is float); each "1 - a cos"
// factor and each product is formed in double.
inline void Initialize(REAL* buff, const int nx, const int ny, const int nz,
                       const REAL kx, const REAL ky, const REAL kz,
                       const REAL dx, const REAL dy, const REAL dz,
                       const REAL kappa, const REAL time, int ndim) {
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
        REAL v = (REAL)((REAL)0.125 * fx * fy);
        if (ndim == 3) v = (REAL)(v * fz);
        row[jx] = v;
      }
    }
  }
}

class Diffusion {
 protected:
  int ndim_;
  int nx_;
  int ny_;
  int nz_;
  REAL kappa_;
  REAL dx_, dy_, dz_;
  REAL kx_, ky_, kz_;
  REAL dt_;
  REAL ce_, cw_, cn_, cs_, ct_, cb_, cc_;

 public:
  // dims holds ndim extents (nx, ny[, nz]); missing ones are 1.  Unit
  // square/cube, kappa = 0.1, wave number 2*pi, dt = 0.1 * dx^2 / kappa;
  // the z pair enters cc (as one sum) only in 3D.
  Diffusion(int ndim, const int* dims) : ndim_(ndim), kappa_(0.1) {
    nx_ = dims[0];
    ny_ = ndim > 1 ? dims[1] : 1;
    nz_ = ndim > 2 ? dims[2] : 1;
    const REAL unit = 1.0;
    dx_ = unit / nx_;
    dy_ = unit / ny_;
    dz_ = unit / nz_;
    kx_ = ky_ = kz_ = 2.0 * 3.14159265358979323846;
    dt_ = 0.1 * dx_ * dx_ / kappa_;  // evaluated in double, stored as REAL
    ce_ = cw_ = kappa_ * dt_ / (dx_ * dx_);
    cn_ = cs_ = kappa_ * dt_ / (dy_ * dy_);
    ct_ = cb_ = kappa_ * dt_ / (dz_ * dz_);
    const REAL zpair = ndim_ == 3 ? (REAL)(ct_ + cb_) : (REAL)0;
    cc_ = 1.0 - (ce_ + cw_ + cn_ + cs_ + zpair);
  }
  virtual ~Diffusion() {}

  virtual std::string GetName() const = 0;
  virtual std::string GetDescription() const = 0;

  // Setup, initialize, optionally warm up (then initialize again), time
  // RunKernel(count) on the wall clock, report, optionally dump, finalize.
  void RunBenchmark(int count, bool dump, bool warmup) {
    std::cout << "*** Diffusion Benchmark ***\n";
    std::cout << "Benchmark: " << GetName() << " (" << GetDescription()
              << ")\n";
    Setup();
    std::cout << "Initializing benchmark input...\n";
    InitializeInput();
    std::cout << "Iteration count: " << count << "\n";
    std::cout << "Grid size: " << nx_ << "x" << ny_;
    if (ndim_ == 3) std::cout << "x" << nz_;
    std::cout << "\n";
    if (warmup) {
      std::cout << "Warming up the kernel...\n";
      WarmingUp();
      std::cout << "Reinitializing benchmark input...\n";
      InitializeInput();
    }
    std::cout << "Running the kernel...\n";
    Stopwatch sw;
    StopwatchStart(&sw);
    RunKernel(count);
    const float seconds = StopwatchStop(&sw);
    std::cout << "Benchmarking finished.\n";
    DisplayResult(count, seconds);
    if (dump) Dump();
    FinalizeBenchmark();
  }

 protected:
  std::string GetDumpPath() const {
    return "diffusion_result." + GetName() + ".out";
  }
  virtual void Setup() = 0;
  virtual void InitializeInput() = 0;
  virtual void RunKernel(int count) = 0;
  virtual void WarmingUp() = 0;
  virtual void Dump() const = 0;
  virtual REAL GetAccuracy(int count) = 0;
  virtual void FinalizeBenchmark() = 0;

  // Bytes moved: one read and one write of every point per step.
  float GetThroughput(int count, float time) {
    return (nx_ * ny_ * nz_) * sizeof(REAL) * 2.0 * ((float)count) / time *
           1.0e-09;
  }
  // 13 flops per point update (the reference counts 13 in 2D as well).
  float GetGFLOPS(int count, float time) {
    return (nx_ * ny_ * nz_) * 13.0 * (float)(count) / time * 1.0e-09;
  }
  virtual void DisplayResult(int count, float time) {
    printf("Elapsed time : %.3f (s)\n", time);
    printf("FLOPS        : %.3f (GFLOPS)\n", GetGFLOPS(count, time));
    printf("Throughput   : %.3f (GB/s)\n", GetThroughput(count, time));
    printf("Accuracy     : %e\n", GetAccuracy(count));
  }
  // The analytic field after `count` steps (caller frees).
  REAL* GetCorrectAnswer(int count) const {
    REAL* f = (REAL*)malloc(sizeof(REAL) * (size_t)nx_ * ny_ * nz_);
    if (!f) abort();
    Initialize(f, nx_, ny_, nz_, kx_, ky_, kz_, dx_, dy_, dz_, kappa_,
               count * dt_, ndim_);
    return f;
  }
};

}  // namespace diffusion

#endif  // DIFFUSION_DIFFUSION_H_
