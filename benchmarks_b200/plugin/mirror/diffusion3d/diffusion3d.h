// The diffusion3d plugin surface, restated for builds without the reference
// tree (the reference's is src/diffusion3d/diffusion3d.h:43-121).
//
// A backend written against the reference's header compiles against this
// one: same namespace, class names, protected members and virtuals.  The
// constructor, Initialize and the reported rates use the reference's
// arithmetic (REAL members, double literals promoting and narrowing where
// the reference's do), so a backend reports the same coefficients,
// accuracy and rates it would report in the reference tree.
#ifndef DIFFUSION3D_DIFFUSION3D_H_
#define DIFFUSION3D_DIFFUSION3D_H_

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
#define OFFSET3D(i, j, k, nx, ny) ((i) + (j) * (nx) + (k) * (nx) * (ny))

namespace diffusion3d {

// Analytic solution at `time` on cell centres:
// 0.125 * prod_d (1 - exp(-kappa*time*k_d^2) * cos(k_d * (idx_d + 0.5) * d_d)).
void Initialize(REAL* buff, const int nx, const int ny, const int nz,
                const REAL kx, const REAL ky, const REAL kz, const REAL dx,
                const REAL dy, const REAL dz, const REAL kappa,
                const REAL time);

class Diffusion3D {
 protected:
  int nx_;
  int ny_;
  int nz_;
  REAL kappa_;
  REAL dx_, dy_, dz_;
  REAL kx_, ky_, kz_;
  REAL dt_;
  REAL ce_, cw_, cn_, cs_, ct_, cb_, cc_;

 public:
  // Unit cube, kappa = 0.1, wave number 2*pi, dt = 0.1 * dx^2 / kappa.
  Diffusion3D(int nx, int ny, int nz) : nx_(nx), ny_(ny), nz_(nz), kappa_(0.1) {
    const REAL unit = 1.0;
    dx_ = unit / nx;
    dy_ = unit / ny;
    dz_ = unit / nz;
    kx_ = ky_ = kz_ = 2.0 * 3.14159265358979323846;
    dt_ = 0.1 * dx_ * dx_ / kappa_;  // evaluated in double, stored as REAL
    ce_ = cw_ = kappa_ * dt_ / (dx_ * dx_);
    cn_ = cs_ = kappa_ * dt_ / (dy_ * dy_);
    ct_ = cb_ = kappa_ * dt_ / (dz_ * dz_);
    cc_ = 1.0 - (ce_ + cw_ + cn_ + cs_ + ct_ + cb_);
  }
  virtual ~Diffusion3D() {}
  virtual std::string GetName() const = 0;

  // Initialize, time RunKernel(count) on the wall clock, report, optionally
  // dump, finalize.
  void RunBenchmark(int count, bool dump) {
    std::cout << "Initializing benchmark input...\n";
    InitializeBenchmark();
    std::cout << "Running diffusion3d/" << GetName() << "\n";
    std::cout << "Iteration count: " << count << "\n";
    std::cout << "Grid size: " << nx_ << "x" << ny_ << "x" << nz_ << "\n";
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
    return "diffusion3d_result." + GetName() + ".out";
  }
  virtual void InitializeBenchmark() = 0;
  virtual void RunKernel(int count) = 0;
  virtual void Dump() const = 0;
  virtual REAL GetAccuracy(int count) = 0;
  virtual void FinalizeBenchmark() = 0;

  // Bytes moved: one read and one write of every point per step.
  float GetThroughput(int count, float time) {
    return (nx_ * ny_ * nz_) * sizeof(REAL) * 2.0 * ((float)count) / time *
           1.0e-09;
  }
  // 13 flops per point update.
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
               count * dt_);
    return f;
  }
};

}  // namespace diffusion3d

#endif  // DIFFUSION3D_DIFFUSION3D_H_
