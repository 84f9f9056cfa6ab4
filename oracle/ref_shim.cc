// Test infrastructure only (the checker, never the product).
//
// A thin extern "C" probe around the reference's own CPU backends, compiled
// from the reference sources in place by oracle/Makefile into
// oracle/_ref/libd3d_ref.so.  It subclasses the reference classes to reach
// their protected state (f1_, the seven coefficients) so that tests can feed
// seeded, non-cubic inputs and read back the field the reference computed.
//
// Backends probed:
//   0  diffusion3d::Diffusion3DOpenMP              diffusion3d_openmp.cc:43-71
//   1  diffusion3d::Baseline                       baseline.cc:22-49
//   2  diffusion3d::Diffusion3DOpenMPTemporalBlocking
//                                                  diffusion3d_openmp_temporal_blocking.cc:8-68
#include <stdlib.h>
#include <string.h>

#include <chrono>

#include "diffusion3d/baseline.h"
#include "diffusion3d/diffusion3d_openmp.h"
#include "diffusion3d/diffusion3d_openmp_temporal_blocking.h"

namespace {

using diffusion3d::Baseline;
using diffusion3d::Diffusion3DOpenMP;
using diffusion3d::Diffusion3DOpenMPTemporalBlocking;

template <class Backend>
class Probe : public Backend {
 public:
  Probe(int nx, int ny, int nz) : Backend(nx, ny, nz) {}

  void Setup() { this->InitializeBenchmark(); }
  void Teardown() { this->FinalizeBenchmark(); }

  // ce, cw, cn, cs, ct, cb, cc (the reference's member order).
  void GetCoeffs(float *c) const {
    c[0] = this->ce_; c[1] = this->cw_; c[2] = this->cn_; c[3] = this->cs_;
    c[4] = this->ct_; c[5] = this->cb_; c[6] = this->cc_;
  }
  void SetCoeffs(const float *c) {
    this->ce_ = c[0]; this->cw_ = c[1]; this->cn_ = c[2]; this->cs_ = c[3];
    this->ct_ = c[4]; this->cb_ = c[5]; this->cc_ = c[6];
  }
  // kappa, dx, dy, dz, kx, ky, kz, dt
  void GetGeometry(float *g) const {
    g[0] = this->kappa_; g[1] = this->dx_; g[2] = this->dy_; g[3] = this->dz_;
    g[4] = this->kx_; g[5] = this->ky_; g[6] = this->kz_; g[7] = this->dt_;
  }
  size_t Points() const {
    return (size_t)this->nx_ * this->ny_ * this->nz_;
  }
  void SetField(const float *in) { memcpy(this->f1_, in, Points() * 4); }
  void GetField(float *out) const { memcpy(out, this->f1_, Points() * 4); }
  void Run(int count) { this->RunKernel(count); }
  float Accuracy(int count) { return this->GetAccuracy(count); }
  void DumpField() const { this->Dump(); }
  float GFlops(int count, float t) { return this->GetGFLOPS(count, t); }
  float Throughput(int count, float t) { return this->GetThroughput(count, t); }
};

template <class Backend>
int RunProbe(int nx, int ny, int nz, const float *coeff, const float *in,
             float *out, int count, float *accuracy, int dump,
             double *run_seconds) {
  Probe<Backend> p(nx, ny, nz);
  p.Setup();
  if (coeff) p.SetCoeffs(coeff);
  if (in) p.SetField(in);
  const auto t0 = std::chrono::steady_clock::now();
  p.Run(count);
  if (run_seconds)
    *run_seconds = std::chrono::duration<double>(
                       std::chrono::steady_clock::now() - t0)
                       .count();
  if (out) p.GetField(out);
  if (accuracy) *accuracy = p.Accuracy(count);
  if (dump) p.DumpField();
  p.Teardown();
  return 0;
}

}  // namespace

extern "C" {

// Runs `count` steps of the chosen reference backend.  `coeff` (7 floats,
// ce..cc) and `in` (nx*ny*nz floats) are optional overrides of what the
// reference's own constructor and InitializeBenchmark produce.  The field
// after `count` steps (the reference's f1_) lands in `out` when non-null;
// `run_seconds`, when non-null, receives the wall time of RunKernel(count)
// alone (InitializeBenchmark and the copies excluded).
int d3dref_run_timed(int backend, int nx, int ny, int nz, const float *coeff,
                     const float *in, float *out, int count, float *accuracy,
                     int dump, double *run_seconds) {
  switch (backend) {
    case 0:
      return RunProbe<Diffusion3DOpenMP>(nx, ny, nz, coeff, in, out, count,
                                         accuracy, dump, run_seconds);
    case 1:
      return RunProbe<Baseline>(nx, ny, nz, coeff, in, out, count, accuracy,
                                dump, run_seconds);
    case 2:
      return RunProbe<Diffusion3DOpenMPTemporalBlocking>(
          nx, ny, nz, coeff, in, out, count, accuracy, dump, run_seconds);
    default:
      return -1;
  }
}

int d3dref_run(int backend, int nx, int ny, int nz, const float *coeff,
               const float *in, float *out, int count, float *accuracy,
               int dump) {
  return d3dref_run_timed(backend, nx, ny, nz, coeff, in, out, count,
                          accuracy, dump, nullptr);
}

// The reference constructor's derived quantities for an nx*ny*nz grid.
// coeff: ce, cw, cn, cs, ct, cb, cc.  geom: kappa, dx, dy, dz, kx, ky, kz, dt.
int d3dref_params(int nx, int ny, int nz, float *coeff, float *geom) {
  Probe<Baseline> p(nx, ny, nz);
  if (coeff) p.GetCoeffs(coeff);
  if (geom) p.GetGeometry(geom);
  return 0;
}

// The reference's free Initialize() (diffusion3d.cc:14-39).
int d3dref_initialize(float *buf, int nx, int ny, int nz, float kx, float ky,
                      float kz, float dx, float dy, float dz, float kappa,
                      float time) {
  diffusion3d::Initialize(buf, nx, ny, nz, kx, ky, kz, dx, dy, dz, kappa,
                          time);
  return 0;
}

// The reference's GetGFLOPS / GetThroughput formulas (diffusion3d.h:97-104).
int d3dref_rates(int nx, int ny, int nz, int count, float time, float *gflops,
                 float *gbs) {
  Probe<Baseline> p(nx, ny, nz);
  if (gflops) *gflops = p.GFlops(count, time);
  if (gbs) *gbs = p.Throughput(count, time);
  return 0;
}

}  // extern "C"
