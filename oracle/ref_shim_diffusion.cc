// Test infrastructure only (the checker, never the product).
//
// The extern "C" probe of oracle/ref_shim.cc, for the reference's second
// plugin surface, diffusion::Diffusion (src/diffusion/diffusion.h:80-180):
// 2D 5-point and 3D 7-point grids through one class family.  Compiled from
// the reference sources in place by oracle/Makefile into
// oracle/_ref/libdif_ref.so.  It subclasses the reference classes to reach
// their protected state (f1_, the seven coefficients, the geometry) so tests
// can feed seeded, non-square inputs and read back what the reference
// computed.
//
// Backends probed:
//   0  diffusion::DiffusionOpenMP   diffusion_openmp.cc:5-121
//   1  diffusion::Baseline          baseline.h:10-109
#include <stdlib.h>
#include <string.h>

#include "diffusion/baseline.h"
#include "diffusion/diffusion_openmp.h"

namespace {

using diffusion::Baseline;
using diffusion::DiffusionOpenMP;

template <class Backend>
class Probe : public Backend {
 public:
  Probe(int nd, const int *dims) : Backend(nd, dims) {}

  void DoSetup() { this->Setup(); }
  void DoInitialize() { this->InitializeInput(); }
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
  float GFlops(int count, float t) { return this->GetGFLOPS(count, t); }
  float Throughput(int count, float t) { return this->GetThroughput(count, t); }
};

template <class Backend>
int RunProbe(int nd, const int *dims, const float *coeff, const float *in,
             float *init_out, float *out, int count, float *accuracy) {
  Probe<Backend> p(nd, dims);
  p.DoSetup();
  p.DoInitialize();
  if (init_out) p.GetField(init_out);
  if (coeff) p.SetCoeffs(coeff);
  if (in) p.SetField(in);
  p.Run(count);
  if (out) p.GetField(out);
  if (accuracy) *accuracy = p.Accuracy(count);
  p.Teardown();
  return 0;
}

}  // namespace

extern "C" {

// Runs `count` steps of the chosen backend on an nd-dimensional grid
// (dims[0..nd-1] = nx, ny[, nz]).  `coeff` (7 floats) and `in` override
// what the reference's constructor and InitializeInput produce; the field
// InitializeInput produced lands in `init_out`, the field after `count`
// steps (the reference's f1_) in `out`, each when non-null.
int difref_run(int backend, int nd, const int *dims, const float *coeff,
               const float *in, float *init_out, float *out, int count,
               float *accuracy) {
  if (nd < 2 || nd > 3) return -1;
  switch (backend) {
    case 0:
      return RunProbe<DiffusionOpenMP>(nd, dims, coeff, in, init_out, out,
                                       count, accuracy);
    case 1:
      return RunProbe<Baseline>(nd, dims, coeff, in, init_out, out, count,
                                accuracy);
    default:
      return -1;
  }
}

// The constructor's derived quantities (diffusion.h:93-108).
int difref_params(int nd, const int *dims, float *coeff, float *geom) {
  if (nd < 2 || nd > 3) return -1;
  Probe<Baseline> p(nd, dims);
  if (coeff) p.GetCoeffs(coeff);
  if (geom) p.GetGeometry(geom);
  return 0;
}

// The header's inline Initialize (diffusion.h:48-77), which Baseline's
// InitializeInput and GetCorrectAnswer call.
int difref_initialize(float *buf, int nx, int ny, int nz, float kx, float ky,
                      float kz, float dx, float dy, float dz, float kappa,
                      float time, int nd) {
  diffusion::Initialize(buf, nx, ny, nz, kx, ky, kz, dx, dy, dz, kappa, time,
                        nd);
  return 0;
}

// GetThroughput / GetGFLOPS (diffusion.h:156-163).
int difref_rates(int nd, const int *dims, int count, float time,
                 float *gflops, float *gbs) {
  if (nd < 2 || nd > 3) return -1;
  Probe<Baseline> p(nd, dims);
  if (gflops) *gflops = p.GFlops(count, time);
  if (gbs) *gbs = p.Throughput(count, time);
  return 0;
}

}  // extern "C"
