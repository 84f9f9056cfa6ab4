// Test-only probe of the restated diffusion plugin surface
// (benchmarks_b200/plugin/mirror/diffusion): exposes the constructor's
// coefficients, InitializeInput, GetAccuracy, the rates and Dump through
// extern "C" so tests can compare them with the reference's golden data.
// Built by tests/test_plugin_diffusion.py.
#include <string.h>

#include "diffusion/baseline.h"

namespace {

class Probe : public diffusion::Baseline {
 public:
  Probe(int nd, const int* dims) : Baseline(nd, dims) {}
  virtual std::string GetName() const { return "probe"; }
  void Coeffs(float* c, float* g) const {
    const float cc[7] = {ce_, cw_, cn_, cs_, ct_, cb_, cc_};
    const float gg[8] = {kappa_, dx_, dy_, dz_, kx_, ky_, kz_, dt_};
    memcpy(c, cc, sizeof cc);
    memcpy(g, gg, sizeof gg);
  }
  void Start() {
    Setup();
    InitializeInput();
  }
  void Teardown() { FinalizeBenchmark(); }
  size_t N() const { return (size_t)nx_ * ny_ * nz_; }
  void Get(float* out) const { memcpy(out, f1_, N() * 4); }
  void Set(const float* in) { memcpy(f1_, in, N() * 4); }
  float Acc(int count) { return GetAccuracy(count); }
  void DumpIt() const { Dump(); }
  float Rates(int count, float t, float* gbs) {
    *gbs = GetThroughput(count, t);
    return GetGFLOPS(count, t);
  }
};

}  // namespace

extern "C" {

int mirror_dif_params(int nd, const int* dims, float* c, float* g) {
  Probe p(nd, dims);
  p.Coeffs(c, g);
  return 0;
}

int mirror_dif_initial_field(int nd, const int* dims, float* out) {
  Probe p(nd, dims);
  p.Start();
  p.Get(out);
  p.Teardown();
  return 0;
}

float mirror_dif_accuracy(int nd, const int* dims, const float* field,
                          int count) {
  Probe p(nd, dims);
  p.Start();
  p.Set(field);
  const float a = p.Acc(count);
  p.Teardown();
  return a;
}

int mirror_dif_dump(int nd, const int* dims, const float* field) {
  Probe p(nd, dims);
  p.Start();
  p.Set(field);
  p.DumpIt();
  p.Teardown();
  return 0;
}

float mirror_dif_rates(int nd, const int* dims, int count, float t,
                       float* gbs) {
  Probe p(nd, dims);
  return p.Rates(count, t, gbs);
}

}  // extern "C"
