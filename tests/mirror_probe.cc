// Test-only probe of the restated plugin surface
// (benchmarks_b200/plugin/mirror): exposes the constructor's coefficients,
// Initialize, GetAccuracy and Dump through extern "C" so tests can compare
// them with the reference's golden data.  Built by tests/test_plugin.py.
#include <string.h>

#include "diffusion3d/baseline.h"

namespace {

class Probe : public diffusion3d::Baseline {
 public:
  Probe(int nx, int ny, int nz) : Baseline(nx, ny, nz) {}
  virtual std::string GetName() const { return "probe"; }
  void Coeffs(float* c, float* g) const {
    const float cc[7] = {ce_, cw_, cn_, cs_, ct_, cb_, cc_};
    const float gg[8] = {kappa_, dx_, dy_, dz_, kx_, ky_, kz_, dt_};
    memcpy(c, cc, sizeof cc);
    memcpy(g, gg, sizeof gg);
  }
  void Setup() { InitializeBenchmark(); }
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

int mirror_params(int nx, int ny, int nz, float* c, float* g) {
  Probe p(nx, ny, nz);
  p.Coeffs(c, g);
  return 0;
}

int mirror_initial_field(int nx, int ny, int nz, float* out) {
  Probe p(nx, ny, nz);
  p.Setup();
  p.Get(out);
  p.Teardown();
  return 0;
}

float mirror_accuracy(int nx, int ny, int nz, const float* field, int count) {
  Probe p(nx, ny, nz);
  p.Setup();
  p.Set(field);
  const float a = p.Acc(count);
  p.Teardown();
  return a;
}

int mirror_dump(int nx, int ny, int nz, const float* field) {
  Probe p(nx, ny, nz);
  p.Setup();
  p.Set(field);
  p.DumpIt();
  p.Teardown();
  return 0;
}

float mirror_rates(int nx, int ny, int nz, int count, float t, float* gbs) {
  Probe p(nx, ny, nz);
  return p.Rates(count, t, gbs);
}

}  // extern "C"
