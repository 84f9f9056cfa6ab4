// Baseline of the diffusion plugin surface, restated for builds without the
// reference tree (the reference's is src/diffusion/baseline.h:10-109).  It
// owns the host field f1_/f2_ and provides the accuracy report and the text
// dump that every backend inherits.  The serial stencil loop itself is not
// restated: a backend built on this surface supplies RunKernel.
#ifndef DIFFUSION_BASELINE_H_
#define DIFFUSION_BASELINE_H_

#include <string>

#include "diffusion/diffusion.h"

namespace diffusion {

class Baseline : public Diffusion {
 protected:
  REAL *f1_, *f2_;

 public:
  Baseline(int ndim, const int* dims)
      : Diffusion(ndim, dims), f1_(NULL), f2_(NULL) {}
  virtual std::string GetName() const {
    return "baseline" + std::to_string(ndim_) + "d";
  }
  virtual std::string GetDescription() const {
    return "baseline serial implementation";
  }
  virtual void Setup();
  virtual void InitializeInput();
  virtual void FinalizeBenchmark();
  virtual void RunKernel(int count);
  virtual void WarmingUp() { RunKernel(1); }
  virtual REAL GetAccuracy(int count);
  virtual void Dump() const;
};

}  // namespace diffusion

#endif  // DIFFUSION_BASELINE_H_
