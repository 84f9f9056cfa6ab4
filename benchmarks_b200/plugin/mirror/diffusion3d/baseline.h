// Baseline of the diffusion3d plugin surface, restated for builds without
// the reference tree (the reference's is src/diffusion3d/baseline.h:8-22).
// It owns the host field f1_/f2_ and provides the accuracy report and the
// text dump that every backend inherits.  The serial stencil loop itself
// is not restated: a backend built on this surface supplies RunKernel.
#ifndef DIFFUSION3D_BASELINE_H_
#define DIFFUSION3D_BASELINE_H_

#include "diffusion3d/diffusion3d.h"

namespace diffusion3d {

class Baseline : public Diffusion3D {
 protected:
  REAL *f1_, *f2_;

 public:
  Baseline(int nx, int ny, int nz)
      : Diffusion3D(nx, ny, nz), f1_(NULL), f2_(NULL) {}
  virtual std::string GetName() const { return std::string("baseline"); }
  virtual void InitializeBenchmark();
  virtual void FinalizeBenchmark();
  virtual void RunKernel(int count);
  virtual REAL GetAccuracy(int count);
  virtual void Dump() const;
};

}  // namespace diffusion3d

#endif  // DIFFUSION3D_BASELINE_H_
