// DiffusionB200: the B200 backend of the diffusion benchmark (2D 5-point
// and 3D 7-point grids), a peer of the reference's DiffusionCUDA
// (src/diffusion/diffusion_cuda.h:30-61).
//
// Drop-in: this header compiles against the reference's own
// "diffusion/baseline.h" (add -I<reference>/src) or against the restated
// plugin surface in plugin/mirror/ (standalone builds).  The class keeps the
// reference's contract: Setup allocates a pinned host f1_ and the device
// buffers; InitializeInput (inherited from Baseline) fills f1_ with the
// analytic field; RunKernel(count) starts from host f1_ and leaves the field
// after `count` steps in host f1_; GetAccuracy and Dump (inherited) read
// f1_; FinalizeBenchmark frees everything.  All device work goes through the
// C ABI of libd3d_b200.so (include/d3d_b200.h); no CUDA headers needed.
#ifndef DIFFUSION_DIFFUSION_B200_H_
#define DIFFUSION_DIFFUSION_B200_H_

#include <string>

#include "diffusion/baseline.h"

extern "C" {
#include "d3d_b200.h"
}

namespace diffusion {

class DiffusionB200 : public Baseline {
 public:
  // kernel: D3D_KERNEL_* (AUTO: the 2D register march in 2D, the TMA
  // z-march where eligible in 3D); tb_depth: fused steps for D3D_KERNEL_TB
  // (3D only); binary_dump: Dump writes a binary checkpoint
  // (d3d_checkpoint_save_host) instead of the "%.7E" text.
  DiffusionB200(int nd, const int* dims, int kernel = D3D_KERNEL_AUTO,
                int tb_depth = 1, bool binary_dump = false)
      : Baseline(nd, dims), kernel_(kernel), tb_depth_(tb_depth),
        binary_dump_(binary_dump) {}
  virtual ~DiffusionB200() {}
  virtual std::string GetName() const;
  virtual std::string GetDescription() const;
  virtual void Setup();
  virtual void WarmingUp() { RunKernel(50); }  // as DiffusionCUDA's
  virtual void RunKernel(int count);
  virtual void FinalizeBenchmark();
  virtual void DisplayResult(int count, float time);
  virtual void Dump() const;

 protected:
  int kernel_, tb_depth_;
  bool binary_dump_;
  int steps_done_ = 0;
  d3d_plan plan_ = nullptr;
  void* f1_d_ = nullptr;
  void* f2_d_ = nullptr;
  float kernel_ms_ = 0.0f;
};

}  // namespace diffusion

#endif  // DIFFUSION_DIFFUSION_B200_H_
