// Diffusion3DB200: the B200 backend of the diffusion3d benchmark, a peer of
// the reference's Diffusion3DCUDA (src/diffusion3d/diffusion3d_cuda.h:26-49).
//
// Drop-in: this header compiles against the reference's own
// "diffusion3d/baseline.h" (add -I<reference>/src) or against the restated
// plugin surface in plugin/mirror/ (standalone builds).  The class keeps the
// reference's contract: InitializeBenchmark fills host f1_ with the analytic
// field and allocates device buffers; RunKernel(count) starts from host f1_
// and leaves the field after `count` steps in host f1_; GetAccuracy and Dump
// (inherited from Baseline) read f1_; FinalizeBenchmark frees everything.
// All device work goes through the C ABI of libd3d_b200.so
// (include/d3d_b200.h); this file needs no CUDA headers.
#ifndef DIFFUSION3D_DIFFUSION3D_B200_H_
#define DIFFUSION3D_DIFFUSION3D_B200_H_

#include <string>

#include "diffusion3d/baseline.h"

extern "C" {
#include "d3d_b200.h"
}

namespace diffusion3d {

class Diffusion3DB200 : public Baseline {
 public:
  // kernel: D3D_KERNEL_* (AUTO = TMA z-march where eligible); tb_depth: the
  // fused step count for D3D_KERNEL_TB; binary_dump: Dump writes a binary
  // checkpoint (d3d_checkpoint_save_host) instead of the "%.7E" text.
  Diffusion3DB200(int nx, int ny, int nz, int kernel = D3D_KERNEL_AUTO,
                  int tb_depth = 1, bool binary_dump = false)
      : Baseline(nx, ny, nz), kernel_(kernel), tb_depth_(tb_depth),
        binary_dump_(binary_dump) {}
  virtual ~Diffusion3DB200() {}
  virtual std::string GetName() const;
  virtual void InitializeBenchmark();
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

}  // namespace diffusion3d

#endif  // DIFFUSION3D_DIFFUSION3D_B200_H_
