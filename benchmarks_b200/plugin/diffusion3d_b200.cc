// Diffusion3DB200 over the C ABI (see diffusion3d_b200.h).
#include "diffusion3d_b200.h"

#include <stdio.h>
#include <stdlib.h>

namespace diffusion3d {

namespace {

// The reference's failure convention (assert / exit, diffusion3d_cuda.cu:6-9
// and common/cuda_util.h:4-12): report and stop.
void Check(int rc, const char* what) {
  if (rc != D3D_OK) {
    fprintf(stderr, "%s failed (%d): %s\n", what, rc, d3d_last_error());
    exit(EXIT_FAILURE);
  }
}

}  // namespace

std::string Diffusion3DB200::GetName() const {
  if (kernel_ == D3D_KERNEL_TB)
    return std::string("b200_tb") + std::to_string(tb_depth_);
  if (kernel_ == D3D_KERNEL_GENERIC) return "b200_generic";
  return "b200";
}

// As Diffusion3DCUDA::InitializeBenchmark (diffusion3d_cuda.cu:329-341):
// pinned host f1_, analytic field at t = 0, two device buffers.
void Diffusion3DB200::InitializeBenchmark() {
  const size_t bytes = sizeof(REAL) * (size_t)nx_ * ny_ * nz_;
  const int dtype = sizeof(REAL) == 8 ? D3D_F64 : D3D_F32;
  Check(d3d_plan_create(nx_, ny_, nz_, dtype, kernel_, tb_depth_, &plan_),
        "d3d_plan_create");
  void* host = nullptr;
  Check(d3d_host_alloc(bytes, &host), "d3d_host_alloc");
  f1_ = static_cast<REAL*>(host);
  f2_ = nullptr;  // the second buffer lives on the device only
  Initialize(f1_, nx_, ny_, nz_, kx_, ky_, kz_, dx_, dy_, dz_, kappa_, 0.0);
  Check(d3d_device_alloc(bytes, &f1_d_), "d3d_device_alloc");
  Check(d3d_device_alloc(bytes, &f2_d_), "d3d_device_alloc");
}

// As Diffusion3DCUDA::RunKernel (diffusion3d_cuda.cu:353-371): host f1_ in,
// `count` steps on the device, result back in host f1_.
void Diffusion3DB200::RunKernel(int count) {
  const REAL coeff[7] = {ce_, cw_, cn_, cs_, ct_, cb_, cc_};
  Check(d3d_run_host(plan_, f1_, f1_d_, f2_d_, coeff, count, nullptr,
                     &kernel_ms_),
        "d3d_run_host");
  steps_done_ = count;
}

// The reference's text dump (Baseline::Dump), or with binary_dump the
// checkpoint of host f1_ beside it: <dump path without ".out">.d3d.
void Diffusion3DB200::Dump() const {
  if (!binary_dump_) return Baseline::Dump();
  std::string path = GetDumpPath();
  if (path.size() > 4 && path.compare(path.size() - 4, 4, ".out") == 0)
    path.resize(path.size() - 4);
  path += ".d3d";
  Check(d3d_checkpoint_save_host(plan_, f1_, steps_done_, path.c_str()),
        "d3d_checkpoint_save_host");
}

void Diffusion3DB200::FinalizeBenchmark() {
  Check(d3d_host_free(f1_), "d3d_host_free");
  f1_ = nullptr;
  Check(d3d_device_free(f1_d_), "d3d_device_free");
  Check(d3d_device_free(f2_d_), "d3d_device_free");
  f1_d_ = f2_d_ = nullptr;
  d3d_plan_destroy(plan_);
  plan_ = nullptr;
}

// Baseline's report plus the kernel-only block of
// Diffusion3DCUDA::DisplayResult (diffusion3d_cuda.cu:373-384).
void Diffusion3DB200::DisplayResult(int count, float time) {
  Baseline::DisplayResult(count, time);
  const float t = kernel_ms_ * 1.0e-03f;
  printf("Kernel-only performance:\n");
  printf("Elapsed time : %.3f (s)\n", t);
  printf("FLOPS        : %.3f (GFLOPS)\n", GetGFLOPS(count, t));
  printf("Throughput   : %.3f (GB/s)\n", GetThroughput(count, t));
}

}  // namespace diffusion3d
