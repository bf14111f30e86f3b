// Host-side launchers for the stage kernels, one per precision. The FP64
// instantiation lives in a translation unit compiled without FMA
// contraction (-fmad=false) so that its arithmetic rounds like the
// reference's x86-64 build; the mixed instantiation keeps contraction on.
#pragma once
#include <cuda_runtime.h>

#include "stage.cuh"

namespace m2c {

// Shared-memory bytes and launch of one fused RK stage.
size_t stage_smem_fp64();
size_t stage_smem_mixed();
cudaError_t launch_stage_fp64(const StageArgs& a, dim3 grid, cudaStream_t s);
cudaError_t launch_stage_mixed(const StageArgs& a, dim3 grid, cudaStream_t s);
constexpr int STAGE_TY = 8;

}  // namespace m2c
