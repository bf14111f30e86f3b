// Mixed-precision instantiation of the fused stage kernel: reconstruction and
// fluxes in FP32 (FP32 accumulation), while the conserved-state RK update,
// the conservative-to-primitive pressure recovery and the residual sum stay
// FP64 (the recovery p = (gamma-1) rho e - gamma p_inf cancels ~1e9 Pa terms
// down to ~1e5 Pa for water and must not be done in FP32).
#include "launch.h"

namespace m2c {

size_t stage_smem_mixed() { return sizeof(StageSmem<float, STAGE_TY>); }

cudaError_t launch_stage_mixed(const StageArgs& a, dim3 grid, cudaStream_t s) {
  static bool configured = false;
  size_t smem = stage_smem_mixed();
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<float, STAGE_TY>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  stage_kernel<float, STAGE_TY><<<grid, dim3(TX, STAGE_TY), smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace m2c
