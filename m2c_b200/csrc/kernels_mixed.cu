// Mixed-precision instantiations of the fused stage kernel: reconstruction
// and fluxes in FP32 (FP32 accumulation), while the conserved-state RK
// update, the conservative-to-primitive pressure recovery and the residual
// sum stay FP64 (the recovery p = (gamma-1) rho e - gamma p_inf cancels
// ~1e9 Pa terms down to ~1e5 Pa for water and must not be done in FP32).
#include "launch.h"

namespace m2c {

size_t stage_smem_mixed(bool multi) {
  return multi ? sizeof(StageSmemAll<float, StageTY<float, true>::value, true>)
               : sizeof(StageSmemAll<float, StageTY<float, false>::value, false>);
}

cudaError_t launch_stage_mixed(const StageArgs& a, cudaStream_t s, bool multi, int* grid_out) {
  return launch_stage_t<float>(a, s, multi, grid_out);
}

int stage_resident_mixed(int flux, bool multi) { return blocks_per_sm_t<float>(flux, multi); }

}  // namespace m2c
