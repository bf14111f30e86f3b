// FP64 instantiations of the fused stage kernel. Built with -fmad=false:
// every multiply and add rounds separately, as in the reference's x86-64
// build, which keeps the FP64 path bit-compatible with it.
#include "launch.h"

namespace m2c {

size_t stage_smem_fp64(bool multi) {
  return multi ? sizeof(StageSmemAll<double, StageTY<double, true>::value, true>)
               : sizeof(StageSmemAll<double, StageTY<double, false>::value, false>);
}

cudaError_t launch_stage_fp64(const StageArgs& a, cudaStream_t s, bool multi, int* grid_out) {
  return launch_stage_t<double>(a, s, multi, grid_out);
}

int stage_resident_fp64(int flux, bool multi) { return blocks_per_sm_t<double>(flux, multi); }

}  // namespace m2c
