// FP64 instantiation of the fused stage kernel. Built with -fmad=false: every
// multiply and add rounds separately, as in the reference's x86-64 build,
// which keeps the FP64 path bit-compatible with it.
#include "launch.h"

namespace m2c {

size_t stage_smem_fp64() { return sizeof(StageSmem<double, STAGE_TY>); }

cudaError_t launch_stage_fp64(const StageArgs& a, dim3 grid, cudaStream_t s) {
  static bool configured = false;
  size_t smem = stage_smem_fp64();
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<double, STAGE_TY>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  stage_kernel<double, STAGE_TY><<<grid, dim3(TX, STAGE_TY), smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace m2c
