// Host-side launchers for the stage kernels, one translation unit per
// precision. The FP64 instantiations live in a unit compiled without FMA
// contraction (-fmad=false) so that their arithmetic rounds like the
// reference's x86-64 build; the mixed instantiations keep contraction on.
#pragma once
#include <cuda_runtime.h>

#include "stage.cuh"

namespace m2c {

constexpr int STAGE_TY = 8;
#ifndef M2C_STAGE_TY_F32
#define M2C_STAGE_TY_F32 16
#endif
// Tile height per instantiation: 32 x 8 for the FP64 kernels, 32 x 16 for
// the FP32 (mixed) kernels.
template <typename T, bool MULTI> struct StageTY { static constexpr int value = STAGE_TY; };
template <bool MULTI> struct StageTY<float, MULTI> { static constexpr int value = M2C_STAGE_TY_F32; };

size_t stage_smem_fp64(bool multi);
size_t stage_smem_mixed(bool multi);
// Launch one stage on a persistent grid of min(nitems, SMs x resident CTAs
// per SM) CTAs sharing the work evenly. *grid_out reports the grid.
cudaError_t launch_stage_fp64(const StageArgs& a, cudaStream_t s, bool multi, int* grid_out);
cudaError_t launch_stage_mixed(const StageArgs& a, cudaStream_t s, bool multi, int* grid_out);
// Resident CTAs on the whole device of the stage kernel for (flux, multi);
// each precision's translation unit instantiates only its own kernels.
int stage_resident_fp64(int flux, bool multi);
int stage_resident_mixed(int flux, bool multi);

template <typename T, int FLUX, bool MULTI, bool CONS = false, bool WALLS = false>
cudaError_t stage_occupancy(int* per_sm, int* nsm) {
  constexpr int TY = StageTY<T, MULTI>::value;
  auto k = stage_kernel<T, TY, FLUX, MULTI, CONS, WALLS>;
  const size_t smem = sizeof(StageSmemAll<T, TY, MULTI>);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0;
  cudaGetDevice(&dev);
  e = cudaDeviceGetAttribute(nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, TX * TY, smem);
  if (*per_sm < 1) *per_sm = 1;
  return e;
}

template <typename T, int FLUX, bool MULTI, bool CONS, bool WALLS = false>
cudaError_t launch_stage_one(const StageArgs& a, cudaStream_t s, int* grid_out) {
  constexpr int TY = StageTY<T, MULTI>::value;
  auto k = stage_kernel<T, TY, FLUX, MULTI, CONS, WALLS>;
  const size_t smem = sizeof(StageSmemAll<T, TY, MULTI>);
  int per_sm = 1, nsm = 148;
  cudaError_t e = stage_occupancy<T, FLUX, MULTI, CONS, WALLS>(&per_sm, &nsm);
  if (e != cudaSuccess) return e;
  int grid = a.nitems < per_sm * nsm ? a.nitems : per_sm * nsm;
  if (grid_out) *grid_out = grid;
  k<<<grid, dim3(TX, TY), smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T, int FLUX>
cudaError_t launch_stage_f(const StageArgs& a, cudaStream_t s, bool multi, int* g) {
  const bool cons = a.s.rec_var != 0 && a.s.rec_linear;
  if (multi && a.wall.mask)  // faces cut by an embedded surface attached
    return cons ? launch_stage_one<T, FLUX, true, true, true>(a, s, g)
                : launch_stage_one<T, FLUX, true, false, true>(a, s, g);
  if (multi)
    return cons ? launch_stage_one<T, FLUX, true, true>(a, s, g) : launch_stage_one<T, FLUX, true, false>(a, s, g);
  return cons ? launch_stage_one<T, FLUX, false, true>(a, s, g) : launch_stage_one<T, FLUX, false, false>(a, s, g);
}

template <typename T>
cudaError_t launch_stage_t(const StageArgs& a, cudaStream_t s, bool multi, int* g) {
  switch (a.s.flux) {
    case FLUX_ROE: return launch_stage_f<T, FLUX_ROE>(a, s, multi, g);
    case FLUX_LLF: return launch_stage_f<T, FLUX_LLF>(a, s, multi, g);
    default: return launch_stage_f<T, FLUX_HLLC>(a, s, multi, g);
  }
}

template <typename T>
int blocks_per_sm_t(int flux, bool multi) {
  int per_sm = 1, nsm = 148;
  switch (flux) {
    case FLUX_ROE:
      multi ? stage_occupancy<T, FLUX_ROE, true>(&per_sm, &nsm) : stage_occupancy<T, FLUX_ROE, false>(&per_sm, &nsm);
      break;
    case FLUX_LLF:
      multi ? stage_occupancy<T, FLUX_LLF, true>(&per_sm, &nsm) : stage_occupancy<T, FLUX_LLF, false>(&per_sm, &nsm);
      break;
    default:
      multi ? stage_occupancy<T, FLUX_HLLC, true>(&per_sm, &nsm) : stage_occupancy<T, FLUX_HLLC, false>(&per_sm, &nsm);
  }
  return per_sm * nsm;
}

}  // namespace m2c
