// Launch interface of the batched exact Riemann kernel (used by the
// m2cg_riemann_batch entry point and by the two-material stage pre-pass).
#pragma once
#include <cuda_runtime.h>

#include "../../include/m2c_gpu.h"
#include "riemann.cuh"

namespace m2c {

constexpr int MAXMAT_RIEMANN = 4;
// Points per integration-path cache (per wave, per problem). The reference
// grows a std::vector without bound; exhausting this capacity is reported.
constexpr int RIEMANN_PATH_CAP = 512;

struct RiemannBatchArgs {
  long long n;
  RiemannParams P;
  const Eos<double>* eos;
  const double* VL;    // [n][5]
  const double* VR;    // [n][5]
  const double* dir;   // [n][3]
  const int* idl;
  const int* idr;
  const double* warm;  // [n] or nullptr
  double* Vs;          // [n][5]
  double* Vsm;
  double* Vsp;
  int* id;
  int* iters;          // or nullptr
  int* evals;          // or nullptr: star-state evaluations per problem
  int* err;
  double* scratch;     // integration paths: [slots][2 waves][path_cap][3]
  int path_cap;
  long long scratch_slots;
};

RiemannParams riemann_params(const m2cg_scheme& s);
cudaError_t launch_riemann_batch(const RiemannBatchArgs& a, cudaStream_t s);

}  // namespace m2c
