// Level-set transport on the GPU: finite-difference UPWIND_CENTRAL_3 residual
// (LevelSetOperator::ComputeResidualFDM_FullDomain, LevelSetOperator.cpp:1066-1140,
// GradientCalculatorFD3.cpp:54-470) or finite-volume residual
// (LevelSetOperator::ComputeResidualFVM, 1237-1297, 1342-1419, 1516-1570), boundary rules
// (LevelSetOperator::ApplyBoundaryConditions, 934-1034) and reinitialisation
// (LevelSetReinitializer::ReinitializeFullDomain).
#pragma once
#include <cuda_runtime.h>

#include "../../include/m2c_gpu.h"
#include "stage.cuh"

namespace m2c {

// Per-axis geometry of the level-set operator, on the device.
struct LsGeom {
  const double* xg[3];   // coordinates incl. one ghost per side: index c+1 for c in [-1, n]
  const double* cl[3];   // left-biased FD3 coefficients [n][4] (third order where i > 0)
  const double* cr[3];   // right-biased FD3 coefficients [n][4] (third order where i < n-1)
  const double* cr1y;    // right-biased first-order y coefficients [ny][4] (see levelset.cu)
  // finite-volume solver: widths incl. one ghost per side (index c+1; a
  // ghost has the width of its boundary cell, SpaceOperator::ResetGhostLayer)
  // and the level set's own limiter coefficients per axis index
  // (Reconstructor::Setup with the level set's ReconstructionData)
  const double* wg[3];
  const double* fA[3];
  const double* fB[3];
  const double* fK[3];   // van Albada exponent (an integer held in a double; 0 otherwise)
  int solver, flux, rec_linear, limiter;
  double delta, alpha;
  int bc[6];             // LevelSetSchemeData::BcType per side
  double* base;          // single allocation holding the arrays above
};

// xc/dx: host cell centres and widths per axis (length n of that axis).
m2cg_status levelset_geom_create(cudaStream_t s, const Grid3& g, const m2cg_levelset& ls, const double* const* xc,
                                 const double* const* dx, LsGeom* out);
void levelset_geom_destroy(LsGeom* geo);
void levelset_unpack(cudaStream_t s, const Grid3& g, const double* aos, double* phi);
void levelset_pack(cudaStream_t s, const Grid3& g, const LsGeom& geo, const double* phi, double* aos);
// One level-set RK stage: out = a_prev*in + a_un*phi_n + (bdt_coef*dt)*R(in, V_stage)
// (stage 1: out = phi_n + dt*R).
m2cg_status levelset_stage(cudaStream_t s, const Grid3& g, const SchemeK& sk, const LsGeom& geo, const StageArgs& a,
                           const double* in, const double* phin, double* out);
// first_layer: LevelSetReinitializationData::firstLayerTreatment (the
// treatments other than FIXED need per-cell correction and normal arrays).
m2cg_status reinit_alloc(long long ncell, int first_layer, double** buf);
// cfl_state: the pseudo-time CFL number, reduced in place on a failed attempt
// and kept for later calls (as LevelSetReinitializer::cfl is).
m2cg_status levelset_reinitialize(cudaStream_t s, const Grid3& g, const LsGeom& geo, const m2cg_levelset& ls,
                                  double* phi, double* buf, DevError* err, double* cfl_state, int* iterations);

}  // namespace m2c

using m2c::LsGeom;
using m2c::levelset_geom_create;
using m2c::levelset_geom_destroy;
using m2c::levelset_unpack;
using m2c::levelset_pack;
using m2c::levelset_stage;
using m2c::reinit_alloc;
using m2c::levelset_reinitialize;
