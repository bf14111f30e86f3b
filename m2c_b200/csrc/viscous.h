// Viscous fluxes of constant-viscosity materials on the GPU
// (ViscosityOperator::AddDiffusionFluxes, ViscosityOperator.cpp:200-408, with
// ViscoFcnConstant, ViscoFcn.h, InterpolatorLinear, Interpolator.cpp, and
// GradientCalculatorCentral, GradientCalculatorCentral.cpp).
//
// One kernel per stage forms, on every cell face, the area-weighted viscous
// flux the right cell adds to its flux sum and the one the left cell
// subtracts (they differ only where the face separates two materials); the
// stage kernel adds them to each cell's flux sum in the reference's order
// before dividing by the volume.
#pragma once
#include <cuda_runtime.h>

#include "../../include/m2c_gpu.h"
#include "stage.cuh"

namespace m2c {

struct Viscous;

// eos: the materials' FP64 EOS (temperature laws); xc/dx: host cell centres
// and widths per axis. *out = NULL (and M2CG_OK) when no material is
// viscous or heat-diffusive.
m2cg_status viscous_create(cudaStream_t s, const Grid3& g, const Eos<double>* eos, const m2cg_material* mats,
                           int nmat, const double* const* xc, const double* const* dx, Viscous** out);
void viscous_destroy(Viscous* v);
// Whether any material is viscous (heat diffusion alone: false).
bool viscous_has_viscosity(const Viscous* v);
// Faces of the stage whose arguments are a (its input state a.Pin in the
// compute type: float when mixed); fills a.visc.
m2cg_status viscous_faces(Viscous* v, cudaStream_t s, StageArgs& a, bool mixed);

}  // namespace m2c

using m2c::Viscous;
using m2c::viscous_create;
using m2c::viscous_destroy;
using m2c::viscous_has_viscosity;
using m2c::viscous_faces;
