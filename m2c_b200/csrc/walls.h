// Faces cut by embedded surfaces (walls) in the fused stage
// (SpaceOperator::ComputeAdvectionFluxes, SpaceOperator.cpp:2438-2484 and its
// y/z analogues 2568-2612, 2695-2739).
//
// The caller supplies, per cut face, what the reference's intersector data
// yields through FindEdgeSurfaceIntersections (SpaceOperator.cpp:3435-3501):
// the unit normal and the velocity of the surface at the intersection seen
// from the face's low cell ("forward") and from its high cell ("backward").
// Each stage, a pre-pass solves the two one-sided Riemann problems of every
// cut face (ExactRiemannSolverBase::ComputeOneSidedRiemannSolution, the
// direction from GetNormalForOneSidedRiemann, 3505-3530) on the stage's
// cell-centred states and clips the star states; the stage kernel then gives
// each side its numerical flux against its own star state.
#pragma once
#include <cuda_runtime.h>

#include "../../include/m2c_gpu.h"
#include "stage.cuh"

namespace m2c {

struct Walls;

// faces [n][4] = (axis d, i, j, k): the face between cell (i, j, k) and its
// low neighbour along d; nf, uf, nb, ub [n][3]. On refusal *out stays NULL
// and msg says why.
m2cg_status walls_create(cudaStream_t s, const Grid3& g, size_t nalloc, const m2cg_scheme& scheme, int n,
                         const int* faces, const double* nf, const double* uf, const double* nb, const double* ub,
                         Walls** out, char* msg, size_t msglen);
void walls_destroy(Walls* w);
// The one-sided solves of the stage whose arguments are a; fills a.wall.
m2cg_status walls_stage(Walls* w, cudaStream_t s, StageArgs& a);
// The cut faces' view without solving (the interface pre-pass skips them).
void walls_view(const Walls* w, StageArgs& a);
// LINEAR reconstruction at the surface: makes a the arguments of the face
// pass that writes the cut faces' reconstructed states (false: none needed).
bool walls_face_pass(const Walls* w, StageArgs& a);
// One-sided solves so far and how many of them the solver reported as
// failed (the reference's riemann_errors, SpaceOperator.cpp:2446-2447).
void walls_counters(Walls* w, cudaStream_t s, long long* solves, long long* failures);

}  // namespace m2c
