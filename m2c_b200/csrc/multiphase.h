// Two-material machinery attached to a context: level set, material IDs,
// interface exact Riemann problems and the post-step multiphase update.
#pragma once
#include <cuda_runtime.h>

#include "../../include/m2c_gpu.h"
#include "stage.cuh"

namespace m2c {
struct Multiphase;
}
using m2c::Multiphase;

// xc/dx: host cell centres and widths per axis.
m2cg_status multiphase_create(cudaStream_t s, const m2c::Grid3& g, const m2c::SchemeK& sk, const m2cg_scheme& scheme,
                              const m2cg_material* mats, int nmat, const m2cg_levelset& ls, const double* const* xc,
                              const double* const* dx, Multiphase** out);
void multiphase_destroy(Multiphase* mp);
m2cg_status multiphase_upload_phi(Multiphase* mp, cudaStream_t s, const double* phi_host, double* staging,
                                  uint8_t* id);
m2cg_status multiphase_download_phi(Multiphase* mp, cudaStream_t s, double* phi_host);
void multiphase_set_step(Multiphase* mp, int time_step);
// Called before the stages of a step (V^n, ID) and before each stage launch
// (fills the interface fields of the stage arguments).
m2cg_status multiphase_begin_step(Multiphase* mp, cudaStream_t s, double* const* Vn, const uint8_t* id);
// LINEAR interface reconstruction: turns a copy of the stage's arguments into
// the face pass (the stage kernel writing the reconstructed states on both
// sides of each interface face, launched before multiphase_stage); false if
// the scheme needs none.
bool multiphase_face_pass(Multiphase* mp, m2c::StageArgs& a);
m2cg_status multiphase_stage(Multiphase* mp, cudaStream_t s, m2c::StageArgs& a);
// After the last stage: level-set update, ID update, reinitialisation,
// state update of cells that changed material.
m2cg_status multiphase_end_step(Multiphase* mp, cudaStream_t s, double* const* Vn, double* const* Vnew,
                                float* const* Vfnew, uint8_t* id,
                                const double* clock, m2c::DevError* err, m2cg_counters* counters);
void multiphase_counters(const Multiphase* mp, m2cg_counters* out);
// Attach (m != NULL) or detach the learned warm start of the interface
// Riemann solves; allocates the per-face feature buffers on first use.
m2cg_status multiphase_set_mlp(Multiphase* mp, const m2cg_mlp* m);
// The state update of cells whose ID differs from the step-start IDs
// (multiphase_idn): Riemann-solution or extrapolation pass, FixUnresolvedNodes,
// clip. use_rs: the stage-1 star states of the last step are valid for these IDs.
// in_step: called at the end of a step (the step's counts go to the run
// totals, no host round trip); otherwise *unresolved (may be NULL) receives
// the cells handed to FixUnresolvedNodes after a read-back.
m2cg_status multiphase_update_states(Multiphase* mp, cudaStream_t s, double* const* V, float* const* Vf, uint8_t* id,
                                     m2c::DevError* err, bool use_rs, bool in_step, int* unresolved);
uint8_t* multiphase_idn(Multiphase* mp);
