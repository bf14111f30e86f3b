/*
 * m2c_gpu.h — C ABI of the B200 (sm_100a) finite-volume step for M2C.
 *
 * The library replaces, on one structured subdomain, the explicit residual
 * and Runge-Kutta update of the M2C reference:
 *   SpaceOperator::ComputeResidual          (SpaceOperator.cpp:3351-3409)
 *   SpaceOperator::ComputeTimeStepSize      (SpaceOperator.cpp:2202-2227)
 *   TimeIntegratorRK2/RK3::AdvanceOneTimeStep (TimeIntegrator.cpp:291-428, 496-690)
 *   ExactRiemannSolverBase::ComputeRiemannSolution (ExactRiemannSolverBase.cpp:59-342)
 *   LevelSetOperator::ComputeResidual / Reinitialize, MultiPhaseOperator updates
 * The reference reaches these through C++ virtual dispatch per face and per
 * state; this boundary is field-level: one call advances a whole field.
 *
 * Conventions
 *  - Every entry point returns m2cg_status (0 = OK). The first failure inside
 *    a kernel is recorded (cell index, code) and readable with
 *    m2cg_last_error(); kernels never trap.
 *  - Host arrays use the reference's ghosted local-vector layout
 *    (SpaceVariable3D::GetDataPointer, SpaceVariable.cpp:254-261): a box of
 *    (nx+2)*(ny+2)*(nz+2) nodes, node (i,j,k) with i,j,k in [-1, n] stored at
 *    ((k+1)*(ny+2) + (j+1))*(nx+2) + (i+1); V carries 5 doubles per node
 *    (rho, u, v, w, p), ID and phi one double per node.
 *  - Host buffers are borrowed only for the duration of a call.
 *  - One context = one CUDA stream; calls are stream-ordered and a context is
 *    not thread-safe. Different contexts may be used from different threads.
 */
#ifndef M2C_GPU_H
#define M2C_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  M2CG_OK = 0,
  M2CG_ERR_ARG = 1,          /* bad argument or unsupported option */
  M2CG_ERR_CUDA = 2,         /* CUDA runtime error (message in m2cg_last_error) */
  M2CG_ERR_STATE = 3,        /* non-physical state (VarFcnBase::CheckState fails) */
  M2CG_ERR_RIEMANN = 4,      /* interface Riemann solver reported failures */
  M2CG_ERR_REINIT = 5,       /* level-set reinitialisation did not converge */
  M2CG_ERR_ITER_CAP = 6,     /* a device loop hit its iteration cap */
  M2CG_ERR_NOMEM = 7,        /* device allocation failed */
  M2CG_ERR_UNSUPPORTED = 8   /* option the GPU path does not implement */
} m2cg_status;

/* Boundary types: values of MeshData::BcType (IoData.h:266-267), plus
 * PERIODIC, which the reference cannot express (extension). */
enum {
  M2CG_BC_NONE = 0, M2CG_BC_INLET = 1, M2CG_BC_OUTLET = 2, M2CG_BC_SLIPWALL = 3,
  M2CG_BC_STICKWALL = 4, M2CG_BC_SYMMETRY = 5, M2CG_BC_PERIODIC = 100
};

/* Mesh and boundary conditions (MeshData, IoData.h:255-278; BcsData inlet/outlet).
 * Cell centres/widths: uniform as MeshGenerator::ComputeMesh1DUniform
 * (MeshGenerator.cpp:146-158) unless xc/dx (etc.) are given (length nx). */
typedef struct {
  int nx, ny, nz;
  double x0, xmax, y0, ymax, z0, zmax;
  const double *xc, *dx, *yc, *dy, *zc, *dz; /* optional non-uniform mesh, else NULL */
  int bc[6];              /* x0, xmax, y0, ymax, z0, zmax */
  double inlet[5];        /* primitive state at INLET ghosts */
  double outlet[5];       /* primitive state at OUTLET ghosts */
} m2cg_grid;

/* Material (MaterialModelData, IoData.h:458-486): SG (VarFcnSG.h) or NASG
 * (VarFcnNASG.h) with clipping bounds. */
enum { M2CG_EOS_SG = 0, M2CG_EOS_NASG = 1 };
typedef struct {
  int eos;
  double gamma;           /* specificHeatRatio */
  double p_c;             /* SG pressureConstant / NASG pressureConstant */
  double b;               /* NASG volumeConstant */
  double q;               /* NASG energyConstant */
  double rhomin, pmin, rhomax, pmax;
  double failsafe_density;
  /* ViscosityModelData CONSTANT (ViscoFcnConstant, ViscoFcn.h): dynamic and
   * bulk viscosity [Pa s]; both 0 = NONE (inviscid). With any material
   * viscous, the stage adds the viscous fluxes of ViscosityOperator::
   * AddDiffusionFluxes (ViscosityOperator.cpp:200-408) to the residual. */
  double mu, mu_bulk;
  /* HeatDiffusionModelData CONSTANT (HeatDiffusionFcn.h): diffusivity;
   * 0 = NONE. With any material diffusive, the stage adds the heat fluxes of
   * HeatDiffusionOperator::AddDiffusionFluxes (HeatDiffusionOperator.cpp:
   * 90-198). Temperature laws (VarFcnSG.h:70-78, VarFcnNASG.h:61): SG
   * T = T0 + (e - e0)/cv, or T = T0 + (e + p/rho - h0)/cp where cp > 0 and
   * cv <= 0; NASG T = (e - q - p_c (1/rho - b))/cv (1/0 read as 0). */
  double heat_diffusivity;
  double cv, T0, e0, cp, h0;
} m2cg_material;

/* Numerical scheme (SchemeData, ReconstructionData, TsData, MultiPhaseData,
 * ExactRiemannSolverData: IoData.h:544-795). Enum values are the reference's. */
enum { M2CG_FLUX_ROE = 0, M2CG_FLUX_LLF = 1, M2CG_FLUX_HLLC = 2 };
enum { M2CG_REC_CONSTANT = 0, M2CG_REC_LINEAR = 1 };
enum { M2CG_LIM_NONE = 0, M2CG_LIM_GENMINMOD = 1, M2CG_LIM_VANALBADA = 2 };
enum { M2CG_RECVAR_PRIMITIVE = 0, M2CG_RECVAR_CONSERVATIVE = 1,
       M2CG_RECVAR_PRIM_CHAR = 2, M2CG_RECVAR_CONS_CHAR = 3 };
enum { M2CG_PREC_FP64 = 0, M2CG_PREC_MIXED = 1 };
enum { M2CG_MPFLUX_EXACT = 0, M2CG_MPFLUX_NUMERICAL = 1, M2CG_MPFLUX_LLF = 2 };

typedef struct {
  int flux;               /* SchemeData::flux */
  double roe_delta;       /* SchemeData::delta (Harten entropy fix) */
  int rec_type;           /* ReconstructionData::type */
  int limiter;            /* ReconstructionData::limiter */
  double minmod_coeff;    /* ReconstructionData::generalized_minmod_coeff */
  int slope_near_interface; /* 0 ZERO, 1 NONZERO */
  int rec_var;            /* ReconstructionData::varType */
  int rk_order;           /* 1 (forward Euler), 2, 3 */
  double cfl;             /* TsData::cfl */
  int precision;          /* M2CG_PREC_FP64 or M2CG_PREC_MIXED */
  /* MultiPhaseData */
  int mp_flux;            /* EXACT / NUMERICAL / LLF */
  int mp_recon;           /* CONSTANT / LINEAR */
  int mp_phasechange_type;/* 0 RIEMANN_SOLUTION, 1 EXTRAPOLATION */
  int mp_phasechange_dir; /* 0 ALL, 1 UPWIND */
  int mp_apply_failsafe_density; /* 0 Off, 1 On */
  /* ExactRiemannSolverData */
  int riem_maxits_main, riem_maxits_bracket, riem_maxits_shock, riem_nsteps_rarefaction;
  double riem_tol_main, riem_tol_shock, riem_tol_rarefaction;
  double riem_min_pressure, riem_failure_threshold, riem_pressure_at_failure;
  /* Warm start of the exact Riemann solve (no reference counterpart): the
   * bracket tried around a proposed star pressure p is [p - d|p|, p + d|p|]
   * (default 3e-4: with proposals a few tenths of a percent off, the root is
   * usually bracketed at once or after the search's first expansions, and one
   * secant iteration meets the stopping test). */
  double riem_warm_delta;
  /* MultiPhaseData::riemann_normal: direction of the interface Riemann
   * problem, 0 LEVEL_SET (gradient of phi), 1 MESH (face normal), 2 AVERAGE */
  int mp_riemann_normal;
  /* Warm-start gate (no reference counterpart): a proposal p is ignored, and
   * the acoustic starting points kept, where |log((p + S) / (pac + S))| <=
   * gate, S = min(pinf_l, pinf_r): near-acoustic problems, which the acoustic
   * estimate already starts within the network's own error. 0 (default):
   * every proposal departing by more than riem_warm_delta is used. */
  double riem_warm_gate;
  /* EmbeddedBoundaryMethodData (IoData.h:1340-1360), for faces cut by an
   * embedded surface (m2cg_set_wall_faces): direction of the one-sided
   * Riemann problems, 0 EMBEDDED_SURFACE, 1 MESH (default), 2 AVERAGE; state
   * reconstruction at the surface, 0 CONSTANT (default: cell-centred states)
   * or 1 LINEAR (the limited face states; a face pass writes them). */
  int ebm_riemann_normal;
  int ebm_recon;
  /* EquationsData::dummy_state (VarFcnDummy): the fixed state of inactive
   * cells, those with material ID = nmat (regions enclosed by an embedded
   * surface; contexts without a level set): density, pressure, internal
   * energy per unit mass (defaults 1e-6, 0, 0, IoData.cpp:30-42). */
  double inactive_density, inactive_pressure, inactive_energy;
} m2cg_scheme;

/* One level set (LevelSetSchemeData, IoData.h:653-679; reinit
 * LevelSetReinitializationData, IoData.h:628-651), full domain, with the
 * finite-difference UPWIND_CENTRAL_3 solver (the reference's default) or the
 * finite-volume solver (MUSCL of phi and of the velocity, ROE / LLF / UPWIND
 * flux, phi div(u) source). Enum values are the reference's. */
enum { M2CG_LSBC_NONE = 0, M2CG_LSBC_ZERO_NEUMANN = 1, M2CG_LSBC_LINEAR_EXTRAPOLATION = 2,
       M2CG_LSBC_NON_NEGATIVE = 3 };
enum { M2CG_LS_FINITE_VOLUME = 0, M2CG_LS_FINITE_DIFFERENCE = 1 };
enum { M2CG_LSFLUX_ROE = 0, M2CG_LSFLUX_LLF = 1, M2CG_LSFLUX_UPWIND = 2 };
typedef struct {
  int material_id;        /* material in the phi<0 region */
  int bc[6];
  int reinit_frequency;   /* <=0: never */
  int reinit_maxits;
  double reinit_cfl;
  double reinit_tol;
  int reinit_first_layer; /* firstLayerTreatment: 0 FIXED, 1 CONSTRAINED1 (CR-1), 2 CONSTRAINED2
                             (CR-2), 3 ITERATIVE_CONSTRAINED1 (HCR-1), 4 ITERATIVE_CONSTRAINED2
                             (HCR-2) */
  int solver;             /* M2CG_LS_FINITE_DIFFERENCE (default) or M2CG_LS_FINITE_VOLUME */
  int flux;               /* finite volume: M2CG_LSFLUX_*, default ROE */
  double delta;           /* finite volume: entropy-fix coefficient of the ROE flux (0.2) */
  int rec_type;           /* finite volume ReconstructionData: 0 CONSTANT, 1 LINEAR (default) */
  int limiter;            /* finite volume: 0 NONE (default), 1 GENERALIZED_MINMOD, 2 VANALBADA */
  double minmod_coeff;    /* finite volume: generalized minmod coefficient (1.2) */
} m2cg_levelset;

/* Fill a scheme/material/level-set struct with the reference's defaults
 * (IoData.cpp:860-871, 1049-1058, 1154-1160, 1205-1265, 1345-1357, 1400-1417,
 * 1472-1503). */
void m2cg_default_scheme(m2cg_scheme* s);
void m2cg_default_material(m2cg_material* m);
void m2cg_default_levelset(m2cg_levelset* l);

typedef struct m2cg_ctx m2cg_ctx;

/* Make `device` the current CUDA device of the calling thread for contexts
 * created afterwards (one process per GPU; no reference counterpart). */
m2cg_status m2cg_set_device(int device);

/* Create a context on the current CUDA device. nls = 0 (one material) or 1.
 * Replaces the setup in Main.cpp:106-379 for this path. */
m2cg_status m2cg_create(const m2cg_grid* grid, const m2cg_scheme* scheme,
                        const m2cg_material* mats, int nmat,
                        const m2cg_levelset* ls, int nls, m2cg_ctx** out);
m2cg_status m2cg_destroy(m2cg_ctx* ctx);

/* Host <-> device state in the ghosted host layout above. ID and phi may be
 * NULL (single material). Upload clips density/pressure and fills ghost
 * nodes as SpaceOperator::SetInitialCondition does at its end
 * (SpaceOperator.cpp:1088-1090), then sets ghost IDs from their images
 * (MultiPhaseOperator::UpdateMaterialIDAtGhostNodes, MultiPhaseOperator.cpp:796-819). */
m2cg_status m2cg_upload_state(m2cg_ctx* ctx, const double* V, const double* ID, const double* phi);
m2cg_status m2cg_download_state(m2cg_ctx* ctx, double* V, double* ID, double* phi);

/* dt = cfl * min over cells of dx/(|u|+c)  (SpaceOperator::ComputeTimeStepSize). */
m2cg_status m2cg_compute_dt(m2cg_ctx* ctx, double* dt_out);

/* R = -(1/vol) * sum of face fluxes for the current state, written to R in
 * the ghosted host layout (interior nodes only are meaningful).
 * (SpaceOperator::ComputeResidual, SpaceOperator.cpp:3351-3409.) */
m2cg_status m2cg_compute_residual(m2cg_ctx* ctx, double* R_host);

/* One full time step of size dt at time t_new (the reference passes the
 * updated time), including level-set advance, material-ID update,
 * reinitialisation and the post-step multiphase update
 * (TimeIntegratorRK*::AdvanceOneTimeStep + UpdateSolutionAfterTimeStepping). */
m2cg_status m2cg_advance(m2cg_ctx* ctx, double t_new, double dt, int time_step);

/* Run nsteps steps with dt from the CFL condition each step, stopping at
 * t_max (the last step is shortened as in Main.cpp:537-541). *t is updated. */
m2cg_status m2cg_run(m2cg_ctx* ctx, int nsteps, double t_max, double* t, int* steps_done);

/* Per-run counters, mirroring the reference's warnings and totals. */
typedef struct {
  long long steps;
  long long cells_updated;       /* interior cells x steps */
  long long riemann_calls;       /* interface Riemann problems solved */
  long long riemann_iterations;  /* outer secant iterations, summed */
  long long riemann_errors;      /* as counted at SpaceOperator.cpp:2818 */
  long long clipped_cells;       /* ClipDensityAndPressure counts */
  long long reinit_calls;
  long long kernel_launches;
  long long unresolved_cells;    /* cells that changed material and that neither the star states nor
                                    the extrapolation could update (handed to FixUnresolvedNodes) */
  long long riemann_evaluations; /* star-state evaluations at trial pressures (bracketing + secant) */
  long long failsafe_cells;      /* cells given the material's failsafe density (no valid neighbour
                                    within 10 layers, MultiPhaseOperator.cpp:1352-1369) */
  long long riemann_nontrivial;  /* interface Riemann problems not answered by the trivial branch
                                    (equal normal velocity and pressure, ExactRiemannSolverBase.cpp:129-134) */
  long long wall_riemann_calls;  /* one-sided Riemann problems at faces cut by an embedded surface (their
                                    failures are counted in riemann_errors, as the reference does) */
} m2cg_counters;
m2cg_status m2cg_get_counters(const m2cg_ctx* ctx, m2cg_counters* c);

/* Faces cut by embedded surfaces (walls), for every following stage until
 * replaced; n = 0 removes them. Replaces the embedded-boundary branch of
 * SpaceOperator::ComputeAdvectionFluxes (SpaceOperator.cpp:2438-2484, and the
 * y/z faces at 2568-2612, 2695-2739): on a cut face each side gets its
 * numerical flux against its own one-sided Riemann star state
 * (ExactRiemannSolverBase::ComputeOneSidedRiemannSolution on its cell-centred
 * stage state, the star state clipped), solved on the device each stage.
 * faces [n][4] = (axis d: 0 x, 1 y, 2 z; i, j, k): the face between interior
 * cell (i, j, k) and its low neighbour along d, which must be interior too
 * (index along d >= 1). What the reference's intersector data yields for
 * that face through SpaceOperator::FindEdgeSurfaceIntersections
 * (SpaceOperator.cpp:3435-3501), [n][3] each: nwall_fwd / uwall_fwd, the
 * surface's unit normal and velocity at the intersection nearest the low
 * cell; nwall_bwd / uwall_bwd, those nearest the high cell. The normals are
 * used by scheme->ebm_riemann_normal EMBEDDED_SURFACE and AVERAGE; with
 * scheme->ebm_recon LINEAR the one-sided problems and fluxes take the face
 * states of the linear reconstruction. A cut face that also separates two
 * materials takes the wall branch and stores no interface Riemann solution,
 * as in the reference. Heat diffusion is unaffected by the surface, as in
 * the reference (HeatDiffusionOperator::AddDiffusionFluxes does not use it).
 * Refused (M2CG_ERR_UNSUPPORTED): viscous materials (the viscosity
 * operator's ghost-fluid population at cut faces is not built), faces on
 * the subdomain boundary. Regions enclosed by a surface: upload their
 * cells with material ID nmat (the reference's INACTIVE_MATERIAL_ID; one
 * material, no level set, no diffusion); they keep the scheme's inactive
 * state, take no slope from or flux across their side, and do not limit
 * the time step. Host pointers. */
m2cg_status m2cg_set_wall_faces(m2cg_ctx* ctx, int n, const int* faces, const double* nwall_fwd,
                                const double* uwall_fwd, const double* nwall_bwd, const double* uwall_bwd);

/* MultiPhaseOperator::UpdateStateVariablesAfterInterfaceMotion
 * (MultiPhaseOperator.cpp:823-1400) on the context's resident state: every
 * interior cell whose ID (the context's, as uploaded or advanced) differs from
 * IDn (host, ghosted layout of m2cg_upload_state) gets its state from the
 * stage-1 star states of its interface faces (phasechange_type
 * RIEMANN_SOLUTION) or from its neighbours (EXTRAPOLATION), then
 * FixUnresolvedNodes, then ClipDensityAndPressure. use_stored_riemann_solutions
 * = 1 uses the star states stored by the last m2cg_advance (IDn must then be
 * the IDs at the start of that step; M2CG_ERR_ARG if no step ran since the
 * last upload); 0 passes none, as an empty RiemannSolutions does. m2cg_advance
 * calls the same update at the end of every step. *unresolved (may be NULL)
 * receives the cells handed to FixUnresolvedNodes. With
 * apply_failsafe_density Off, a background cell with no valid neighbour
 * within 10 layers would need the level-set correction of
 * TimeIntegrator.cpp:742-761, which is not built: M2CG_ERR_UNSUPPORTED. */
m2cg_status m2cg_update_states_after_interface_motion(m2cg_ctx* ctx, const double* IDn,
                                                      int use_stored_riemann_solutions, int* unresolved);

/* Run nsteps CFL-limited steps with the state resident in device memory and
 * report their device time (CUDA events on the context's stream) and the
 * number of kernels launched. Used by the benchmark; no reference counterpart
 * (the reference times with clock(), Main.cpp:559). */
m2cg_status m2cg_time_steps(m2cg_ctx* ctx, int nsteps, float* ms, long long* launches);

/* Device time of the fused stage kernel alone over nsteps CFL steps (CUDA
 * events around each stage launch): summed milliseconds, number of stage
 * launches, and the whole-step milliseconds. Benchmark support; no
 * reference counterpart. */
m2cg_status m2cg_profile_stages(m2cg_ctx* ctx, int nsteps, float* stage_ms, int* stage_launches,
                                float* step_ms);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work after the library's. */
m2cg_status m2cg_get_stream(const m2cg_ctx* ctx, void** stream);

/* Probes (ProbeOutput::SetupInterpolation / InterpolateSolutionAtProbe,
 * ProbeOutput.cpp:219-340, 636-673): the primitive state at n fixed points
 * xyz [n][3], interpolated trilinearly from the cell centres and the ghost
 * layer the boundary rule fills, exactly as the reference does (invalid edge
 * ghosts replaced by the average of the valid corners). m2cg_run and
 * m2cg_advance sample them on the device after every `every`-th step
 * (0: only on m2cg_sample_probes) into a device buffer of `capacity`
 * records, with no host round trip; a record is t, the step count, then
 * rho, u, v, w, p of each probe (2 + 5n doubles). A probe outside the
 * ghosted mesh is M2CG_ERR_ARG, as the reference aborts. The device record
 * buffer and the sampling schedule have no reference counterpart (the
 * reference writes a text line per sample). */
m2cg_status m2cg_set_probes(m2cg_ctx* ctx, int n, const double* xyz, int every, int capacity);
m2cg_status m2cg_sample_probes(m2cg_ctx* ctx);
/* Copy the records taken since the last read into `records` (room for the
 * capacity given to m2cg_set_probes; NULL drops them), their number into
 * *nrec, and empty the buffer. */
m2cg_status m2cg_read_probes(m2cg_ctx* ctx, double* records, int* nrec);

/* Text of the last error on this thread (never NULL). */
const char* m2cg_last_error(void);

/* ---------------------------------------------------------------------------
 * Batched interface Riemann problems (ExactRiemannSolverBase::ComputeRiemannSolution,
 * ExactRiemannSolverBase.cpp:59-342), FP64, one problem per thread.
 * Inputs per problem: VL[5], VR[5] primitive states, idl/idr material ids,
 * dir[3] unit normal. Outputs: Vs[5] state at xi=0, id, Vsm[5], Vsp[5]
 * star states, iterations (outer secant iterations, both solver variants),
 * err: 0 OK; bit 1 not solved (where the adaptive solve cannot bracket or
 * converge, the non-adaptive variant of ExactRiemannSolverBase.cpp:2199-2945
 * solves again, as the reference does, and bit 1 means it failed too; the
 * outputs then hold the reference's best-effort answer); bit 2 the
 * integration-path scratch ran out; bit 4 a state the reference aborts on.
 * Host pointers; the call copies in and out.
 * warm (optional, may be NULL): an initial star-pressure guess per problem;
 * NaN entries mean "no guess".
 * ------------------------------------------------------------------------- */
m2cg_status m2cg_riemann_batch(const m2cg_scheme* scheme, const m2cg_material* mats, int nmat,
                               int n, const double* VL, const int* idl, const double* VR,
                               const int* idr, const double* dir, const double* warm,
                               double* Vs, int* id, double* Vsm, double* Vsp, int* iters, int* err);

/* The same solve where every problem carries its own material pair:
 * problem q has material mats[2q] on the left and mats[2q+1] on the right;
 * id[q] is 0 (left material) or 1 (right); evals (optional) counts the
 * star-state evaluations at trial pressures. Host pointers. */
m2cg_status m2cg_riemann_batch_pairs(const m2cg_scheme* scheme, const m2cg_material* mats, int n,
                                     const double* VL, const double* VR, const double* dir,
                                     const double* warm, double* Vs, int* id, double* Vsm,
                                     double* Vsp, int* iters, int* evals, int* err);

/* One-sided (wall) Riemann problems: the fluid state Vm[q] (material
 * idm[q]) against a wall moving with velocity uwall[q] (3 components), dir[q]
 * the unit normal pointing from the fluid towards the wall. Replaces
 * ExactRiemannSolverBase::ComputeOneSidedRiemannSolution
 * (ExactRiemannSolverBase.cpp:1931-2195), which the embedded-boundary branch
 * of SpaceOperator::ComputeAdvectionFluxes calls on each side of a face the
 * surface cuts (SpaceOperator.cpp:2438-2484). Outputs per problem: Vs, the
 * state at the wall (xi = 0; zeros where id = -1, i.e. where the wall
 * recedes from the fluid), id (idm[q] or -1), Vsm, the fluid's star state
 * (normal velocity = the wall's), iters (optional; secant iterations of a
 * shock), err: 0, or 1 where the reference reports a failure (it then
 * returns the input state with the wall's normal velocity, or its best
 * bracket point), | 2 integration-path capacity exhausted, | 4 a state the
 * reference aborts on. Host pointers. */
m2cg_status m2cg_riemann_wall_batch(const m2cg_scheme* scheme, const m2cg_material* mats, int nmat, int n,
                                    const double* Vm, const int* idm, const double* uwall,
                                    const double* dir, double* Vs, int* id, double* Vsm, int* iters,
                                    int* err);

/* The same batched Riemann solve for callers that cannot allocate device
 * memory: a host application whose memory pool owns the whole GPU, or a
 * runtime that forbids allocation on the path that calls it. No counterpart
 * in the reference.
 *  - All array arguments are DEVICE pointers the caller owns; the call makes
 *    no allocation (no cudaMalloc or cudaFree, no allocating library call).
 *  - The solver's integration-path scratch is a file-scope device array of
 *    M2CG_NOALLOC_MAX_PROBLEMS slots of 24 KiB (24 MiB), held by every device
 *    that loads the library until the process exits. n beyond
 *    M2CG_NOALLOC_MAX_PROBLEMS is rejected with M2CG_ERR_ARG and a message.
 *  - Each call outside a stream capture looks up that array's device address
 *    with the current device (so a device reset cannot leave a stale one);
 *    a call made while `stream` is captured reuses the address of the last
 *    uncaptured call on that device, so make one call (n = 0 is enough)
 *    before any capture. Under lazy module loading (the CUDA default) that
 *    first call is also when the driver places the 24 MiB array on the
 *    device: a caller whose memory pool will take the whole device makes it
 *    before the pool reserves its memory.
 *  - The work is queued on `stream` (a cudaStream_t, NULL = legacy default
 *    stream); the call returns without waiting. All calls share the scratch
 *    array, so calls that overlap on the GPU (different streams, devices
 *    excepted) race; order them on one stream.
 *  - err gains M2CG_RIEMANN_ERR_MATERIAL_ID where idl/idr is outside
 *    [0, nmat) (outputs of that problem are NaN, id -1). */
#define M2CG_NOALLOC_MAX_PROBLEMS 1024
#define M2CG_RIEMANN_ERR_MATERIAL_ID 8
m2cg_status m2cg_riemann_batch_noalloc(const m2cg_scheme* scheme, const m2cg_material* mats, int nmat,
                                       int n, const double* VL, const int* idl, const double* VR,
                                       const int* idr, const double* dir, const double* warm,
                                       double* Vs, int* id, double* Vsm, double* Vsp, int* iters,
                                       int* err, void* stream);

/* ---------------------------------------------------------------------------
 * Learned warm start for the interface Riemann solve (no counterpart in the
 * reference). A 16 -> 64 -> 64 -> 64 -> 1 tanh MLP maps dimensionless
 * features of a problem to log((pstar + S) / B), S = min(pinf_l, pinf_r) and
 * B = max(pac + S, 1e-3 (max(|pl|, |pr|) + S)), pac the acoustic estimate the
 * solver's bracket search starts from; where the proposal p departs from pac
 * by more than riem_warm_delta (and passes riem_warm_gate),
 * p -+ riem_warm_delta |p| replaces the acoustic starting points of that
 * search. The solver's own iteration and stopping test are
 * unchanged, so results agree with the cold solve within tol_main.
 * Training runs on the GPU (FP32 forward + backward kernels, Adam);
 * inference runs BF16 on tensor cores with FP32 accumulation.
 * ------------------------------------------------------------------------- */
#define M2CG_MLP_INPUTS 16
#define M2CG_MLP_NPARAMS 9473  /* W1[64][16] b1[64] W2[64][64] b2 W3[64][64] b3 w4[64] b4 */
#define M2CG_MLP_NNORM 34      /* xmean[16] xstd[16] ymean ystd */
typedef struct m2cg_mlp m2cg_mlp;
m2cg_status m2cg_mlp_create(unsigned long long seed, m2cg_mlp** out);
m2cg_status m2cg_mlp_destroy(m2cg_mlp* m);
m2cg_status m2cg_mlp_get_params(const m2cg_mlp* m, float* params, float* norm);
m2cg_status m2cg_mlp_set_params(m2cg_mlp* m, const float* params, const float* norm);
/* Mean-squared-error loss and its gradient with respect to the parameters
 * for n network inputs Xn [n][16] and targets yn, both already normalised
 * (host arrays); no update. */
m2cg_status m2cg_mlp_loss_grad(m2cg_mlp* m, const float* Xn, const float* yn, int n, float* loss,
                               float* grad);
/* Train on raw features X [n][16] and targets y = log(pstar / pac): the
 * normalisation is set from the data, then `steps` Adam steps of `batch`
 * samples (cosine-decayed learning rate from lr). final_loss: mean loss of
 * the last 5% of steps, in normalised units. */
m2cg_status m2cg_mlp_train(m2cg_mlp* m, const float* X, const float* y, int n, int steps, int batch,
                           float lr, unsigned long long seed, float* final_loss);
/* Features of problems with per-pair materials (as m2cg_riemann_batch_pairs):
 * X [n][16], scale [n][2] = (base B, shift S) of the target log((p* + S) / B),
 * valid [n] (0 where no proposal can be made). */
m2cg_status m2cg_mlp_features_pairs(const m2cg_material* mats, int n, const double* VL,
                                    const double* VR, const double* dir, float* X, double* scale, int* valid);
/* Network output (target units) for raw feature rows, BF16 tensor cores. */
m2cg_status m2cg_mlp_infer(m2cg_mlp* m, const float* X, const int* valid, int n, float* y);
/* Proposed star pressures for per-pair problems (NaN where none). */
m2cg_status m2cg_mlp_predict_pairs(m2cg_mlp* m, const m2cg_material* mats, int n, const double* VL,
                                   const double* VR, const double* dir, double* p);

/* ---------------------------------------------------------------------------
 * Batched 1D two-material shock tubes of uneven lengths, all advanced in one
 * persistent launch per RK stage, captured in a CUDA graph.
 * ------------------------------------------------------------------------- */
typedef struct m2cg_batch m2cg_batch;
typedef struct {
  int cells_per_block;   /* cells handled by one CTA per work item; 0 = autotune */
  int threads_per_block; /* 0 = autotune */
  int use_graph;         /* launch mode: 0 kernels per phase, launched one by one; 1 the same
                            captured in CUDA graphs and replayed; 2 one persistent launch per
                            run, each CTA advancing whole tubes through all their steps (tubes
                            are independent, so no CTA waits on another); -1 measure 1 and 2
                            and take the faster */
} m2cg_batch_tuning;

/* ntubes tubes; tube t has len[t] cells on [0, 1] (cell width 1/len[t]),
 * material mats[2t] on the left half and mats[2t+1] on the right half, left
 * and right primitive states VL[5t..], VR[5t..], interface at x = 0.5 as the
 * zero of phi = 0.5 - x. Boundary ghosts are OUTLET-type Dirichlet copies of
 * the initial end states. */
m2cg_status m2cg_batch_create(const m2cg_scheme* scheme, int ntubes, const int* len,
                              const m2cg_material* mats, const double* VL, const double* VR,
                              const m2cg_batch_tuning* tuning, m2cg_batch** out);
/* Advance every tube by nsteps steps with a per-tube CFL dt. */
m2cg_status m2cg_batch_run(m2cg_batch* b, int nsteps);
/* Download tube states: V (5 doubles per cell, tubes concatenated), ID per
 * cell, time per tube. After a tube reported an error the arrays are still
 * written (the other tubes' states are valid) and the status names the
 * error. */
m2cg_status m2cg_batch_download(m2cg_batch* b, double* V, int* ID, double* t_per_tube);
/* The tuning in use (the autotuner's choice where the caller passed 0). */
m2cg_status m2cg_batch_get_tuning(const m2cg_batch* b, m2cg_batch_tuning* t);
/* Counters over all tubes: steps, cell updates, interface Riemann calls,
 * iterations and errors (as counted at SpaceOperator.cpp:2818), unresolved
 * cells of the post-step update, kernel launches. */
m2cg_status m2cg_batch_get_counters(m2cg_batch* b, m2cg_counters* c);
/* First device error code of each tube (0 = none), ntubes entries. A tube
 * that reported an error is not advanced further (the reference aborts the
 * run there); its downloaded state and time are those of the step where it
 * failed, left part-way, and are not defined. The other tubes go on. */
m2cg_status m2cg_batch_tube_errors(m2cg_batch* b, int* codes);
/* Advance nsteps and return the device time of those steps (CUDA events on
 * the batch's stream). *ms is written even when a tube reported an error
 * (the status then says which error; m2cg_batch_tube_errors says where). */
m2cg_status m2cg_batch_time_steps(m2cg_batch* b, int nsteps, float* ms);
/* Attach a trained network (NULL detaches): every interface Riemann solve
 * of the batch then starts from its proposal. The network must outlive the
 * batch's use of it. */
m2cg_status m2cg_batch_set_mlp(m2cg_batch* b, const m2cg_mlp* m);
/* Attach a trained network (NULL detaches) to a two-material context: every
 * interface Riemann problem of its steps starts from the network's proposal
 * (features of the stage states the solve uses; BF16 inference on the
 * device, no host round trip). No reference counterpart. The network must
 * outlive the context's use of it; the first attachment allocates per-face
 * buffers (about 90 bytes per interface-face slot). */
m2cg_status m2cg_set_mlp(m2cg_ctx* ctx, const m2cg_mlp* m);
m2cg_status m2cg_batch_destroy(m2cg_batch* b);

#ifdef __cplusplus
}
#endif
#endif
