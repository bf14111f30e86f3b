// Host side of the C ABI declared in include/m2c_gpu.h: context set-up
// (mesh, limiter coefficients, EOS tables, device buffers), state transfer
// between the reference's ghosted AoS host layout and the device SoA layout,
// the device clock (dt from the CFL reduction, last step shortened to t_max),
// and the RK step driver.
//
// Compiled with -fmad=false (the small kernels here feed the FP64 path).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/m2c_gpu.h"
#include "launch.h"
#include "multiphase.h"
#include "viscous.h"
#include "walls.h"

using namespace m2c;

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error = "";

static m2cg_status fail(m2cg_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return st;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t _e = (call);                                                                  \
    if (_e != cudaSuccess)                                                                    \
      return fail(M2CG_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
  } while (0)

extern "C" const char* m2cg_last_error(void) { return g_last_error.c_str(); }

namespace m2c {
// Sets the text m2cg_last_error() returns, for entry points in other files.
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace m2c

// ---------------------------------------------------------------------------
// Defaults: IoData constructors of the reference.
// ---------------------------------------------------------------------------
extern "C" void m2cg_default_scheme(m2cg_scheme* s) {
  memset(s, 0, sizeof *s);
  s->flux = M2CG_FLUX_HLLC;            // SchemeData::SchemeData (IoData.cpp:1154-1160)
  s->roe_delta = 0.2;
  s->rec_type = M2CG_REC_LINEAR;       // ReconstructionData (IoData.cpp:1049-1058)
  s->limiter = M2CG_LIM_NONE;
  s->minmod_coeff = 1.2;
  s->slope_near_interface = 1;
  s->rec_var = M2CG_RECVAR_PRIMITIVE;
  s->rk_order = 2;                     // TsData / ExplicitData (IoData.cpp:1472-1503)
  s->cfl = 0.5;
  s->precision = M2CG_PREC_FP64;
  s->mp_flux = M2CG_MPFLUX_NUMERICAL;  // MultiPhaseData (IoData.cpp:1400-1417)
  s->mp_recon = 0;
  s->mp_phasechange_type = 0;
  s->mp_phasechange_dir = 1;
  s->mp_apply_failsafe_density = 1;
  s->riem_maxits_main = 200;           // ExactRiemannSolverData (IoData.cpp:1345-1357)
  s->riem_maxits_bracket = 100;
  s->riem_maxits_shock = 200;
  s->riem_nsteps_rarefaction = 200;
  s->riem_tol_main = 1.0e-4;
  s->riem_tol_shock = 1.0e-12;
  s->riem_tol_rarefaction = 1.0e-8;
  s->riem_min_pressure = -1.0e8;
  s->riem_failure_threshold = 0.2;
  s->riem_pressure_at_failure = 1.0e-8;
  s->riem_warm_gate = 0.0;
  s->riem_warm_delta = 3.0e-4;  // measured: the narrowest bracket that keeps the evaluations low
  s->mp_riemann_normal = 1;  // MultiPhaseData::MESH (IoData.cpp:1408)
  s->ebm_riemann_normal = 1; // EmbeddedBoundaryMethodData::MESH (IoData.cpp:2937-2938)
  s->ebm_recon = 0;          // CONSTANT
  s->inactive_density = 1.0e-6;  // StateVariable::StateVariable (IoData.cpp:30-42)
  s->inactive_pressure = 0.0;
  s->inactive_energy = 0.0;
}

extern "C" void m2cg_default_material(m2cg_material* m) {
  memset(m, 0, sizeof *m);             // MaterialModelData (IoData.cpp:860-871)
  m->eos = M2CG_EOS_SG;
  m->gamma = 1.4;
  m->rhomin = 0.0;
  m->pmin = -DBL_MAX;
  m->rhomax = DBL_MAX;
  m->pmax = DBL_MAX;
  m->failsafe_density = 1.0e-10;
}

extern "C" void m2cg_default_levelset(m2cg_levelset* l) {
  memset(l, 0, sizeof *l);             // LevelSetSchemeData (IoData.cpp:1245-1265)
  l->material_id = 1;
  for (int q = 0; q < 6; q++) l->bc[q] = M2CG_LSBC_ZERO_NEUMANN;
  l->reinit_frequency = -1;            // LevelSetReinitializationData (IoData.cpp:1205-1213)
  l->reinit_maxits = 30;
  l->reinit_cfl = 0.8;
  l->reinit_tol = 2.0e-4;
  l->reinit_first_layer = 0;
  l->solver = M2CG_LS_FINITE_DIFFERENCE;
  l->flux = M2CG_LSFLUX_ROE;
  l->delta = 0.2;
  l->rec_type = 1;                     // ReconstructionData (IoData.cpp:1049-1058)
  l->limiter = 0;
  l->minmod_coeff = 1.2;
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct m2cg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  m2cg_scheme scheme;
  std::vector<m2cg_material> mats;
  Grid3 g;
  SchemeK sk;
  int nx = 0, ny = 0, nz = 0;
  long long px = 0, plane = 0, nalloc = 0;
  // SoA state: V double-buffered (step state), U two stage buffers
  double* V[2][5] = {};
  double* U[2][5] = {};
  // stage inputs in the compute type: P two stage buffers (clip(C2P(U_s))),
  // and for the mixed path an FP32 copy of V (Vf, double-buffered with V)
  void* P[2][5] = {};
  float* Vf[2][5] = {};
  // Each five-component buffer is one allocation (component c at c * cstride
  // elements), so that one 4D tensor map covers all five arrays: the stage
  // kernel stages a plane of all components with one tensor copy.
  long long cstride = 0;
  void* blk[4][2] = {};      // allocations of V, U, P, Vf (per buffer b)
  // tensor maps of the stage inputs: [0..1] the step state in the compute
  // type (Vf[b] mixed, V[b] FP64), [2..3] P[b]
  CUtensorMap tmap[4];
  bool tma_ok = false;       // maps built (else the kernel copies values one by one)
  int cur = 0;
  uint8_t* id = nullptr;
  // mesh
  double *dx = nullptr, *dy = nullptr, *dz = nullptr;
  double* lA[3] = {};
  double* lB[3] = {};
  int* lK[3] = {};
  double* lC[3] = {};
  int ntx = 1, nty = 1, nitems = 1;
  std::vector<double> hdx, hdy, hdz, hxc, hyc, hzc;
  // device scratch: clock [t, dt, tmax, cfl], dtmin bits, flags, error
  double* clock = nullptr;
  unsigned long long* dtmin = nullptr;
  int* clipflags = nullptr;  // [4]
  DevError* err = nullptr;
  // staging buffers for host transfers (ghosted AoS)
  double* stage_buf = nullptr;
  size_t stage_bytes = 0;
  bool dtmin_valid = false;
  bool rs_valid = false;  // the multiphase star states stored by the last step match the resident state
  m2cg_counters counters = {};
  Multiphase* mp = nullptr;  // two-material machinery (nullptr for one material)
  Viscous* visc = nullptr;   // viscous fluxes (nullptr when every material is inviscid)
  Walls* walls = nullptr;    // faces cut by embedded surfaces (nullptr: none)
  // probes (ProbeOutput): per probe the lower node (i, j, k), the trilinear
  // coordinates and the valid-corner mask; records sampled on the device
  int nprobe = 0, probe_every = 0, probe_cap = 0, probe_count = 0;
  int* probe_ijk = nullptr;        // [n][4]: i, j, k, valid mask
  double* probe_xi = nullptr;      // [n][3]
  double* probe_rec = nullptr;     // [cap][2 + 5n]: t, step, V of each probe
    // optional per-stage event timing (benchmark roofline)
  bool profile = false;
  std::vector<cudaEvent_t> ev;  // pairs (before, after) per stage launch
};

// Tensor maps (cuTensorMapEncodeTiled, reached through the runtime's
// driver entry point, so the library links only the CUDA runtime) of the
// stage kernel's plane input: 4D (x, y, z, component) over one
// five-component buffer, box = one plane of a tile with its halo,
// STAGE_TMA_BX x (TY + 4) x 1 x 5 elements. Out-of-range x/y cells read as
// zero; the kernel rebuilds them by the boundary rule.
static m2cg_status encode_stage_map(m2cg_ctx* c, CUtensorMap* m, const void* base, bool f32, int ty) {
  static PFN_cuTensorMapEncodeTiled encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return fail(M2CG_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
    encode = (PFN_cuTensorMapEncodeTiled)fn;
  }
  const size_t es = f32 ? 4 : 8;
  cuuint64_t dims[4] = {(cuuint64_t)c->nx, (cuuint64_t)c->ny, (cuuint64_t)c->nz, 5};
  cuuint64_t strides[3] = {(cuuint64_t)(c->px * es), (cuuint64_t)(c->plane * es), (cuuint64_t)(c->cstride * es)};
  cuuint32_t box[4] = {(cuuint32_t)STAGE_TMA_BX, (cuuint32_t)(ty + 4), 1, 5};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = encode(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                      const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(M2CG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return M2CG_OK;
}

// A map that cannot be encoded leaves tma_ok false: the stage kernel then
// copies plane values one by one.
static m2cg_status make_stage_tensor_maps(m2cg_ctx* c) {
  const bool mixed = c->scheme.precision == M2CG_PREC_MIXED;
  const int ty = mixed ? StageTY<float, false>::value : StageTY<double, false>::value;
  for (int b = 0; b < 2; b++) {
    m2cg_status st = encode_stage_map(c, &c->tmap[b], mixed ? c->blk[3][b] : c->blk[0][b], mixed, ty);
    if (!st) st = encode_stage_map(c, &c->tmap[2 + b], c->blk[2][b], mixed, ty);
    if (st) return st;  // the stage kernel then copies plane values one by one
  }
  c->tma_ok = true;
  return M2CG_OK;
}

static double* dalloc(size_t n, m2cg_status* st) {
  void* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) {
    *st = fail(M2CG_ERR_NOMEM, "cudaMalloc of %zu doubles failed", n);
    return nullptr;
  }
  return (double*)p;
}

// Cell centres and widths per axis: uniform as MeshGenerator::ComputeMesh1DUniform
// (MeshGenerator.cpp:146-158: x_i = x0 + h/2 + i h) unless given.
static void axis_mesh(int n, double a, double b, const double* wc, const double* w, std::vector<double>& xc,
                      std::vector<double>& dx) {
  dx.assign(n, 0.0);
  xc.assign(n, 0.0);
  double h = (b - a) / n;
  for (int i = 0; i < n; i++) {
    dx[i] = w ? w[i] : h;
    xc[i] = wc ? wc[i] : a + 0.5 * h + i * h;
  }
}

// Limiter coefficients per axis index (Reconstructor::Setup, Reconstructor.cpp:53-99,
// CalculateSlopeLimiterCoefficientK, 103-121). Ghost widths equal the
// adjacent interior width (SpaceOperator::PopulateGhostBoundaryCoordinates,
// SpaceOperator.cpp:218-300); periodic axes wrap.
static bool axis_limiter(const std::vector<double>& dx, bool periodic, int limiter, std::vector<double>& A,
                         std::vector<double>& B, std::vector<int>& K) {
  int n = (int)dx.size();
  A.resize(n);
  B.resize(n);
  K.resize(n);
  for (int i = 0; i < n; i++) {
    double dm = i > 0 ? dx[i - 1] : (periodic ? dx[n - 1] : dx[0]);
    double dp = i < n - 1 ? dx[i + 1] : (periodic ? dx[0] : dx[n - 1]);
    A[i] = (dm + dx[i]) / (dx[i] + dp);
    B[i] = 2.0 * dx[i] / (dx[i] + dp);
    K[i] = 0;
    if (limiter == M2CG_LIM_VANALBADA) {
      int k;
      for (k = 2; k < 1000; k++) {
        double rhs = 2.0 / (1.0 + m2c::cr_pow_int((k - 1.0) / k, k - 1) / k) * std::min(A[i], 1.0);
        if (B[i] <= rhs) break;
      }
      if (k >= 999) return false;
      K[i] = k;
    }
  }
  return true;
}

template <typename T>
static void upload_vec(T** d, const std::vector<T>& h, cudaStream_t s, m2cg_status* st) {
  if (cudaMalloc((void**)d, h.size() * sizeof(T)) != cudaSuccess) {
    *st = fail(M2CG_ERR_NOMEM, "cudaMalloc failed");
    return;
  }
  cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

static m2cg_status check_scheme(const m2cg_scheme* s, const m2cg_material* mats, int nmat) {
  if (nmat < 1 || nmat > MAXMAT) return fail(M2CG_ERR_ARG, "nmat must be in [1,%d]", MAXMAT);
  if (s->flux < 0 || s->flux > 2) return fail(M2CG_ERR_UNSUPPORTED, "flux %d not supported (ROE/LLF/HLLC)", s->flux);
  if (s->rec_var < M2CG_RECVAR_PRIMITIVE || s->rec_var > M2CG_RECVAR_CONS_CHAR)
    return fail(M2CG_ERR_ARG, "unknown reconstruction variable type %d", s->rec_var);
  if (s->rk_order < 1 || s->rk_order > 3) return fail(M2CG_ERR_ARG, "rk_order must be 1, 2 or 3");
  // SpaceOperator.cpp:78-83: the LLF interface flux stores no star states
  if (nmat > 1 && s->mp_flux == M2CG_MPFLUX_LLF && s->mp_phasechange_type == 0)
    return fail(M2CG_ERR_ARG, "MultiPhase::Flux = LocalLaxFriedrichs is incompatible with PhaseChange = "
                              "RiemannSolution");
  for (int m = 0; m < nmat; m++)
    if (mats[m].eos != M2CG_EOS_SG && mats[m].eos != M2CG_EOS_NASG)
      return fail(M2CG_ERR_UNSUPPORTED, "material %d: only stiffened gas and NASG are supported", m);
  return M2CG_OK;
}

static MatParams to_params(const m2cg_material& m) {
  MatParams p;
  p.kind = m.eos;
  p.gam = m.gamma;
  p.pc = m.p_c;
  p.b = m.b;
  p.q = m.q;
  p.rhomin = m.rhomin;
  p.pmin = m.pmin;
  p.rhomax = m.rhomax;
  p.pmax = m.pmax;
  p.failsafe_density = m.failsafe_density;
  return p;
}

static void set_stage_items(m2cg_ctx* c, bool multi);

extern "C" m2cg_status m2cg_create(const m2cg_grid* grid, const m2cg_scheme* scheme, const m2cg_material* mats,
                                   int nmat, const m2cg_levelset* ls, int nls, m2cg_ctx** out) {
  if (!grid || !scheme || !mats || !out) return fail(M2CG_ERR_ARG, "null argument");
  *out = nullptr;
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1) return fail(M2CG_ERR_ARG, "grid sizes must be positive");
  if (nls < 0 || nls > 1) return fail(M2CG_ERR_UNSUPPORTED, "at most one level set is supported");
  for (int q = 0; q < 6; q++) {
    int b = grid->bc[q];
    if (b != M2CG_BC_INLET && b != M2CG_BC_OUTLET && b != M2CG_BC_SLIPWALL && b != M2CG_BC_STICKWALL &&
        b != M2CG_BC_SYMMETRY && b != M2CG_BC_PERIODIC)
      return fail(M2CG_ERR_UNSUPPORTED, "boundary %d: type %d not supported", q, b);
  }
  for (int a = 0; a < 3; a++)
    if ((grid->bc[2 * a] == M2CG_BC_PERIODIC) != (grid->bc[2 * a + 1] == M2CG_BC_PERIODIC))
      return fail(M2CG_ERR_ARG, "periodic boundaries must be set on both sides of an axis");
  m2cg_status st = check_scheme(scheme, mats, nmat);
  if (st) return st;
  if (nls == 1 && nmat != 2) return fail(M2CG_ERR_UNSUPPORTED, "a level set needs exactly two materials");

  m2cg_ctx* c = new m2cg_ctx;
  cudaGetDevice(&c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(M2CG_ERR_CUDA, "cudaStreamCreate failed (no CUDA device?)");
  }
  c->scheme = *scheme;
  c->mats.assign(mats, mats + nmat);
  c->nx = grid->nx;
  c->ny = grid->ny;
  c->nz = grid->nz;
  c->px = (grid->nx + 15) / 16 * 16;
  c->plane = c->px * grid->ny;
  c->nalloc = c->plane * grid->nz;
  st = M2CG_OK;
  const bool mixed = scheme->precision == M2CG_PREC_MIXED;
  c->cstride = (c->nalloc + 63) / 64 * 64;
  const long long cs = c->cstride;
  for (int b = 0; b < 2; b++) {
    double* v = dalloc(5 * cs, &st);
    double* u = dalloc(5 * cs, &st);
    void* pb = mixed ? (void*)dalloc(5 * cs / 2, &st) : (void*)dalloc(5 * cs, &st);
    float* vf = mixed ? (float*)dalloc(5 * cs / 2, &st) : nullptr;
    c->blk[0][b] = v;
    c->blk[1][b] = u;
    c->blk[2][b] = pb;
    c->blk[3][b] = vf;
    for (int p = 0; p < 5; p++) {
      c->V[b][p] = v ? v + p * cs : nullptr;
      c->U[b][p] = u ? u + p * cs : nullptr;
      if (mixed) {
        c->P[b][p] = pb ? (void*)((float*)pb + p * cs) : nullptr;
        c->Vf[b][p] = vf ? vf + p * cs : nullptr;
      } else {
        c->P[b][p] = pb ? (void*)((double*)pb + p * cs) : nullptr;
      }
    }
  }
  if (!st) make_stage_tensor_maps(c);
  if (cudaMalloc((void**)&c->id, c->nalloc) != cudaSuccess) st = fail(M2CG_ERR_NOMEM, "cudaMalloc id failed");
  if (!st) cudaMemsetAsync(c->id, 0, c->nalloc, c->stream);
  axis_mesh(grid->nx, grid->x0, grid->xmax, grid->xc, grid->dx, c->hxc, c->hdx);
  axis_mesh(grid->ny, grid->y0, grid->ymax, grid->yc, grid->dy, c->hyc, c->hdy);
  axis_mesh(grid->nz, grid->z0, grid->zmax, grid->zc, grid->dz, c->hzc, c->hdz);
  upload_vec(&c->dx, c->hdx, c->stream, &st);
  upload_vec(&c->dy, c->hdy, c->stream, &st);
  upload_vec(&c->dz, c->hdz, c->stream, &st);
  const std::vector<double>* ax[3] = {&c->hdx, &c->hdy, &c->hdz};
  for (int a = 0; a < 3; a++) {
    std::vector<double> A, B;
    std::vector<int> K;
    if (!axis_limiter(*ax[a], grid->bc[2 * a] == M2CG_BC_PERIODIC, scheme->limiter, A, B, K)) {
      st = fail(M2CG_ERR_ARG, "cannot set up the van Albada exponent on axis %d", a);
      break;
    }
    std::vector<double> Cm(A.size());
    for (size_t q = 0; q < A.size(); q++) Cm[q] = B[q] / (A[q] + 1.0);  // Reconstructor.h:97
    bool uni = true;
    for (size_t q = 1; q < A.size(); q++)
      uni = uni && A[q] == A[0] && B[q] == B[0] && K[q] == K[0] && Cm[q] == Cm[0];
    c->g.lu[a] = uni && !A.empty() ? 1 : 0;
    if (!A.empty()) {
      c->g.lA0[a] = A[0]; c->g.lB0[a] = B[0]; c->g.lK0[a] = K[0]; c->g.lC0[a] = Cm[0];
    }
    upload_vec(&c->lA[a], A, c->stream, &st);
    upload_vec(&c->lB[a], B, c->stream, &st);
    upload_vec(&c->lK[a], K, c->stream, &st);
    upload_vec(&c->lC[a], Cm, c->stream, &st);
  }
  if (cudaMalloc((void**)&c->clock, 8 * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&c->dtmin, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc((void**)&c->clipflags, 4 * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&c->err, sizeof(DevError)) != cudaSuccess)
    st = fail(M2CG_ERR_NOMEM, "cudaMalloc of scalars failed");
  if (!st) {
    cudaMemsetAsync(c->clock, 0, 8 * sizeof(double), c->stream);
    cudaMemsetAsync(c->clipflags, 0, 4 * sizeof(int), c->stream);
    cudaMemsetAsync(c->err, 0, sizeof(DevError), c->stream);
  }
  // kernel parameter blocks
  Grid3& g = c->g;
  g.nx = c->nx; g.ny = c->ny; g.nz = c->nz;
  g.px = c->px; g.plane = c->plane;
  for (int q = 0; q < 6; q++) g.bc[q] = grid->bc[q];
  for (int p = 0; p < 5; p++) { g.inlet[p] = grid->inlet[p]; g.outlet[p] = grid->outlet[p]; }
  g.dx = c->dx; g.dy = c->dy; g.dz = c->dz;
  for (int a = 0; a < 3; a++) { g.lA[a] = c->lA[a]; g.lB[a] = c->lB[a]; g.lK[a] = c->lK[a]; g.lC[a] = c->lC[a]; }
  SchemeK& sk = c->sk;
  sk.flux = scheme->flux;
  sk.limiter = scheme->limiter;
  sk.rec_linear = scheme->rec_type == M2CG_REC_LINEAR;
  sk.slope_zero_at_interface = scheme->slope_near_interface == 0;
  sk.rec_var = scheme->rec_var;
  sk.alpha = scheme->minmod_coeff;
  sk.delta = scheme->roe_delta;
  sk.nmat = nmat;
  sk.dummy[0] = scheme->inactive_density;  // EquationsData::dummy_state (VarFcnDummy)
  sk.dummy[1] = scheme->inactive_pressure;
  sk.dummy[2] = scheme->inactive_energy;
  for (int m = 0; m < MAXMAT; m++) {
    MatParams p = to_params(mats[m < nmat ? m : 0]);
    sk.ed[m] = make_eos<double>(p);
    sk.ef[m] = make_eos<float>(p);
  }
  size_t smem = scheme->precision == M2CG_PREC_MIXED ? stage_smem_mixed(nls == 1) : stage_smem_fp64(nls == 1);
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if (!st && (size_t)maxsm < smem) st = fail(M2CG_ERR_CUDA, "stage kernel needs %zu B shared memory, device has %d", smem, maxsm);
  if (!st && nls == 1) {
    const double* xc[3] = {c->hxc.data(), c->hyc.data(), c->hzc.data()};
    const double* dxs[3] = {c->hdx.data(), c->hdy.data(), c->hdz.data()};
    st = multiphase_create(c->stream, g, sk, *scheme, mats, nmat, *ls, xc, dxs, &c->mp);
    if (st) fail(st, "two-material setup refused or failed (status %d): interface options or level-set settings", (int)st);
  }
  if (!st) {
    const double* xc[3] = {c->hxc.data(), c->hyc.data(), c->hzc.data()};
    const double* dxs[3] = {c->hdx.data(), c->hdy.data(), c->hdz.data()};
    st = viscous_create(c->stream, g, sk.ed, mats, nmat, xc, dxs, &c->visc);
    if (st) fail(st, "viscous-flux buffers could not be allocated");
  }
  if (st) {
    m2cg_destroy(c);
    return st;
  }
  // The (x,y) tiles x z planes are shared evenly by a persistent grid of
  // resident CTAs, each share at least 8 planes long (the plane pipeline's
  // prologue costs about 2.5 planes per segment).
  const int ty = scheme->precision == M2CG_PREC_MIXED
                     ? StageTY<float, false>::value
                     : (nls == 1 ? StageTY<double, true>::value : StageTY<double, false>::value);
  c->ntx = (c->nx + TX - 1) / TX;
  c->nty = (c->ny + ty - 1) / ty;
  set_stage_items(c, nls == 1);
  CK(cudaStreamSynchronize(c->stream));
  *out = c;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_destroy(m2cg_ctx* c) {
  if (!c) return M2CG_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int q = 0; q < 4; q++)
    for (int b = 0; b < 2; b++) cudaFree(c->blk[q][b]);
  cudaFree(c->id);
  cudaFree(c->dx); cudaFree(c->dy); cudaFree(c->dz);
  for (int a = 0; a < 3; a++) { cudaFree(c->lA[a]); cudaFree(c->lB[a]); cudaFree(c->lK[a]); cudaFree(c->lC[a]); }
  cudaFree(c->clock); cudaFree(c->dtmin); cudaFree(c->clipflags); cudaFree(c->err);
  cudaFree(c->stage_buf);
  cudaFree(c->probe_ijk); cudaFree(c->probe_xi); cudaFree(c->probe_rec);
  if (c->mp) multiphase_destroy(c->mp);
  if (c->walls) walls_destroy(c->walls);
  if (c->visc) viscous_destroy(c->visc);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return M2CG_OK;
}

// ---------------------------------------------------------------------------
// Small kernels
// ---------------------------------------------------------------------------
// Ghosted AoS (host layout) -> interior SoA, with clipping of the primitive
// state (the end of SpaceOperator::SetInitialCondition clips, 1088).
__global__ void k_unpack_state(const double* aos, int nx, int ny, int nz, long long px, long long plane, int dof,
                               double* const* soa_ptrs_unused, double* s0, double* s1, double* s2, double* s3,
                               double* s4) {
  long long n = (long long)nx * ny * nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % nx);
    int j = (int)((q / nx) % ny);
    int k = (int)(q / ((long long)nx * ny));
    long long h = (((long long)(k + 1) * (ny + 2) + (j + 1)) * (nx + 2) + (i + 1)) * dof;
    long long o = (long long)k * plane + (long long)j * px + i;
    double* d[5] = {s0, s1, s2, s3, s4};
    for (int p = 0; p < dof; p++) d[p][o] = aos[h + p];
  }
}

__global__ void k_clip_state(Grid3 g, SchemeK sk, double* v0, double* v1, double* v2, double* v3, double* v4,
                             const uint8_t* id, DevError* err) {
  long long n = (long long)g.nx * g.ny * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % g.nx);
    int j = (int)((q / g.nx) % g.ny);
    int k = (int)(q / ((long long)g.nx * g.ny));
    long long o = (long long)k * g.plane + (long long)j * g.px + i;
    double V[5] = {v0[o], v1[o], v2[o], v3[o], v4[o]};
    if (id[o] >= sk.nmat) {  // inactive: VarFcnDummy::ClipDensityAndPressure sets its fixed state
      V[0] = sk.dummy[0]; V[1] = V[2] = V[3] = 0.0; V[4] = sk.dummy[1];
    } else {
      const Eos<double>& e = sk.ed[id[o]];
      e.clip(V);
      if (e.bad(V)) report(err, ERR_STATE, (int)q, 0);
    }
    v0[o] = V[0]; v1[o] = V[1]; v2[o] = V[2]; v3[o] = V[3]; v4[o] = V[4];
  }
}

struct F5 {
  float* p[5];
};

// FP32 copy of the interior state (the mixed path's stage-1 input).
__global__ void k_to_float(Grid3 g, const double* v0, const double* v1, const double* v2, const double* v3,
                           const double* v4, F5 f) {
  long long n = (long long)g.nx * g.ny * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % g.nx);
    int j = (int)((q / g.nx) % g.ny);
    int k = (int)(q / ((long long)g.nx * g.ny));
    long long o = (long long)k * g.plane + (long long)j * g.px + i;
    f.p[0][o] = (float)v0[o]; f.p[1][o] = (float)v1[o]; f.p[2][o] = (float)v2[o];
    f.p[3][o] = (float)v3[o]; f.p[4][o] = (float)v4[o];
  }
}

// IDs 0..nmat-1, or nmat (inactive) where the context allows it (no level
// set, no diffusive material); anything else is reported and stored as 0.
__global__ void k_unpack_id(const double* aos, int nx, int ny, int nz, long long px, long long plane, uint8_t* id,
                            int nmat, int allow_inactive, DevError* err) {
  long long n = (long long)nx * ny * nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % nx);
    int j = (int)((q / nx) % ny);
    int k = (int)(q / ((long long)nx * ny));
    long long h = ((long long)(k + 1) * (ny + 2) + (j + 1)) * (nx + 2) + (i + 1);
    const double v = aos[h];
    const int top = allow_inactive ? nmat : nmat - 1;
    const bool ok = v >= 0.0 && v <= (double)top;
    if (!ok) report(err, ERR_MATERIAL_ID, (int)q, 0);
    id[(long long)k * plane + (long long)j * px + i] = ok ? (uint8_t)v : (uint8_t)0;
  }
}

// Interior SoA -> ghosted AoS with face ghosts filled by the boundary rule
// (SpaceOperator::ApplyBoundaryConditions, 1667-1745). Edge/corner ghosts are
// left at zero (the reference never populates them).
__global__ void k_pack_state(Grid3 g, const double* s0, const double* s1, const double* s2, const double* s3,
                             const double* s4, const uint8_t* id, double* aos, double* idaos) {
  int gx = g.nx + 2, gy = g.ny + 2, gz = g.nz + 2;
  long long n = (long long)gx * gy * gz;
  const double* s[5] = {s0, s1, s2, s3, s4};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % gx) - 1;
    int j = (int)((q / gx) % gy) - 1;
    int k = (int)(q / ((long long)gx * gy)) - 1;
    int out[3] = {i < 0 ? 0 : i >= g.nx ? 1 : -1, j < 0 ? 0 : j >= g.ny ? 1 : -1, k < 0 ? 0 : k >= g.nz ? 1 : -1};
    int nout = (out[0] >= 0) + (out[1] >= 0) + (out[2] >= 0);
    double V[5] = {0, 0, 0, 0, 0};
    double idv = 0.0;
    if (nout <= 1) {
      int ii = i < 0 ? 0 : i >= g.nx ? g.nx - 1 : i;
      int jj = j < 0 ? 0 : j >= g.ny ? g.ny - 1 : j;
      int kk = k < 0 ? 0 : k >= g.nz ? g.nz - 1 : k;
      int axis = out[0] >= 0 ? 0 : out[1] >= 0 ? 1 : out[2] >= 0 ? 2 : -1;
      if (axis >= 0 && g.bc[2 * axis] == BC_PERIODIC) {
        int c3[3] = {i, j, k};
        int n3[3] = {g.nx, g.ny, g.nz};
        int w = (c3[axis] + n3[axis]) % n3[axis];
        if (axis == 0) ii = w; else if (axis == 1) jj = w; else kk = w;
        axis = -1;  // plain copy of the periodic image
      }
      long long o = (long long)kk * g.plane + (long long)jj * g.px + ii;
      for (int p = 0; p < 5; p++) V[p] = s[p][o];
      idv = id ? (double)id[o] : 0.0;
      if (axis >= 0) {
        int bc = g.bc[2 * axis + out[axis]];
        if (bc == BC_INLET) for (int p = 0; p < 5; p++) V[p] = g.inlet[p];
        else if (bc == BC_OUTLET) for (int p = 0; p < 5; p++) V[p] = g.outlet[p];
        else if (bc == BC_STICKWALL) { V[1] = -V[1]; V[2] = -V[2]; V[3] = -V[3]; }
        else V[axis + 1] = -V[axis + 1];
      }
    }
    for (int p = 0; p < 5; p++) aos[q * 5 + p] = V[p];
    if (idaos) idaos[q] = idv;
  }
}

// CFL sweep (SpaceOperator::FindExtremeValuesOfFlowVariables, 2128-2198):
// min over cells of min(dx/(|u|+c), dy/(|v|+c), dz/(|w|+c)).
// 2D CTAs of 32 x 8 cells over (i, j) walking a column of planes; the
// minimum is reduced per CTA (one atomic each).
__global__ void __launch_bounds__(256) k_cfl(Grid3 g, SchemeK sk, const double* v0, const double* v1,
                                             const double* v2, const double* v3, const double* v4,
                                             const uint8_t* id, unsigned long long* dtmin, DevError* err) {
  double best = 1.0e300;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long q = ((long long)k * g.ny + j) * g.nx + i;
    long long o = (long long)k * g.plane + (long long)j * g.px + i;
    if (id && id[o] >= sk.nmat) continue;  // inactive cells do not limit the step (SpaceOperator.cpp:2154)
    const Eos<double>& e = sk.ed[id ? id[o] : 0];
    double rho = v0[o], p = v4[o];
    double c2 = e.c2(rho, e.energy(rho, p));
    if (c2 < 0.0) report(err, ERR_SOUND, (int)q, 5);
    double c = sqrt(c2);
    double r = smin(g.dx[i] / (fabs(v1[o]) + c), smin(g.dy[j] / (fabs(v2[o]) + c), g.dz[k] / (fabs(v3[o]) + c)));
    best = smin(best, r);
  }
  for (int o = 16; o > 0; o >>= 1) best = smin(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ double wbest[8];
  if (threadIdx.x == 0) wbest[threadIdx.y] = best;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int w = 1; w < 8; w++) best = smin(best, wbest[w]);
    if (best < 1.0e300) atomicMin(dtmin, (unsigned long long)__double_as_longlong(best));
  }
}

__global__ void k_reset_dtmin(unsigned long long* dtmin) { *dtmin = 0x7ff0000000000000ull; }

// Device clock: dt = cfl * min(dx/lambda) (SpaceOperator::ComputeTimeStepSize,
// 2202-2227), shortened so the run ends at t_max (Main.cpp:537-541), t += dt.
// clock = [t, dt, t_max, cfl].
__global__ void k_clock_from_cfl(double* clock, unsigned long long* dtmin) {
  double m = __longlong_as_double((long long)*dtmin);
  double t = clock[0], tmax = clock[2], cfl = clock[3];
  double dt = cfl * m;
  if (t + dt > tmax) dt = tmax - t;
  clock[1] = dt;
  clock[0] = t + dt;
  *dtmin = 0x7ff0000000000000ull;
}

__global__ void k_set_clock(double* clock, double t, double dt, double tmax, double cfl) {
  clock[0] = t;
  clock[1] = dt;
  clock[2] = tmax;
  clock[3] = cfl;
}

static int grid1d(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

static m2cg_status sample_probes(m2cg_ctx* c);

static m2cg_status check_device_error(m2cg_ctx* c) {
  DevError e;
  CK(cudaMemcpyAsync(&e, c->err, sizeof e, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (e.code) {
    cudaMemsetAsync(c->err, 0, sizeof(DevError), c->stream);
    m2cg_status st = e.code == ERR_STATE || e.code == ERR_SOUND || e.code == ERR_HLLC ? M2CG_ERR_STATE
                     : e.code == ERR_RIEMANN ? M2CG_ERR_RIEMANN
                     : e.code == ERR_ITER_CAP ? M2CG_ERR_ITER_CAP
                     : e.code == ERR_UNSUPPORTED ? M2CG_ERR_UNSUPPORTED : M2CG_ERR_STATE;
    if (e.code == ERR_UNSUPPORTED)
      return fail(st, "unresolved background cells with apply_failsafe_density Off need the level-set "
                      "correction of unresolved cells, which is not supported");
    if (e.code == ERR_MATERIAL_ID)
      return fail(M2CG_ERR_ARG, "material ID out of range at cell %d: 0..nmat-1, or nmat (inactive, enclosed by "
                                "an embedded surface) in a context without a level set or diffusive materials",
                  e.cell);
    return fail(st, "device error code %d at cell %d (site %d)", e.code, e.cell, e.where);
  }
  return M2CG_OK;
}

static m2cg_status ensure_stage_buf(m2cg_ctx* c, size_t bytes) {
  if (c->stage_bytes >= bytes) return M2CG_OK;
  cudaFree(c->stage_buf);
  c->stage_buf = nullptr;
  c->stage_bytes = 0;
  if (cudaMalloc((void**)&c->stage_buf, bytes) != cudaSuccess) return fail(M2CG_ERR_NOMEM, "staging alloc failed");
  c->stage_bytes = bytes;
  return M2CG_OK;
}

static m2cg_status compute_dtmin(m2cg_ctx* c) {
  k_reset_dtmin<<<1, 1, 0, c->stream>>>(c->dtmin);
  double** V = c->V[c->cur];
  k_cfl<<<dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz < 64 ? c->nz : 64), dim3(32, 8), 0, c->stream>>>(
      c->g, c->sk, V[0], V[1], V[2], V[3], V[4],
                                                                         c->id, c->dtmin, c->err);
  c->counters.kernel_launches += 2;
  CK(cudaGetLastError());
  c->dtmin_valid = true;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_upload_state(m2cg_ctx* c, const double* V, const double* ID, const double* phi) {
  if (!c || !V) return fail(M2CG_ERR_ARG, "null argument");
  size_t ng = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  m2cg_status st = ensure_stage_buf(c, ng * 5 * sizeof(double));
  if (st) return st;
  long long n = (long long)c->nx * c->ny * c->nz;
  double** D = c->V[c->cur];
  if (ID) {
    CK(cudaMemcpyAsync(c->stage_buf, ID, ng * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    // inactive cells (ID = nmat): one material without a level set, no diffusive material
    const int allow_inactive = (!c->mp && !c->visc) ? 1 : 0;
    k_unpack_id<<<grid1d(n), 256, 0, c->stream>>>(c->stage_buf, c->nx, c->ny, c->nz, c->px, c->plane, c->id,
                                                  c->sk.nmat, allow_inactive, c->err);
  }
  CK(cudaMemcpyAsync(c->stage_buf, V, ng * 5 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  k_unpack_state<<<grid1d(n), 256, 0, c->stream>>>(c->stage_buf, c->nx, c->ny, c->nz, c->px, c->plane, 5, nullptr,
                                                    D[0], D[1], D[2], D[3], D[4]);
  k_clip_state<<<grid1d(n), 256, 0, c->stream>>>(c->g, c->sk, D[0], D[1], D[2], D[3], D[4], c->id, c->err);
  c->counters.kernel_launches += ID ? 3 : 2;
  if (c->scheme.precision == M2CG_PREC_MIXED) {
    F5 f;
    for (int p = 0; p < 5; p++) f.p[p] = c->Vf[c->cur][p];
    k_to_float<<<grid1d(n), 256, 0, c->stream>>>(c->g, D[0], D[1], D[2], D[3], D[4], f);
    c->counters.kernel_launches += 1;
  }
  CK(cudaGetLastError());
  c->rs_valid = false;
  if (c->mp) {
    st = multiphase_upload_phi(c->mp, c->stream, phi, c->stage_buf, c->id);
    if (st) return st;
  }
  st = compute_dtmin(c);
  if (st) return st;
  return check_device_error(c);
}

extern "C" m2cg_status m2cg_update_states_after_interface_motion(m2cg_ctx* c, const double* IDn, int use_rs,
                                                                 int* unresolved) {
  if (!c || !IDn) return fail(M2CG_ERR_ARG, "null argument");
  if (!c->mp) return fail(M2CG_ERR_ARG, "no level set: no cell changes material");
  if (use_rs && !c->rs_valid) return fail(M2CG_ERR_ARG, "no star states stored since the last upload");
  size_t ng = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  m2cg_status st = ensure_stage_buf(c, ng * sizeof(double));
  if (st) return st;
  long long n = (long long)c->nx * c->ny * c->nz;
  CK(cudaMemcpyAsync(c->stage_buf, IDn, ng * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  k_unpack_id<<<grid1d(n), 256, 0, c->stream>>>(c->stage_buf, c->nx, c->ny, c->nz, c->px, c->plane,
                                                 multiphase_idn(c->mp), c->sk.nmat, 0, c->err);
  CK(cudaGetLastError());
  const bool mixed = c->scheme.precision == M2CG_PREC_MIXED;
  st = multiphase_update_states(c->mp, c->stream, c->V[c->cur], mixed ? c->Vf[c->cur] : nullptr, c->id, c->err,
                                use_rs != 0, false, unresolved);
  if (st) return st;
  c->counters.kernel_launches += 5;
  st = compute_dtmin(c);
  if (st) return st;
  return check_device_error(c);
}

extern "C" m2cg_status m2cg_download_state(m2cg_ctx* c, double* V, double* ID, double* phi) {
  if (!c) return fail(M2CG_ERR_ARG, "null argument");
  size_t ng = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  m2cg_status st = ensure_stage_buf(c, ng * 6 * sizeof(double));
  if (st) return st;
  double** D = c->V[c->cur];
  k_pack_state<<<grid1d((long long)ng), 256, 0, c->stream>>>(c->g, D[0], D[1], D[2], D[3], D[4], c->id, c->stage_buf,
                                                             c->stage_buf + ng * 5);
  c->counters.kernel_launches += 1;
  CK(cudaGetLastError());
  if (V) CK(cudaMemcpyAsync(V, c->stage_buf, ng * 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (ID) CK(cudaMemcpyAsync(ID, c->stage_buf + ng * 5, ng * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (phi && c->mp) {
    st = multiphase_download_phi(c->mp, c->stream, phi);
    if (st) return st;
  }
  CK(cudaStreamSynchronize(c->stream));
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_compute_dt(m2cg_ctx* c, double* dt_out) {
  if (!c || !dt_out) return fail(M2CG_ERR_ARG, "null argument");
  m2cg_status st = compute_dtmin(c);
  if (st) return st;
  unsigned long long bits;
  CK(cudaMemcpyAsync(&bits, c->dtmin, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double m;
  memcpy(&m, &bits, sizeof m);
  *dt_out = c->scheme.cfl * m;
  return check_device_error(c);
}

// RK coefficients of stage s (1-based) for order r: U_new = a_prev*U_s + a_un*U^n + (b*dt)*R
// (TimeIntegrator.cpp:367-372, 588-593, 644-649).
static void rk_coeffs(int r, int s, double& a_prev, double& a_un, double& b) {
  a_prev = 0.0; a_un = 1.0; b = 1.0;
  if (s == 1) return;
  if (r == 2) { a_prev = 0.5; a_un = 0.5; b = 0.5; return; }
  if (s == 2) { a_prev = 0.25; a_un = 0.75; b = 0.25; return; }
  a_prev = 2.0 / 3.0; a_un = 1.0 / 3.0; b = 2.0 / 3.0;
}

// Persistent grid size of the stage kernel variant (two-material or not).
static void set_stage_items(m2cg_ctx* c, bool multi) {
  const int resident = c->scheme.precision == M2CG_PREC_MIXED ? stage_resident_mixed(c->scheme.flux, multi)
                                                               : stage_resident_fp64(c->scheme.flux, multi);
  const long long units = (long long)c->ntx * c->nty * c->nz;
  const long long by_len = (units + 7) / 8;
  c->nitems = (int)std::max<long long>(1, std::min<long long>(resident, by_len));
}

extern "C" m2cg_status m2cg_set_wall_faces(m2cg_ctx* c, int n, const int* faces, const double* nwall_fwd,
                                           const double* uwall_fwd, const double* nwall_bwd,
                                           const double* uwall_bwd) {
  if (!c || n < 0) return fail(M2CG_ERR_ARG, "bad argument");
  CK(cudaStreamSynchronize(c->stream));
  if (n == 0) {
    walls_destroy(c->walls);
    c->walls = nullptr;
    set_stage_items(c, c->mp != nullptr);
    return M2CG_OK;
  }
  // HeatDiffusionOperator::AddDiffusionFluxes leaves cut faces alone (its
  // EBDS argument is unused); ViscosityOperator's ghost-fluid population at
  // cut faces (ViscosityOperator.cpp:208-213) is not built
  if (viscous_has_viscosity(c->visc))
    return fail(M2CG_ERR_UNSUPPORTED,
                "cut faces with viscous materials (the viscosity operator's ghost-fluid branch) are not implemented");
  const size_t smem = c->scheme.precision == M2CG_PREC_MIXED ? stage_smem_mixed(true) : stage_smem_fp64(true);
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if ((size_t)maxsm < smem) return fail(M2CG_ERR_CUDA, "stage kernel needs %zu B shared memory, device has %d", smem, maxsm);
  Walls* w = nullptr;
  char msg[200] = {0};
  const m2cg_status st = walls_create(c->stream, c->g, c->nalloc, c->scheme, n, faces, nwall_fwd, uwall_fwd, nwall_bwd,
                                      uwall_bwd, &w, msg, sizeof msg);
  if (st) return fail(st, "cut faces refused: %s", msg);
  walls_destroy(c->walls);
  c->walls = w;
  set_stage_items(c, true);
  return M2CG_OK;
}

static m2cg_status launch_stage(m2cg_ctx* c, StageArgs& a) {
  a.ntx = c->ntx;
  a.nty = c->nty;
  a.nitems = c->nitems;
  int grid = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->profile) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c->stream);
  }
  // the two-material kernel variant also carries the branch of cut faces
  const bool multi = c->mp != nullptr || c->walls != nullptr;
  cudaError_t e = c->scheme.precision == M2CG_PREC_MIXED ? launch_stage_mixed(a, c->stream, multi, &grid)
                                                          : launch_stage_fp64(a, c->stream, multi, &grid);
  if (c->profile) {
    cudaEventRecord(e1, c->stream);
    c->ev.push_back(e0);
    c->ev.push_back(e1);
  }
  c->counters.kernel_launches += 1;
  if (e != cudaSuccess) return fail(M2CG_ERR_CUDA, "stage launch: %s", cudaGetErrorString(e));
  return M2CG_OK;
}

static void base_args(m2cg_ctx* c, StageArgs& a) {
  memset(&a, 0, sizeof a);
  a.use_tma = c->tma_ok && c->g.bc[0] != BC_PERIODIC && c->g.bc[2] != BC_PERIODIC;
  a.g = c->g;
  a.s = c->sk;
  a.id = c->id;
  a.clock = c->clock;
  a.err = c->err;
}

// All RK stages of one step; dt is already in the device clock.
static m2cg_status rk_step(m2cg_ctx* c, bool want_dtmin) {
  int r = c->scheme.rk_order;
  double** Vn = c->V[c->cur];
  double** Vo = c->V[1 - c->cur];
  cudaMemsetAsync(c->clipflags, 0, 4 * sizeof(int), c->stream);
  if (c->mp) {
    m2cg_status st = multiphase_begin_step(c->mp, c->stream, Vn, c->id);
    if (st) return st;
  }
  const bool mixed = c->scheme.precision == M2CG_PREC_MIXED;
  for (int s = 1; s <= r; s++) {
    StageArgs a;
    base_args(c, a);
    a.stage = s;
    a.final_stage = s == r;
    rk_coeffs(r, s, a.a_prev, a.a_un, a.bdt_coef);
    for (int p = 0; p < 5; p++) {
      a.Vn[p] = Vn[p];
      a.Us[p] = s == 1 ? nullptr : c->U[(s - 2) & 1][p];
      a.Uo[p] = c->U[(s - 1) & 1][p];
      a.Vo[p] = Vo[p];
      if (s == 1)
        a.Pin[p] = mixed ? (const void*)c->Vf[c->cur][p] : (const void*)Vn[p];
      else
        a.Pin[p] = c->P[(s - 2) & 1][p];
      a.Po[p] = s == r ? nullptr : c->P[(s - 1) & 1][p];
      a.Vfo[p] = (s == r && mixed) ? c->Vf[1 - c->cur][p] : nullptr;
    }
    a.tin = c->tmap[s == 1 ? c->cur : 2 + ((s - 2) & 1)];
    a.us_clipped = s > 1 ? c->clipflags + (s - 2) : nullptr;
    a.clipped_out = c->clipflags + (s - 1);
    a.dtmin_bits = (a.final_stage && want_dtmin && !c->mp) ? c->dtmin : nullptr;
    {  // face pass: reconstructed states of the interface / cut faces (LINEAR)
      StageArgs fa = a;
      bool fp = c->mp && multiphase_face_pass(c->mp, fa);
      if (c->walls && walls_face_pass(c->walls, fa)) fp = true;
      if (fp) {
        m2cg_status st = launch_stage(c, fa);
        if (st) return st;
      }
    }
    if (c->walls) walls_view(c->walls, a);  // the interface pre-pass skips cut faces
    if (c->mp) {
      m2cg_status st = multiphase_stage(c->mp, c->stream, a);
      if (st) return st;
    }
    if (c->visc) {
      m2cg_status sv = viscous_faces(c->visc, c->stream, a, mixed);
      if (sv) return fail(sv, "viscous-flux launch failed");
    }
    if (c->walls && walls_stage(c->walls, c->stream, a)) return fail(M2CG_ERR_CUDA, "cut-face pre-pass launch failed");
    m2cg_status st = launch_stage(c, a);
    if (st) return st;
  }
  c->cur = 1 - c->cur;
  if (c->mp) {
    m2cg_status st = multiphase_end_step(c->mp, c->stream, c->V[1 - c->cur], c->V[c->cur],
                                         mixed ? c->Vf[c->cur] : nullptr, c->id, c->clock, c->err, &c->counters);
    if (st) return st;
    c->dtmin_valid = false;
    c->rs_valid = true;
  } else {
    c->dtmin_valid = want_dtmin;
  }
  c->counters.steps += 1;
  c->counters.cells_updated += (long long)c->nx * c->ny * c->nz;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_advance(m2cg_ctx* c, double t_new, double dt, int time_step) {
  if (!c) return fail(M2CG_ERR_ARG, "null argument");
  (void)time_step;
  k_set_clock<<<1, 1, 0, c->stream>>>(c->clock, t_new, dt, 1.0e300, c->scheme.cfl);
  k_reset_dtmin<<<1, 1, 0, c->stream>>>(c->dtmin);
  c->counters.kernel_launches += 2;
  if (c->mp) multiphase_set_step(c->mp, time_step);
  m2cg_status st = rk_step(c, true);
  if (st) return st;
  if (c->nprobe && c->probe_every > 0 && c->counters.steps % c->probe_every == 0) {
    st = sample_probes(c);
    if (st) return st;
  }
  return check_device_error(c);
}

// Steps with dt from the CFL condition; no host synchronisation per step
// unless t_max is finite (then t is read back each step to stop exactly
// where the reference's loop stops, Main.cpp:514).
static m2cg_status run_steps(m2cg_ctx* c, int nsteps, double t_max, double t0, double* t, int* done, bool check) {
  k_set_clock<<<1, 1, 0, c->stream>>>(c->clock, t0, 0.0, t_max, c->scheme.cfl);
  c->counters.kernel_launches += 1;
  int n = 0;
  double tnow = t0;
  bool finite = std::isfinite(t_max);
  while (n < nsteps && (!finite || tnow < t_max)) {
    if (!c->dtmin_valid) {
      m2cg_status st = compute_dtmin(c);
      if (st) return st;
    }
    k_clock_from_cfl<<<1, 1, 0, c->stream>>>(c->clock, c->dtmin);
    c->counters.kernel_launches += 1;
    if (c->mp) multiphase_set_step(c->mp, -1);
    m2cg_status st = rk_step(c, true);
    if (st) return st;
    if (c->nprobe && c->probe_every > 0 && c->counters.steps % c->probe_every == 0) {
      st = sample_probes(c);
      if (st) return st;
    }
    n++;
    if (finite) {
      CK(cudaMemcpyAsync(&tnow, c->clock, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
  }
  if (!finite) {
    CK(cudaMemcpyAsync(&tnow, c->clock, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  if (done) *done = n;
  if (check) {
    m2cg_status st = check_device_error(c);
    if (st) return st;
  }
  if (t) *t = tnow;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_run(m2cg_ctx* c, int nsteps, double t_max, double* t, int* steps_done) {
  if (!c) return fail(M2CG_ERR_ARG, "null argument");
  double t0 = t ? *t : 0.0;
  return run_steps(c, nsteps, t_max, t0, t, steps_done, true);
}

extern "C" m2cg_status m2cg_compute_residual(m2cg_ctx* c, double* R_host) {
  if (!c || !R_host) return fail(M2CG_ERR_ARG, "null argument");
  StageArgs a;
  base_args(c, a);
  a.stage = 1;
  a.final_stage = 0;
  a.bdt_coef = 0.0;
  double** Vn = c->V[c->cur];
  for (int p = 0; p < 5; p++) {
    a.Vn[p] = Vn[p];
    a.Uo[p] = c->U[0][p];
    a.Ro[p] = c->U[1][p];
    a.Pin[p] = c->scheme.precision == M2CG_PREC_MIXED ? (const void*)c->Vf[c->cur][p] : (const void*)Vn[p];
  }
  a.tin = c->tmap[c->cur];
  if (c->mp) {
    c->rs_valid = false;  // the interface slots are reassigned
    m2cg_status st = multiphase_begin_step(c->mp, c->stream, Vn, c->id);
    if (st) return st;
  }
  {  // face pass: reconstructed states of the interface / cut faces (LINEAR)
    StageArgs fa = a;
    bool fp = c->mp && multiphase_face_pass(c->mp, fa);
    if (c->walls && walls_face_pass(c->walls, fa)) fp = true;
    if (fp) {
      m2cg_status st = launch_stage(c, fa);
      if (st) return st;
    }
  }
  if (c->walls) walls_view(c->walls, a);  // the interface pre-pass skips cut faces
  if (c->mp) {
    m2cg_status st = multiphase_stage(c->mp, c->stream, a);
    if (st) return st;
  }
  if (c->visc) {
    m2cg_status sv = viscous_faces(c->visc, c->stream, a, c->scheme.precision == M2CG_PREC_MIXED);
    if (sv) return fail(sv, "viscous-flux launch failed");
  }
  if (c->walls && walls_stage(c->walls, c->stream, a)) return fail(M2CG_ERR_CUDA, "cut-face pre-pass launch failed");
  m2cg_status st = launch_stage(c, a);
  if (st) return st;
  // pack R (interior) into the ghosted AoS layout
  size_t ng = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  st = ensure_stage_buf(c, ng * 6 * sizeof(double));
  if (st) return st;
  Grid3 gz = c->g;
  for (int q = 0; q < 6; q++) gz.bc[q] = M2CG_BC_OUTLET;  // ghosts of R are not meaningful
  for (int p = 0; p < 5; p++) { gz.outlet[p] = 0.0; gz.inlet[p] = 0.0; }
  double** R = c->U[1];
  k_pack_state<<<grid1d((long long)ng), 256, 0, c->stream>>>(gz, R[0], R[1], R[2], R[3], R[4], nullptr, c->stage_buf,
                                                             nullptr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(R_host, c->stage_buf, ng * 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

extern "C" m2cg_status m2cg_get_counters(const m2cg_ctx* c, m2cg_counters* out) {
  if (!c || !out) return fail(M2CG_ERR_ARG, "null argument");
  *out = c->counters;
  if (c->mp) multiphase_counters(c->mp, out);
  if (c->walls) {
    long long solves = 0, failures = 0;
    walls_counters(c->walls, c->stream, &solves, &failures);
    out->wall_riemann_calls += solves;
    out->riemann_errors += failures;
  }
  return M2CG_OK;
}

// ---------------------------------------------------------------------------
// Timing entry point used by the benchmark: nsteps CFL steps with the state
// resident in HBM, bracketed by CUDA events on the context's stream.
// ---------------------------------------------------------------------------
extern "C" m2cg_status m2cg_time_steps(m2cg_ctx* c, int nsteps, float* ms_out, long long* launches_out) {
  if (!c) return fail(M2CG_ERR_ARG, "null argument");
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  long long l0 = c->counters.kernel_launches;
  CK(cudaEventRecord(e0, c->stream));
  double t = 0.0;
  int done = 0;
  m2cg_status st = run_steps(c, nsteps, INFINITY, 0.0, &t, &done, false);
  if (st) return st;
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms_out) *ms_out = ms;
  if (launches_out) *launches_out = c->counters.kernel_launches - l0;
  return check_device_error(c);
}

// Stream of the context (cudaStream_t), for callers that time on it.
extern "C" m2cg_status m2cg_get_stream(const m2cg_ctx* c, void** stream) {
  if (!c || !stream) return fail(M2CG_ERR_ARG, "null argument");
  *stream = (void*)c->stream;
  return M2CG_OK;
}

// Per-launch device time of the fused stage kernel over nsteps CFL steps
// (CUDA events around each launch on the context's stream): total stage
// milliseconds, number of stage launches, and whole-step milliseconds.
extern "C" m2cg_status m2cg_profile_stages(m2cg_ctx* c, int nsteps, float* stage_ms, int* stage_launches,
                                           float* step_ms) {
  if (!c) return fail(M2CG_ERR_ARG, "null argument");
  c->profile = true;
  c->ev.clear();
  float total = 0.f;
  m2cg_status st = m2cg_time_steps(c, nsteps, &total, nullptr);
  c->profile = false;
  if (st) return st;
  float sum = 0.f;
  for (size_t q = 0; q + 1 < c->ev.size(); q += 2) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[q], c->ev[q + 1]);
    sum += ms;
    cudaEventDestroy(c->ev[q]);
    cudaEventDestroy(c->ev[q + 1]);
  }
  if (stage_ms) *stage_ms = sum;
  if (stage_launches) *stage_launches = (int)(c->ev.size() / 2);
  if (step_ms) *step_ms = total;
  c->ev.clear();
  return M2CG_OK;
}

// ---------------------------------------------------------------------------
// Probes (ProbeOutput::SetupInterpolation / InterpolateSolutionAtProbe,
// ProbeOutput.cpp:219-340, 636-673)
// ---------------------------------------------------------------------------
struct V5 {
  double* p[5];
};

// Node value of component p at (i, j, k), interior or face ghost (the
// boundary rule of ApplyBoundaryConditions, as written into the ghosted
// host layout by m2cg_download_state).
__device__ double node_value(const Grid3& g, double* const* V, int i, int j, int k, int p) {
  int out[3] = {i < 0 ? 0 : i >= g.nx ? 1 : -1, j < 0 ? 0 : j >= g.ny ? 1 : -1, k < 0 ? 0 : k >= g.nz ? 1 : -1};
  int ii = i < 0 ? 0 : i >= g.nx ? g.nx - 1 : i;
  int jj = j < 0 ? 0 : j >= g.ny ? g.ny - 1 : j;
  int kk = k < 0 ? 0 : k >= g.nz ? g.nz - 1 : k;
  int axis = out[0] >= 0 ? 0 : out[1] >= 0 ? 1 : out[2] >= 0 ? 2 : -1;
  if (axis >= 0 && g.bc[2 * axis] == BC_PERIODIC) {
    const int c3[3] = {i, j, k}, n3[3] = {g.nx, g.ny, g.nz};
    const int w = (c3[axis] + n3[axis]) % n3[axis];
    if (axis == 0) ii = w; else if (axis == 1) jj = w; else kk = w;
    axis = -1;
  }
  double v = V[p][(long long)kk * g.plane + (long long)jj * g.px + ii];
  if (axis >= 0) {
    const int bc = g.bc[2 * axis + out[axis]];
    if (bc == BC_INLET) v = g.inlet[p];
    else if (bc == BC_OUTLET) v = g.outlet[p];
    else if (bc == BC_STICKWALL) v = (p >= 1 && p <= 3) ? -v : v;
    else if (p == axis + 1) v = -v;
  }
  return v;
}

// One record: every component of every probe; invalid corners count as
// zero, and with fewer than 8 valid corners they take the average of the
// others (636-669); then the trilinear interpolation of
// MathTools::trilinear_interpolation (the local-coordinate form).
__global__ void k_sample_probes(Grid3 g, V5 V, const int* ijk, const double* xi, int n, const double* clock,
                                double step, double* rec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q == 0) {
    rec[0] = clock[0];
    rec[1] = step;
  }
  if (q >= 5 * n) return;
  const int pr = q / 5, p = q - 5 * pr;
  const int i = ijk[4 * pr], j = ijk[4 * pr + 1], k = ijk[4 * pr + 2], valid = ijk[4 * pr + 3];
  double c[8];
  int nv = 0;
  for (int a = 0; a < 8; a++) {  // c000, c100, c010, c110, c001, c101, c011, c111
    const bool ok = (valid >> a) & 1;
    c[a] = ok ? node_value(g, V.p, i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1), p) : 0.0;
    nv += ok;
  }
  if (nv < 8) {
    const double avg = (c[0] + c[1] + c[2] + c[3] + c[4] + c[5] + c[6] + c[7]) / nv;
    for (int a = 0; a < 8; a++)
      if (!((valid >> a) & 1)) c[a] = avg;
  }
  const double* x = xi + 3 * pr;
  const double c00 = c[0] * (1.0 - x[0]) + c[1] * x[0];
  const double c01 = c[4] * (1.0 - x[0]) + c[5] * x[0];
  const double c10 = c[2] * (1.0 - x[0]) + c[3] * x[0];
  const double c11 = c[6] * (1.0 - x[0]) + c[7] * x[0];
  const double c0 = c00 * (1.0 - x[1]) + c10 * x[1];
  const double c1 = c01 * (1.0 - x[1]) + c11 * x[1];
  rec[2 + q] = c0 * (1.0 - x[2]) + c1 * x[2];
}

static m2cg_status sample_probes(m2cg_ctx* c) {
  if (!c->nprobe) return M2CG_OK;
  if (c->probe_count >= c->probe_cap) return fail(M2CG_ERR_ARG, "probe record buffer full (read it with m2cg_read_probes)");
  V5 v;
  for (int p = 0; p < 5; p++) v.p[p] = c->V[c->cur][p];
  double* rec = c->probe_rec + (size_t)c->probe_count * (2 + 5 * c->nprobe);
  k_sample_probes<<<(5 * c->nprobe + 127) / 128, 128, 0, c->stream>>>(c->g, v, c->probe_ijk, c->probe_xi, c->nprobe,
                                                                      c->clock, (double)c->counters.steps, rec);
  c->counters.kernel_launches += 1;
  c->probe_count++;
  CK(cudaGetLastError());
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_set_probes(m2cg_ctx* c, int n, const double* xyz, int every, int capacity) {
  if (!c || n < 0 || (n > 0 && (!xyz || capacity < 1))) return fail(M2CG_ERR_ARG, "bad probe arguments");
  cudaStreamSynchronize(c->stream);
  cudaFree(c->probe_ijk); cudaFree(c->probe_xi); cudaFree(c->probe_rec);
  c->probe_ijk = nullptr; c->probe_xi = nullptr; c->probe_rec = nullptr;
  c->nprobe = 0;
  c->probe_count = 0;
  if (n == 0) return M2CG_OK;
  // ghosted coordinates (SpaceOperator::PopulateGhostBoundaryCoordinates: x_0 - dx_0, x_{N-1} + dx_{N-1})
  const std::vector<double>* xc[3] = {&c->hxc, &c->hyc, &c->hzc};
  const std::vector<double>* dx[3] = {&c->hdx, &c->hdy, &c->hdz};
  const int N[3] = {c->nx, c->ny, c->nz};
  std::vector<double> X[3];
  for (int a = 0; a < 3; a++) {
    X[a].resize(N[a] + 2);
    X[a][0] = (*xc[a])[0] - (*dx[a])[0];
    for (int q = 0; q < N[a]; q++) X[a][q + 1] = (*xc[a])[q];
    X[a][N[a] + 1] = (*xc[a])[N[a] - 1] + (*dx[a])[N[a] - 1];
  }
  auto crd = [&](int a, int idx) { return X[a][idx + 1]; };
  // SpaceVariable3D::OutsidePhysicalDomainAndUnpopulated (SpaceVariable.h:150-159), with its test of
  // j (not i) against NX on the x axis kept: a node outside in more than one count is not populated
  auto unpopulated = [&](int i, int j, int k) {
    int count = 0;
    if (i < 0 || j >= N[0]) count++;
    if (j < 0 || j >= N[1]) count++;
    if (k < 0 || k >= N[2]) count++;
    return count > 1;
  };
  std::vector<int> ijk(4 * (size_t)n);
  std::vector<double> xi(3 * (size_t)n);
  for (int q = 0; q < n; q++) {
    int id3[3];
    for (int a = 0; a < 3; a++) {
      const double pa = xyz[3 * q + a];
      if (pa < crd(a, -1) || pa >= crd(a, N[a])) return fail(M2CG_ERR_ARG, "cannot locate probe node %d in the domain", q);
      int found = -2;
      for (int i = -2; i < N[a]; i++)
        if (pa < crd(a, i + 1)) { found = i; break; }
      id3[a] = found;
      xi[3 * q + a] = (pa - crd(a, found)) / (crd(a, found + 1) - crd(a, found));
    }
    int mask = 0, nv = 0;
    for (int b = 0; b < 8; b++) {
      const bool ok = !unpopulated(id3[0] + (b & 1), id3[1] + ((b >> 1) & 1), id3[2] + ((b >> 2) & 1));
      mask |= ok ? (1 << b) : 0;
      nv += ok;
    }
    if (nv == 0) return fail(M2CG_ERR_ARG, "probe node %d is too close to the edges of the domain boundary", q);
    ijk[4 * q] = id3[0]; ijk[4 * q + 1] = id3[1]; ijk[4 * q + 2] = id3[2]; ijk[4 * q + 3] = mask;
  }
  const size_t rec = (size_t)capacity * (2 + 5 * (size_t)n) * sizeof(double);
  if (cudaMalloc((void**)&c->probe_ijk, ijk.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&c->probe_xi, xi.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&c->probe_rec, rec) != cudaSuccess)
    return fail(M2CG_ERR_NOMEM, "probe buffers: allocation failed");
  CK(cudaMemcpy(c->probe_ijk, ijk.data(), ijk.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->probe_xi, xi.data(), xi.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->nprobe = n;
  c->probe_every = every;
  c->probe_cap = capacity;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_sample_probes(m2cg_ctx* c) {
  if (!c) return fail(M2CG_ERR_ARG, "null argument");
  return sample_probes(c);
}

extern "C" m2cg_status m2cg_read_probes(m2cg_ctx* c, double* records, int* nrec) {
  if (!c || !nrec) return fail(M2CG_ERR_ARG, "null argument");
  *nrec = c->probe_count;
  if (c->probe_count && records)
    CK(cudaMemcpyAsync(records, c->probe_rec, (size_t)c->probe_count * (2 + 5 * c->nprobe) * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->probe_count = 0;
  return M2CG_OK;
}

// Attach the learned warm start to the context's interface Riemann solves.
extern "C" m2cg_status m2cg_set_mlp(m2cg_ctx* c, const m2cg_mlp* m) {
  if (!c) return fail(M2CG_ERR_ARG, "null argument");
  if (!c->mp) return fail(M2CG_ERR_ARG, "no level set: the context has no interface Riemann problems");
  m2cg_status st = multiphase_set_mlp(c->mp, m);
  if (st) return fail(st, "allocation of the warm-start buffers failed");
  return M2CG_OK;
}

// Select the CUDA device for contexts created afterwards on this thread.
extern "C" m2cg_status m2cg_set_device(int device) {
  CK(cudaSetDevice(device));
  return M2CG_OK;
}
