// One fused Runge-Kutta stage of the finite-volume step on a structured box:
//   load state (C2P + clip on the fly) -> MUSCL slopes + face states with the
//   reference's revert rules -> numerical fluxes on every face once ->
//   per-cell residual in the reference's summation order -> RK update ->
//   (last stage) primitive output + CFL reduction.
//
// Replaces, per stage, SpaceOperator::ComputeResidual (SpaceOperator.cpp:3351-3409)
// = Reconstructor::Reconstruct (Reconstructor.cpp:332-904) +
//   SpaceOperator::CheckReconstructedStates (SpaceOperator.cpp:3198-3347) +
//   the face loop of SpaceOperator::ComputeAdvectionFluxes (2423-2815),
// and the RK arithmetic of TimeIntegratorRK2/RK3::AdvanceOneTimeStep
// (TimeIntegrator.cpp:291-428, 496-690) with ConservativeToPrimitive,
// ClipDensityAndPressure and ApplyBoundaryConditions (SpaceOperator.cpp:553-649, 1667-1745).
//
// Layout in HBM: structure-of-arrays FP64, interior cells only
// (index (k*ny + j)*px + i, row pitch px); ghost values are never stored:
// they are rebuilt from interior cells by the boundary rule when loaded.
//
// Work decomposition: a CTA owns a 32 x TY column of cells and marches along
// z through a chunk of planes, keeping a ring of 4 primitive planes (with a
// 2-cell x/y halo) in shared memory. The stage's input is a primitive state
// in the compute type (V^n for stage 1; for later stages clip(C2P(U_s)),
// written by the previous stage's update), so planes are copied into the
// ring as they lie in HBM and only ghost cells are rewritten by the boundary
// rule. A plane of all five components lands with ONE tensor copy
// (cp.async.bulk.tensor over a 4D map x, y, z, component of the
// five-component buffer; box 40 x (TY+4) x 1 x 5 starting at x = i0-4, a
// 16-byte boundary; completion counted on an mbarrier per ring slot),
// issued by one thread; cells outside the domain in x/y arrive as zeros and
// take their value from their image cell by the boundary rule. Where x or y
// is periodic the halo wraps around the domain, which a tiled copy cannot
// express; those launches copy each value with cp.async from its wrapped
// position instead. Iteration m of the plane pipeline:
//   (1) ghost rules on plane m+2 (landed), copy of plane m+3 into the
//       slot plane m-1 has freed,
//   (2) slopes + revert mask of every cell of plane m+1 (x -1..32, y -1..TY),
//   (3) every face flux once: x/y faces of plane m and the z faces m+1/2,
//   (4) residual + RK update of plane m (z faces m-1/2 and m+1/2 from the
//       two-plane z-flux ring), writing the next stage's primitive input.
// Face states follow Reconstructor.cpp: slope-limited primitive values, the
// first face (in the order l,r,b,t,k,f) failing CheckState reverted to the
// cell value, every face needing clipping reverted to the cell value, and a
// remaining CheckState failure reported as an error (never a trap).
#pragma once
#include <cuda.h>  // CUtensorMap

#include "physics.cuh"

namespace m2c {

constexpr int MAXMAT = 4;
constexpr int TX = 32;
// Width of the plane box in x: cells i0-4 .. i0+35 (the tile's loaded
// columns i0-2 .. i0+33 plus two unused columns each side, so that the box
// starts on a 16-byte boundary for 4- and 8-byte elements).
constexpr int STAGE_TMA_BX = 40;
// Upper bound of mbarrier polls for one plane copy (a copy from valid
// addresses always lands; the bound turns a fault into an error status).
constexpr int STAGE_TMA_POLLS = 1 << 22;

enum { BC_NONE = 0, BC_INLET = 1, BC_OUTLET = 2, BC_SLIPWALL = 3, BC_STICKWALL = 4, BC_SYMMETRY = 5,
       BC_PERIODIC = 100 };

struct DevError {
  int code;
  int cell;   // linear interior index of the first failing cell (or -1)
  int where;  // stage * 16 + site
  int pad;
};

struct Grid3 {
  int nx, ny, nz;
  long long px, plane;  // row pitch, plane size (elements)
  int bc[6];
  double inlet[5], outlet[5];
  const double* dx;     // per axis cell widths (interior, length n)
  const double* dy;
  const double* dz;
  const double* lA[3];  // limiter coefficient A per axis index
  const double* lB[3];  // limiter coefficient B per axis index
  const int* lK[3];     // van Albada exponent per axis index
  const double* lC[3];  // generalized minmod B/(A+1) per axis index
  // per axis: 1 if A, B, K and C are the same at every index (uniform
  // meshes), which then stand in for the arrays
  int lu[3];
  double lA0[3], lB0[3], lC0[3];
  int lK0[3];
};

struct SchemeK {
  int flux, limiter, rec_linear, slope_zero_at_interface;
  int rec_var;             // ReconstructionData::VariableType: 0 primitive, 1 conservative,
                           // 2 primitive characteristic, 3 conservative characteristic
  double alpha, delta;
  int nmat;               // material IDs 0..nmat-1; nmat = inactive (enclosed by an embedded surface)
  double dummy[3];         // the inactive cells' fixed state: density, pressure, internal energy per mass
  Eos<double> ed[MAXMAT];  // per-material EOS, FP64 (built on the host)
  Eos<float> ef[MAXMAT];   // the same in FP32 for the mixed path's flux half
};

// Interface faces of a two-material stage: for a cell, the star states of
// the exact Riemann problems on its three low faces (x, y, z), found through
// slot[cell] (written only where a low face separates two materials).
struct IfaceView {
  const int* slot;       // per cell; valid only where a low face is an interface
  const double* Vsm;     // [slot][3 faces][5]: left star state  (Riemann side idl)
  const double* Vsp;     // [slot][3 faces][5]: right star state (Riemann side idr)
  const double* Vmid;    // [slot][3 faces][5]: state at xi = 0 (EXACT flux)
  const int* midid;      // [slot][3 faces]
  int mp_flux;           // 0 EXACT, 1 NUMERICAL, 2 LLF
  int mp_recon;          // 0 CONSTANT (cell states), 1 LINEAR (face states)
  // Face pass (LINEAR interface reconstruction): if set, the kernel only
  // writes the reconstructed states on both sides of every interface face,
  // [slot][3 faces][left, right][5], for the exact Riemann problems solved
  // before the stage proper; no flux, no update.
  double* faces_out;
};

// Viscous face fluxes (area-weighted; momentum x, y, z and energy, the mass
// component being zero): fr[d] is added by the right cell of a face of axis
// d, fl[d] subtracted by its left cell; [4][faces], faces of axis d indexed
// x: (k ny + j)(nx + 1) + i, y: (k (ny + 1) + j) nx + i, z: (k ny + j) nx + i
// with (i, j, k) the face's right cell. fr[0] == NULL: inviscid.
struct ViscView {
  const double* fr[3];
  const double* fl[3];
  const double* fh[3];  // heat-diffusion flux per face (energy only), same indexing; NULL: none
  long long nf[3];
};

// Faces cut by an embedded surface (walls) and the one-sided Riemann star
// states of their two sides for this stage, from the wall pre-pass
// (SpaceOperator.cpp:2438-2484 and the y/z analogues). mask == NULL: no walls.
struct WallView {
  const uint8_t* mask;  // per cell: bit d set where the low face along axis d is a wall
  const int* slot;      // per cell; valid only where mask != 0
  const double* Vsm;    // [slot][3 faces][5]: the low neighbour's star state (its flux against it)
  const double* Vsp;    // [slot][3 faces][5]: this cell's star state
  int linear;           // EmbeddedBoundaryMethodData::recon LINEAR: reconstructed face states
  // Face pass (LINEAR): if set, the kernel writes the reconstructed states
  // on both sides of every cut face, [slot][3 faces][low, high][5], for the
  // one-sided problems solved before the stage proper; no flux, no update.
  double* faces_out;
};

struct StageArgs {
  Grid3 g;
  SchemeK s;
  const void* Pin[5];    // stage input: primitive state in the compute type (see above)
  void* Po[5];           // non-final stages: clip(C2P(U_new)) in the compute type
  float* Vfo[5];         // final stage, FP32 compute type: FP32 copy of the new state
  const double* Vn[5];   // V^n (primitive) - step state
  const double* Us[5];   // flux source of stages >= 2 (conserved, raw)
  double* Uo[5];         // stage output (conserved) for non-final stages
  double* Vo[5];         // final-stage output (primitive)
  const uint8_t* id;     // material id per cell
  int stage;             // 1-based
  int final_stage;
  double a_prev, a_un;   // U_new = a_prev*U_s + a_un*U^n (stages >= 2)
  double bdt_coef;       // U_new += (bdt_coef*dt)*R; 1.0 for stage 1
  const double* clock;   // device clock: [0] t, [1] dt
  const int* us_clipped; // non-zero: U_s := P2C(clip(C2P(U_s))) everywhere (TimeIntegrator.cpp:542-545)
  int* clipped_out;      // set if any cell of this stage's output was clipped
  unsigned long long* dtmin_bits;  // final stage: min dx/(|u|+c) as ordered bits
  DevError* err;
  int ntx, nty;          // tiles in x and y
  int nitems;            // CTAs that share the (tile, plane) units evenly
  double* Ro[5];         // if set: write the residual R only (no RK update)
  IfaceView iface;
  ViscView visc;
  WallView wall;
  int use_tma;           // planes by tensor copy (x and y not periodic, maps built)
  CUtensorMap tin;       // 4D map of the stage input (Pin as one five-component buffer)
};

__device__ __forceinline__ void report(DevError* e, int code, int cell, int where) {
  if (atomicCAS(&e->code, 0, code) == 0) {
    e->cell = cell;
    e->where = where;
  }
}

template <typename T, int TY>
struct StageSmem {
  static constexpr int RX = TX + 4, RY = TY + 4;   // loaded region: x -2..TX+1, y -2..TY+1
  static constexpr int BX = STAGE_TMA_BX;          // stored columns: x -4..TX+3 (loaded column lx at lx + 2)
  static constexpr int MX = TX + 2, MY = TY + 2;   // mask region: x -1..TX, y -1..TY
  static constexpr int NFX = (TX + 1) * TY;        // x faces of a plane
  static constexpr int NFY = TX * (TY + 1);        // y faces of a plane
  static constexpr int NFZ = TX * TY;              // z faces between two planes
  alignas(128) T v[4][5][RY][BX];  // ring of primitive planes, slot = plane & 3 (tensor-copy boxes)
  T sig[2][3][5][MY][MX];     // limited slopes (x, y, z) of the mask region, two planes
  T fx[5][NFX];
  T fy[5][NFY];
  T fz[2][5][NFZ];
  uint8_t mask[2][MY][MX];
  uint8_t real[4][RY][RX];    // 1 = real (interior or periodic image), 0 = ghost / unused
  uint8_t ids[4][RY][RX];
  double red[TY * TX / 32];
  unsigned long long bar[4];  // one mbarrier per ring slot (tensor copies)
};

// Shared memory of one CTA. At a material interface face the left and the
// right cell see different fluxes; only the left cell's is stored, and the
// right cell's (NUMERICAL interface flux) is recomputed by that cell in the
// update phase, so the two-material kernel needs no second set of flux tiles.
template <typename T, int TY, bool MULTI>
struct StageSmemAll {
  StageSmem<T, TY> b;
};

// Value c of loaded cell (lx, ly) in ring slot sl.
#define M2C_VV(sl, c, ly, lx) sm.v[sl][c][ly][(lx) + 2]

// Resolve a possibly-outside index along one axis (at most two cells out).
// Returns the interior index to read; sets ghost side (-1 none, 0 low, 1 high)
// or far (outside by more than one cell, not periodic).
__device__ __forceinline__ int resolve_axis(int c, int n, bool periodic, int& side, bool& far) {
  side = -1;
  if (c >= 0 && c < n) return c;
  if (periodic) {
    int w = c < 0 ? c + n : c - n;
    if (w < 0) w += n;
    if (w >= n) w -= n;
    return w;
  }
  if (c == -1) { side = 0; return 0; }
  if (c == n) { side = 1; return n - 1; }
  far = true;
  return c < 0 ? 0 : n - 1;
}

__device__ __forceinline__ int wrap_index(int c, int n) {
  if (c < 0) c += n;
  if (c >= n) c -= n;
  if (c < 0) c += n;
  if (c >= n) c -= n;
  return c;
}

template <typename T> struct EosPick;
template <> struct EosPick<double> {
  __device__ static const Eos<double>& get(const SchemeK& s, int id) { return s.ed[id]; }
};
template <> struct EosPick<float> {
  __device__ static const Eos<float>& get(const SchemeK& s, int id) { return s.ef[id]; }
};

template <typename T, bool MULTI>
__device__ __forceinline__ const Eos<T>& eos_of(const SchemeK& s, int id) {
  return EosPick<T>::get(s, MULTI ? (id < s.nmat ? id : 0) : 0);
}

// Boundary face state built from the interior neighbour's face state
// (Reconstructor.cpp:822-875) followed by the clip check of
// CheckReconstructedStates on the ghost's inward face (3279-3318).
template <typename T>
__device__ __forceinline__ void ghost_face(int bc, int axis, const T* inner_face, const T* ghost_cell,
                                           const Eos<T>& e, T* out) {
  if (bc == BC_INLET || bc == BC_OUTLET) {
#pragma unroll
    for (int p = 0; p < 5; p++) out[p] = ghost_cell[p];
  } else {
#pragma unroll
    for (int p = 0; p < 5; p++) out[p] = inner_face[p];
    if (bc == BC_STICKWALL) {
      out[1] = -out[1]; out[2] = -out[2]; out[3] = -out[3];
    } else {
      if (axis == 0) out[1] = -out[1];
      else if (axis == 1) out[2] = -out[2];
      else out[3] = -out[3];
    }
  }
  if (e.needs_clip(out)) {
#pragma unroll
    for (int p = 0; p < 5; p++) out[p] = ghost_cell[p];
  }
}

template <typename T, int FLUX>
__device__ __forceinline__ int flux_of(const Eos<T>& e, int d, const T* VL, const T* VR, T delta, T* F) {
  if (FLUX == FLUX_HLLC) return flux_hllc(e, d, VL, VR, F);
  if (FLUX == FLUX_ROE) return flux_roe(e, d, VL, VR, delta, F);
  return flux_llf2(e, e, d, VL, VR, F);
}

// Asynchronous 8-byte global -> shared copy (cp.async, L1-allocating) and
// its completion wait; used to prefetch the next plane while the current one
// is being computed.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_t(T* smem, const T* gmem) {
  if constexpr (sizeof(T) == 8) cp_async8(smem, gmem);
  else cp_async4(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Resident CTAs per SM each instantiation is compiled for. The FP32 kernel
// runs 32 x 16 tiles, one 512-thread CTA per SM (126 registers); measured
// against 32 x 8 tiles at two CTAs per SM it is 2.5% faster on the 256^3 box
// (less halo work, same 16 warps), and 32 x 4 tiles at four CTAs per SM are
// 25% slower.
template <typename T> struct StageOcc { static constexpr int value = 1; };
#ifndef M2C_STAGE_OCC_F32
#define M2C_STAGE_OCC_F32 1
#endif
template <> struct StageOcc<float> { static constexpr int value = M2C_STAGE_OCC_F32; };

// CONS: reconstruction in conservative or characteristic variables (a
// separate instantiation so the primitive-variable kernels carry none of it).
// WALLS (two-material variant only): the branch of faces cut by an embedded
// surface is compiled in; without it the kernel carries none of its tests.
template <typename T, int TY, int FLUX, bool MULTI, bool CONS, bool WALLS = false>
__global__ void __launch_bounds__(TX * TY, StageOcc<T>::value) stage_kernel(const __grid_constant__ StageArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  typedef StageSmem<T, TY> S;
  typedef StageSmemAll<T, TY, MULTI> SA;
  SA& all = *reinterpret_cast<SA*>(smem_raw);
  S& sm = all.b;
  const Grid3& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  constexpr int NT = TX * TY;
  constexpr int NLOAD = S::RY * S::RX;
  constexpr int LPT = (NLOAD + NT - 1) / NT;  // loaded cells per thread
  const bool xper = g.bc[0] == BC_PERIODIC, yper = g.bc[2] == BC_PERIODIC, zper = g.bc[4] == BC_PERIODIC;
  const double dt = a.clock[1];
  const double bdt = a.bdt_coef * dt;
  const bool us_clip = (a.stage > 1) && a.us_clipped && *a.us_clipped;
  const T alpha = T(a.s.alpha), delta = T(a.s.delta);
  const int where = a.stage * 16;
  const int limiter = a.s.limiter;
  const bool rec_linear = a.s.rec_linear;
  const bool slope_zero = MULTI && a.s.slope_zero_at_interface;

  int i0 = 0, j0 = 0;  // tile origin of the current work item
  uint8_t idreg[LPT];
  // Plane copies: tensor copies unless x or y is periodic (CTA-uniform).
  const bool use_tma = a.use_tma != 0;
  constexpr unsigned TMA_BYTES = 5u * S::RY * S::BX * sizeof(T);
  unsigned tma_phase = 0;  // bit s: parity of the next completion of slot s's mbarrier
  if (use_tma) {
    if (tid == 0) {
      for (int q = 0; q < 4; q++) {
        const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.bar[q]);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&a.tin)) : "memory");
    }
    __syncthreads();
  }

  auto slot4 = [](int p) { return p & 3; };
  auto plane_is_ghost = [&](int p) { return !zper && (p < 0 || p >= g.nz); };

  // Per tile, for each loaded cell of this thread: its in-plane offset (the
  // image cell for ghosts, the wrapped cell for periodic halos) and its kind
  // in x and y: bits 0-1 x ghost side + 1 (0 none, 1 low, 2 high), bits 2-3
  // the same for y, bit 4 far (outside by more than one cell, not periodic).
  int xyoff[LPT];
  uint8_t xyinfo[LPT];
  auto tile_setup = [&]() {
#pragma unroll
    for (int r = 0; r < LPT; r++) {
      const int q = tid + r * NT;
      if (q >= NLOAD) break;
      const int ly = q / S::RX, lx = q - ly * S::RX;
      int sx, sy;
      bool far = false;
      const int ii = resolve_axis(i0 + lx - 2, g.nx, xper, sx, far);
      const int jj = resolve_axis(j0 + ly - 2, g.ny, yper, sy, far);
      xyoff[r] = jj * (int)g.px + ii;
      xyinfo[r] = uint8_t((sx + 1) | ((sy + 1) << 2) | (far ? 16 : 0));
    }
  };

  // (1a) start copying plane p into its ring slot. Tensor path: one thread
  // issues the plane's copy (all components) against the slot's mbarrier,
  // after a proxy fence orders the slot's earlier generic accesses (every
  // thread passed a barrier since) before the asynchronous write. Element
  // path (periodic x or y): one cp.async per value from the image or
  // wrapped position.
  auto issue_plane = [&](int p) {
    int sz;
    bool farz = false;
    const int kk = resolve_axis(p, g.nz, zper, sz, farz);
    const int s = slot4(p);
    if (use_tma) {
      if (tid == 0) {
        const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.bar[s]);
        const unsigned dst = (unsigned)__cvta_generic_to_shared(&sm.v[s][0][0][0]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(TMA_BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
            "[%6];" ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(&a.tin)), "r"(i0 - 4), "r"(j0 - 2), "r"(kk),
            "r"(0), "r"(bar)
            : "memory");
      }
    } else {
#pragma unroll
      for (int r = 0; r < LPT; r++) {
        const int q = tid + r * NT;
        if (q >= NLOAD) break;
        const int ly = q / S::RX, lx = q - ly * S::RX;
        const long long off = (long long)kk * g.plane + xyoff[r];
#pragma unroll
        for (int c = 0; c < 5; c++) cp_async_t(&M2C_VV(s, c, ly, lx), static_cast<const T*>(a.Pin[c]) + off);
      }
      cp_async_commit();
    }
    if (MULTI) {
#pragma unroll
      for (int r = 0; r < LPT; r++) {
        const int q = tid + r * NT;
        if (q >= NLOAD) break;
        idreg[r] = a.id[(long long)kk * g.plane + xyoff[r]];
      }
    }
  };

  // (1b) wait for plane p, then a CTA barrier (which also keeps the plane's
  // commit from overwriting ids and kinds the previous iteration's update
  // still reads). Tensor path: every thread polls the slot's mbarrier
  // (bounded; a copy that never lands is reported and the CTA stops).
  auto wait_plane = [&](int p) -> bool {
    if (!use_tma) {
      cp_async_wait_all();
      __syncthreads();
      return true;
    }
    const int s = slot4(p);
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.bar[s]);
    const unsigned parity = (tma_phase >> s) & 1u;
    unsigned ok = 0;
    for (int it = 0; it < STAGE_TMA_POLLS && !ok; it++) {
      asm volatile(
          "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}"
          : "=r"(ok)
          : "r"(bar), "r"(parity)
          : "memory");
    }
    tma_phase ^= 1u << s;
    if (!ok) report(a.err, ERR_ITER_CAP, -1, where + 5);
    __syncthreads();
    return ok != 0;
  };

  // (1c) the landed plane: boundary rule on ghost cells
  // (SpaceOperator::ApplyBoundaryConditions), cell kinds and ids. A ghost
  // cell takes its image cell's value (the element path copied it there; the
  // tensor path reads it from the neighbour in x or y, or finds it in place
  // for a ghost plane in z), then the rule of its face.
  auto commit_plane = [&](int p) {
    const int s = slot4(p);
    int sz;
    bool farz = false;
    resolve_axis(p, g.nz, zper, sz, farz);
#pragma unroll
    for (int r = 0; r < LPT; r++) {
      const int q = tid + r * NT;
      if (q >= NLOAD) break;
      const int ly = q / S::RX, lx = q - ly * S::RX;
      const int gx = xyinfo[r] & 3, gy = (xyinfo[r] >> 2) & 3;
      const bool far = (xyinfo[r] & 16) || farz;
      const int nghost = (gx != 0) + (gy != 0) + (sz >= 0);
      const bool real = nghost == 0 && !far;
      if (nghost == 1 && !far) {
        const int axis = gx ? 0 : (gy ? 1 : 2);
        const int side = gx ? gx - 1 : (gy ? gy - 1 : sz);
        const int bc = g.bc[2 * axis + side];
        if (use_tma && axis < 2 && bc != BC_INLET && bc != BC_OUTLET) {
          const int ix = axis == 0 ? lx + (side ? -1 : 1) : lx, iy = axis == 1 ? ly + (side ? -1 : 1) : ly;
#pragma unroll
          for (int c = 0; c < 5; c++) M2C_VV(s, c, ly, lx) = M2C_VV(s, c, iy, ix);
        }
        if (bc == BC_INLET) {
#pragma unroll
          for (int c = 0; c < 5; c++) M2C_VV(s, c, ly, lx) = T(g.inlet[c]);
        } else if (bc == BC_OUTLET) {
#pragma unroll
          for (int c = 0; c < 5; c++) M2C_VV(s, c, ly, lx) = T(g.outlet[c]);
        } else if (bc == BC_STICKWALL) {
          M2C_VV(s, 1, ly, lx) = -M2C_VV(s, 1, ly, lx);
          M2C_VV(s, 2, ly, lx) = -M2C_VV(s, 2, ly, lx);
          M2C_VV(s, 3, ly, lx) = -M2C_VV(s, 3, ly, lx);
        } else {  // SYMMETRY / SLIPWALL: normal velocity flipped
          M2C_VV(s, 1 + axis, ly, lx) = -M2C_VV(s, 1 + axis, ly, lx);
        }
      }
      sm.real[s][ly][lx] = real ? 1 : 0;
      sm.ids[s][ly][lx] = MULTI ? idreg[r] : 0;
    }
    // order this thread's generic writes to the slot before the tensor copy
    // that refills it four planes later
    if (use_tma) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  };

  // Limiter coefficients (Reconstructor::Setup) of the cell at loaded
  // position (lx, ly) of plane p along axis d: the axis' constants on a
  // uniform axis, else its per-index arrays. The generalized minmod uses
  // C = B/(A+1) only (carried in B).
  auto limiter_coeffs = [&](int p, int lx, int ly, int d, T& A, T& B, int& K) {
    if (g.lu[d]) {
      if (limiter == LIM_VANALBADA) {
        A = T(g.lA0[d]); B = T(g.lB0[d]); K = g.lK0[d];
      } else {
        A = T(0); B = T(g.lC0[d]);
      }
      return;
    }
    const int ix = d == 0 ? wrap_index(i0 + lx - 2, g.nx) : (d == 1 ? wrap_index(j0 + ly - 2, g.ny)
                                                                    : wrap_index(p, g.nz));
    if (limiter == LIM_VANALBADA) {
      A = T(g.lA[d][ix]); B = T(g.lB[d][ix]); K = g.lK[d][ix];
    } else {
      A = T(0); B = T(g.lC[d][ix]);
    }
  };

  // Limited slopes in direction d of the real cell at loaded position
  // (lx, ly) of plane p (needs planes p-1, p, p+1 for d = 2).
  auto slopes = [&](int p, int lx, int ly, int d, T* sd) {
    const int s0 = slot4(p);
    int sm1 = s0, sp1 = s0, lxm = lx, lxp = lx, lym = ly, lyp = ly;
    if (d == 0) { lxm = lx - 1; lxp = lx + 1; }
    else if (d == 1) { lym = ly - 1; lyp = ly + 1; }
    else { sm1 = slot4(p - 1); sp1 = slot4(p + 1); }
    if (!rec_linear) {
#pragma unroll
      for (int c = 0; c < 5; c++) sd[c] = T(0);
      return;
    }
    T A, B;
    int K = 0;
    limiter_coeffs(p, lx, ly, d, A, B, K);
    bool zero = false;
    if (slope_zero) {
      const uint8_t id = sm.ids[s0][ly][lx];
      zero = id != sm.ids[sm1][lym][lxm] || id != sm.ids[sp1][lyp][lxp];
    }
    // no difference toward an inactive neighbour (Reconstructor.cpp:475-502)
    const bool offm = WALLS && sm.ids[sm1][lym][lxm] == a.s.nmat;
    const bool offp = WALLS && sm.ids[sp1][lyp][lxp] == a.s.nmat;
#pragma unroll
    for (int c = 0; c < 5; c++) {
      const T vc = M2C_VV(s0, c, ly, lx);
      const T dm = offm ? T(0) : vc - M2C_VV(sm1, c, lym, lxm);
      const T dp = offp ? T(0) : M2C_VV(sp1, c, lyp, lxp) - vc;
      T sl = limited_slope_c(limiter, A, B, K, alpha, dm, dp);
      sd[c] = zero ? T(0) : sl;
    }
  };

  // Limited slopes in direction d of the real cell at (lx, ly) of plane p in
  // the scheme's non-primitive variables (Reconstructor.cpp:397-404, 469-651):
  // differences of the conservative variables (rv 1, 3; neighbours converted
  // with their own EOS) or of the primitive ones (rv 2), projected on the
  // characteristic basis at the cell state (rv 2, 3) and limited there, then
  // mapped back. u is the cell's conservative state. Returns false where the
  // basis does not exist (c^2 < 0; the reference aborts).
  auto nonprim_slopes = [&](int p, int lx, int ly, int d, int rv, const Eos<T>& e, const T* v, const T* u,
                            T* sd) -> bool {
    const int s0 = slot4(p);
    int sm1 = s0, sp1 = s0, lxm = lx, lxp = lx, lym = ly, lyp = ly;
    if (d == 0) { lxm = lx - 1; lxp = lx + 1; }
    else if (d == 1) { lym = ly - 1; lyp = ly + 1; }
    else { sm1 = slot4(p - 1); sp1 = slot4(p + 1); }
    T A, B;
    int K = 0;
    limiter_coeffs(p, lx, ly, d, A, B, K);
    const uint8_t idm = sm.ids[sm1][lym][lxm], idp = sm.ids[sp1][lyp][lxp];
    bool zero = false;
    if (slope_zero) {
      const uint8_t id = sm.ids[s0][ly][lx];
      zero = id != idm || id != idp;
    }
    T qm[5], qp[5], dl[5], dr[5];
#pragma unroll
    for (int c = 0; c < 5; c++) {
      qm[c] = M2C_VV(sm1, c, lym, lxm);
      qp[c] = M2C_VV(sp1, c, lyp, lxp);
    }
    const bool uspace = rv != 2;
    if (uspace) {
      T t[5];
      eos_of<T, MULTI>(a.s, idm).p2c(qm, t);
#pragma unroll
      for (int c = 0; c < 5; c++) qm[c] = t[c];
      eos_of<T, MULTI>(a.s, idp).p2c(qp, t);
#pragma unroll
      for (int c = 0; c < 5; c++) qp[c] = t[c];
    }
    const T* q0 = uspace ? u : v;
    const bool offm = WALLS && idm == a.s.nmat, offp = WALLS && idp == a.s.nmat;  // Reconstructor.cpp:529-556
#pragma unroll
    for (int c = 0; c < 5; c++) {
      dl[c] = offm ? T(0) : q0[c] - qm[c];
      dr[c] = offp ? T(0) : qp[c] - q0[c];
    }
    bool ok = true;
    if (rv == 1) {
#pragma unroll
      for (int c = 0; c < 5; c++) sd[c] = limited_slope_c(limiter, A, B, K, alpha, dl[c], dr[c]);
    } else {
      CharBasis<T> cb;
      char_basis(e, d, v, cb);
      ok = cb.ok;
      T wl[5], wr[5], sw[5];
      if (rv == 2) {
        prim_to_char(cb, v, dl, wl);
        prim_to_char(cb, v, dr, wr);
      } else {
        char_rinv(cb, v, dl, wl);
        char_rinv(cb, v, dr, wr);
      }
#pragma unroll
      for (int c = 0; c < 5; c++) sw[c] = limited_slope_c(limiter, A, B, K, alpha, wl[c], wr[c]);
      if (rv == 2) char_to_prim(cb, v, sw, sd);
      else char_r(cb, v, sw, sd);
    }
    if (zero) {
#pragma unroll
      for (int c = 0; c < 5; c++) sd[c] = T(0);
    }
    return ok;
  };

  // (2) slopes and revert bits of the real cell at mask-region (mx, my) of
  // plane p. A cell of the tile (own) gets all three directions; a halo cell
  // only the direction dh (0: x, 1: y) across which the tile's faces read it
  // (x-halo cells feed only the tile's x faces, y-halo cells its y faces).
  // Its revert bits then follow the revert rule below for that direction's
  // two faces alone; the rule differs from the full cell's only where two
  // faces are non-physical, which the cell's own tile reports as an error.
  // Revert bits: bit 2d + side (0 minus face, 1 plus face), 0x40 for a
  // conservative-variable face state.
  auto mask_cell = [&](int p, int mx, int my, bool own, int dh) {
    const int s0 = slot4(p), ms = p & 1;
    const int ly = my + 1, lx = mx + 1;  // position in the loaded region
    if (!sm.real[s0][ly][lx]) {
      sm.mask[ms][my][mx] = 0;
      return;
    }
    const uint8_t id = sm.ids[s0][ly][lx];
    if (WALLS && id == a.s.nmat) {
      // inactive: constant reconstruction, no checks (Reconstructor.cpp:452-462,
      // SpaceOperator.cpp:3236-3237)
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int c = 0; c < 5; c++) sm.sig[ms][d][c][my][mx] = T(0);
      sm.mask[ms][my][mx] = 0;
      return;
    }
    const Eos<T>& e = eos_of<T, MULTI>(a.s, id);
    T v[5];
#pragma unroll
    for (int c = 0; c < 5; c++) v[c] = M2C_VV(s0, c, ly, lx);
    uint8_t m = 0;
    int err = ERR_NONE;
    bool cons = false;
    if (CONS && rec_linear) {
      // non-primitive variables; any non-physical face sends the cell back
      // to primitive variables (the RETRY of Reconstructor.cpp:719-775).
      // Halo cells take this path whole (the tile's cells and its halo ring).
      T sx[5], sy[5], sz[5];
      const int rv = a.s.rec_var;
      const bool uspace = rv != 2;
      T u[5];
      e.p2c(v, u);
      bool okb = nonprim_slopes(p, lx, ly, 0, rv, e, v, u, sx);
      okb = nonprim_slopes(p, lx, ly, 1, rv, e, v, u, sy) && okb;
      okb = nonprim_slopes(p, lx, ly, 2, rv, e, v, u, sz) && okb;
      if (!okb) err = ERR_SOUND;
      cons = true;
      uint8_t clipm = 0;
#pragma unroll
      for (int q = 0; q < 6; q++) {
        const T* sg = q < 2 ? sx : (q < 4 ? sy : sz);
        T f[5];
        if (uspace) {
          T uf[5];
#pragma unroll
          for (int c = 0; c < 5; c++) uf[c] = (q & 1) ? u[c] + T(0.5) * sg[c] : u[c] - T(0.5) * sg[c];
          e.c2p(uf, f);
        } else {
#pragma unroll
          for (int c = 0; c < 5; c++) f[c] = (q & 1) ? v[c] + T(0.5) * sg[c] : v[c] - T(0.5) * sg[c];
        }
        if (e.bad(f)) cons = false;
        else if (e.needs_clip(f)) clipm |= uint8_t(1u << q);  // SpaceOperator.cpp:3240-3273
      }
      if (cons) {
        m = uint8_t(clipm | (uspace ? 0x40 : 0));
#pragma unroll
        for (int c = 0; c < 5; c++) {
          sm.sig[ms][0][c][my][mx] = sx[c];
          sm.sig[ms][1][c][my][mx] = sy[c];
          sm.sig[ms][2][c][my][mx] = sz[c];
        }
      }
    }
    if (!cons) {
      // primitive slopes direction by direction, each direction's faces in
      // the reference's order (l, r, b, t, k, f)
      const int dlo = (own || CONS) ? 0 : dh, dhi = (own || CONS) ? 2 : dh;
      bool chain_done = false;
#pragma unroll 1
      for (int d = dlo; d <= dhi; d++) {
        T sd[5];
        slopes(p, lx, ly, d, sd);
#pragma unroll
        for (int c = 0; c < 5; c++) sm.sig[ms][d][c][my][mx] = sd[c];
#pragma unroll
        for (int side = 0; side < 2; side++) {
          T f[5];
#pragma unroll
          for (int c = 0; c < 5; c++) f[c] = side ? v[c] + T(0.5) * sd[c] : v[c] - T(0.5) * sd[c];
          const bool bad = e.bad(f);
          bool reverted = false;
          // Reconstructor.cpp:719-775: only the first non-physical face is reverted.
          if (!chain_done && bad) { reverted = true; chain_done = true; }
          // SpaceOperator.cpp:3240-3273: a face needing clipping reverts to the cell value.
          if (!reverted && e.needs_clip(f)) reverted = true;
          if (reverted) m |= uint8_t(1u << (2 * d + side));
          // SpaceOperator.cpp:3275-3277: a face still non-physical is fatal.
          else if (bad) err = ERR_STATE;
        }
      }
    }
    sm.mask[ms][my][mx] = m;
    if (err && (own || CONS)) {
      const int ka = wrap_index(p, g.nz);
      const int ia = wrap_index(i0 + mx - 1, g.nx), ja = wrap_index(j0 + my - 1, g.ny);
      report(a.err, err, (int)(((long long)ka * g.ny + ja) * g.nx + ia), where + 1);
    }
  };

  // Final face state of the real cell at mask-region (mx,my) of plane p:
  // direction d, side 0 = minus face (v - s/2), 1 = plus face (v + s/2).
  auto cell_face = [&](int p, int mx, int my, int d, int side, T* out) {
    const int s0 = slot4(p), ms = p & 1;
    const uint8_t mk = sm.mask[ms][my][mx];
    const bool rev = (mk >> (2 * d + side)) & 1u;
    if (CONS && (mk & 0x40)) {  // conservative-variable face state
      T v[5], u[5], uf[5];
#pragma unroll
      for (int c = 0; c < 5; c++) v[c] = M2C_VV(s0, c, my + 1, mx + 1);
      if (rev) {
#pragma unroll
        for (int c = 0; c < 5; c++) out[c] = v[c];
        return;
      }
      const Eos<T>& e = eos_of<T, MULTI>(a.s, sm.ids[s0][my + 1][mx + 1]);
      e.p2c(v, u);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        const T sd = sm.sig[ms][d][c][my][mx];
        uf[c] = side ? u[c] + T(0.5) * sd : u[c] - T(0.5) * sd;
      }
      e.c2p(uf, out);
      return;
    }
#pragma unroll
    for (int c = 0; c < 5; c++) {
      const T v = M2C_VV(s0, c, my + 1, mx + 1);
      const T sd = sm.sig[ms][d][c][my][mx];
      out[c] = rev ? v : (side ? v + T(0.5) * sd : v - T(0.5) * sd);
    }
  };

  // (3) flux across the face between mask-region cells L (plane pL) and
  // R = L + e_d (plane pR): the flux seen by the left cell (F). F2 (the right
  // cell's) equals F except at NUMERICAL interface faces, where the update
  // phase forms it.
  auto face_flux = [&](int d, int pL, int mxL, int myL, int pR, int mxR, int myR, T* F, T* F2) {
    const int sL = slot4(pL), sR = slot4(pR);
    const bool rL = sm.real[sL][myL + 1][mxL + 1], rR = sm.real[sR][myR + 1][mxR + 1];
    if (!rL && !rR) {
#pragma unroll
      for (int c = 0; c < 5; c++) { F[c] = T(0); F2[c] = T(0); }
      return;
    }
    T VL[5], VR[5];
    const uint8_t idL = sm.ids[sL][myL + 1][mxL + 1], idR = sm.ids[sR][myR + 1][mxR + 1];
    // a face cut by an embedded surface (interior faces only) takes the wall
    // branch, which the reference tests before the material-interface one
    bool wall = false;
    long long offW = 0;
    if (WALLS && rL && rR) {
      const int gi = wrap_index(i0 + mxR - 1, g.nx), gj = wrap_index(j0 + myR - 1, g.ny);
      offW = (long long)wrap_index(pR, g.nz) * g.plane + (long long)gj * g.px + gi;
      wall = (a.wall.mask[offW] >> d) & 1;
    }
    // face pass: only the faces whose states a pre-pass solves from
    const bool fp_iface = MULTI && a.iface.faces_out && idL != idR;
    const bool fp_wall = WALLS && a.wall.faces_out && wall;
    if (MULTI && (a.iface.faces_out || (WALLS && a.wall.faces_out)) && !fp_iface && !fp_wall) {
#pragma unroll
      for (int c = 0; c < 5; c++) { F[c] = T(0); F2[c] = T(0); }
      return;
    }
    if (rL) cell_face(pL, mxL, myL, d, 1, VL);
    if (rR) cell_face(pR, mxR, myR, d, 0, VR);
    if (!rL) {  // low-side boundary face
      T gc[5];
#pragma unroll
      for (int c = 0; c < 5; c++) gc[c] = M2C_VV(sL, c, myL + 1, mxL + 1);
      ghost_face(g.bc[2 * d], d, VR, gc, eos_of<T, MULTI>(a.s, idL), VL);
    }
    if (!rR) {  // high-side boundary face
      T gc[5];
#pragma unroll
      for (int c = 0; c < 5; c++) gc[c] = M2C_VV(sR, c, myR + 1, mxR + 1);
      ghost_face(g.bc[2 * d + 1], d, VL, gc, eos_of<T, MULTI>(a.s, idR), VR);
    }
    int err = ERR_NONE;
    if (fp_iface || fp_wall) {  // face pass: the interface or cut faces' states only
#pragma unroll
      for (int c = 0; c < 5; c++) { F[c] = T(0); F2[c] = T(0); }
      const int gi = wrap_index(i0 + mxR - 1, g.nx), gj = wrap_index(j0 + myR - 1, g.ny);
      const int gk = wrap_index(pR, g.nz);
      const long long offR = (long long)gk * g.plane + (long long)gj * g.px + gi;
      for (int q = 0; q < 2; q++) {
        if (q == 0 ? !fp_iface : !fp_wall) continue;
        const int slot = q == 0 ? a.iface.slot[offR] : a.wall.slot[offR];
        double* o = (q == 0 ? a.iface.faces_out : a.wall.faces_out) + ((long long)slot * 3 + d) * 10;
#pragma unroll
        for (int c = 0; c < 5; c++) {
          o[c] = double(VL[c]);
          o[5 + c] = double(VR[c]);
        }
      }
      return;
    }
    if (WALLS && (idL == a.s.nmat || idR == a.s.nmat) && !(wall && idL != a.s.nmat)) {
      // an inactive side gets no flux, and a face with an inactive cell that
      // no surface cuts carries none (SpaceOperator.cpp:2441-2483, 2537-2551);
      // the right cell of a cut face forms its own flux in its update
#pragma unroll
      for (int c = 0; c < 5; c++) { F[c] = T(0); F2[c] = T(0); }
      return;
    }
    if (MULTI && (wall || idL != idR)) {
      // Material interface (SpaceOperator.cpp:2486-2542): two one-sided fluxes
      // against the exact Riemann star states, or LLF across the interface.
      // Wall (2438-2484, CONSTANT reconstruction at the wall): the left
      // cell's flux against its one-sided star state.
      const IfaceView& iv = a.iface;
      T WL[5], WR[5];
      if (wall ? !a.wall.linear : iv.mp_recon == 0) {  // constant reconstruction: cell-centred states
#pragma unroll
        for (int c = 0; c < 5; c++) {
          WL[c] = M2C_VV(sL, c, myL + 1, mxL + 1);
          WR[c] = M2C_VV(sR, c, myR + 1, mxR + 1);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 5; c++) { WL[c] = VL[c]; WR[c] = VR[c]; }
      }
      if (!wall && iv.mp_flux == 2) {
        err = flux_llf2(eos_of<T, MULTI>(a.s, idL), eos_of<T, MULTI>(a.s, idR), d, WL, WR, F);
#pragma unroll
        for (int c = 0; c < 5; c++) F2[c] = F[c];
      } else {
        // the right cell's index carries the slot of its low faces
        const int gi = wrap_index(i0 + mxR - 1, g.nx), gj = wrap_index(j0 + myR - 1, g.ny);
        const int gk = wrap_index(pR, g.nz);
        const int slot = wall ? a.wall.slot[offW] : iv.slot[(long long)gk * g.plane + (long long)gj * g.px + gi];
        const long long base = ((long long)slot * 3 + d) * 5;
        if (!wall && iv.mp_flux == 0) {  // Godunov flux of the state at xi = 0
          T Vm[5];
#pragma unroll
          for (int c = 0; c < 5; c++) Vm[c] = T(iv.Vmid[base + c]);
          phys_flux(eos_of<T, MULTI>(a.s, iv.midid[slot * 3 + d]), d, Vm, F);
#pragma unroll
          for (int c = 0; c < 5; c++) F2[c] = F[c];
        } else {
          const double* src = wall ? a.wall.Vsm : iv.Vsm;
          T Sm[5];
#pragma unroll
          for (int c = 0; c < 5; c++) Sm[c] = T(src[base + c]);
          // the right cell's flux against its own star state is formed in its update
          err = flux_of<T, FLUX>(eos_of<T, MULTI>(a.s, idL), d, WL, Sm, delta, F);
        }
      }
    } else {
      // same material: flux with the right cell's EOS, as the reference's
      // face loop does (myid = id of the right cell)
      err = flux_of<T, FLUX>(eos_of<T, MULTI>(a.s, rR ? idR : idL), d, VL, VR, delta, F);
#pragma unroll
      for (int c = 0; c < 5; c++) F2[c] = F[c];
    }
    if (err) report(a.err, err, -1, where + 2);
  };

  // (3a) the faces of plane m owned by this thread: the x face left of its
  // cell, the y face below it (if do_xy) and the z face m+1/2 above it; one
  // call site, so the flux code is inlined once.
  auto faces = [&](int m, bool do_xy) {
    const int zs = (m + 1) & 1;
#pragma unroll 1
    for (int k = do_xy ? 0 : 2; k < 3; k++) {
      const int d = k;
      const int mxL = k == 0 ? tx : tx + 1, myL = k == 1 ? ty : ty + 1;
      const int pR = k == 2 ? m + 1 : m;
      T* dst = k == 0 ? &sm.fx[0][ty * (TX + 1) + tx] : (k == 1 ? &sm.fy[0][ty * TX + tx] : &sm.fz[zs][0][ty * TX + tx]);
      const int stride = k == 0 ? S::NFX : (k == 1 ? S::NFY : S::NFZ);
      T F[5], F2[5];
      face_flux(d, m, mxL, myL, pR, tx + 1, ty + 1, F, F2);
#pragma unroll
      for (int c = 0; c < 5; c++) dst[c * stride] = F[c];
    }
  };

  // (2) + (3b) one phase: slopes and revert bits of plane p (do_mask): the
  // tile's cells, one per thread, then the halo cells in their single
  // direction; and the tile's right x faces and top y faces of plane mf
  // (do_bf), whose cells' slopes are complete since the previous plane.
  // Spreading the halo cells and those faces over the threads that have no
  // second item keeps the phase at about one cell and a third per thread.
  auto mask_and_edge_faces = [&](int p, bool do_mask, int mf, bool do_bf) {
    constexpr int NH = CONS ? S::MX * S::MY - NT : 2 * (TX + TY);  // halo items
    constexpr int NB = TX + TY;                                     // edge faces
    for (int q = tid; q < NT + NH + NB; q += NT) {
      if (q < NT + NH) {
        if (!do_mask) continue;
        const int r = q - NT;
        int mx = tx + 1, my = ty + 1, dh = 0;
        if (r < 0) {
          // a cell of the tile
        } else if (CONS) {  // the ring of the mask region: bottom row, top row, then the two side columns
          if (r < S::MX) { mx = r; my = 0; }
          else if (r < 2 * S::MX) { mx = r - S::MX; my = S::MY - 1; }
          else { const int r2 = r - 2 * S::MX; mx = (r2 & 1) ? S::MX - 1 : 0; my = 1 + (r2 >> 1); }
        } else if (r < 2 * TY) {  // x-halo columns (mx = 0, TX + 1)
          mx = r < TY ? 0 : TX + 1;
          my = (r < TY ? r : r - TY) + 1;
        } else {                  // y-halo rows (my = 0, TY + 1)
          const int r2 = r - 2 * TY;
          mx = (r2 < TX ? r2 : r2 - TX) + 1;
          my = r2 < TX ? 0 : TY + 1;
          dh = 1;
        }
        mask_cell(p, mx, my, r < 0, dh);
      } else {
        if (!do_bf) continue;
        const int r = q - NT - NH;
        const bool xf = r < TY;  // x face right of the tile's last column (row r), else
                                 // y face above its top row (column r - TY)
        const int fx = r - TY;
        T F[5], F2[5];
        face_flux(xf ? 0 : 1, mf, xf ? TX : fx + 1, xf ? r + 1 : TY, mf, xf ? TX + 1 : fx + 1, xf ? r + 1 : TY + 1, F,
                  F2);
        T* dst = xf ? &sm.fx[0][r * (TX + 1) + TX] : &sm.fy[0][TY * TX + fx];
        const int stride = xf ? S::NFX : S::NFY;
#pragma unroll
        for (int c = 0; c < 5; c++) dst[c * stride] = F[c];
      }
    }
  };

  double dtmin_local = 1.0e300;
  int clipped_local = 0;
  const int tiles = a.ntx * a.nty;

  // Balanced segments: the (tile, plane) units, ordered tile by tile and
  // plane by plane within a tile, are split evenly over the CTAs; a CTA runs
  // the plane pipeline over each tile segment of its share (at most a few).
  const long long units = (long long)tiles * g.nz;
  const long long ubeg = units * blockIdx.x / gridDim.x, uend = units * (blockIdx.x + 1) / gridDim.x;
  for (long long u = ubeg; u < uend;) {
    const int t2 = (int)(u / g.nz);
    const int kb = (int)(u - (long long)t2 * g.nz);
    const int ke = (int)min((long long)g.nz, kb + (uend - u));
    u += ke - kb;
    const int tyi = t2 / a.ntx, txi = t2 - tyi * a.ntx;
    i0 = txi * TX;
    j0 = tyi * TY;
    const int gi = i0 + tx, gj = j0 + ty;
    const bool own = gi < g.nx && gj < g.ny;
    double dxi = 0, dyj = 0;
    if (own) { dxi = g.dx[gi]; dyj = g.dy[gj]; }

    // pipeline prologue: planes kb-2 and kb-1 committed, plane kb in flight
    // (a plane copy that never lands stops the CTA, all threads together)
    tile_setup();
    __syncthreads();
    issue_plane(kb - 2);
    bool landed = wait_plane(kb - 2);
    commit_plane(kb - 2);
    if (__syncthreads_or(!landed)) return;
    issue_plane(kb - 1);
    landed = wait_plane(kb - 1);
    commit_plane(kb - 1);
    if (__syncthreads_or(!landed)) return;
    issue_plane(kb);
    for (int m = kb - 2; m < ke; m++) {
      landed = wait_plane(m + 2);
      commit_plane(m + 2);
      if (__syncthreads_or(!landed)) return;
      if (m + 3 <= ke + 1) issue_plane(m + 3);  // in flight during the work below
      if (m >= kb && own) {  // the update's FP64 inputs of plane m into L1 while the faces are computed
        const long long offp = (long long)m * g.plane + (long long)gj * g.px + gi;
#pragma unroll
        for (int c = 0; c < 5; c++) asm volatile("prefetch.global.L1 [%0];" ::"l"(a.Vn[c] + offp));
        if (a.stage != 1) {
#pragma unroll
          for (int c = 0; c < 5; c++) asm volatile("prefetch.global.L1 [%0];" ::"l"(a.Us[c] + offp));
        }
      }
      mask_and_edge_faces(m + 1, m + 1 >= kb - 1 && !plane_is_ghost(m + 1), m, m >= kb);
      __syncthreads();
      if (m >= kb - 1) faces(m, m >= kb);
      __syncthreads();
      if (m < kb || !own || (MULTI && (a.iface.faces_out || (WALLS && a.wall.faces_out)))) continue;
      // (4) residual + RK update of plane m
      const double dzk = g.dz[m];
      const double ax = dyj * dzk, ay = dxi * dzk, az = dxi * dyj;
      const float axf = float(ax), ayf = float(ay), azf = float(az);
      const double vol = dxi * dyj * dzk;
      // Vec5D::operator/= multiplies by the reciprocal (Vector5D.h:172-181)
      const double inv_mvol = 1.0 / (-vol);
      const long long off = (long long)m * g.plane + (long long)gj * g.px + gi;
      const uint8_t id = MULTI ? a.id[off] : 0;
      if (WALLS && id == a.s.nmat) {
        // inactive: no residual (every face gives it a zero flux), and
        // VarFcnDummy's fixed states after every stage (VarFcnDummy.h:44-57)
        if (a.Ro[0]) {
#pragma unroll
          for (int c = 0; c < 5; c++) a.Ro[c][off] = 0.0 * inv_mvol;
          continue;
        }
        const double Vd[5] = {a.s.dummy[0], 0.0, 0.0, 0.0, a.s.dummy[1]};
        if (a.final_stage) {
#pragma unroll
          for (int c = 0; c < 5; c++) a.Vo[c][off] = Vd[c];
          if (a.Vfo[0]) {
#pragma unroll
            for (int c = 0; c < 5; c++) a.Vfo[c][off] = float(Vd[c]);
          }
        } else {
          const double Ud[5] = {a.s.dummy[0], 0.0, 0.0, 0.0, a.s.dummy[0] * a.s.dummy[2]};
#pragma unroll
          for (int c = 0; c < 5; c++) {
            a.Uo[c][off] = Ud[c];
            static_cast<T*>(a.Po[c])[off] = T(Vd[c]);
          }
        }
        continue;
      }
      const Eos<double>& e = eos_of<double, MULTI>(a.s, id);
      double Un[5], Unew[5], Vn[5];
#pragma unroll
      for (int c = 0; c < 5; c++) Vn[c] = a.Vn[c][off];
      e.p2c(Vn, Un);
      if (a.stage == 1) {
#pragma unroll
        for (int c = 0; c < 5; c++) Unew[c] = Un[c];
      } else {
        double Us[5];
#pragma unroll
        for (int c = 0; c < 5; c++) Us[c] = a.Us[c][off];
        if (us_clip) {
          double Vs[5];
          e.c2p(Us, Vs);
          e.clip(Vs);
          e.p2c(Vs, Us);
        }
#pragma unroll
        for (int c = 0; c < 5; c++) Unew[c] = a.a_prev * Us[c] + a.a_un * Un[c];
      }
      const int fxl = ty * (TX + 1) + tx, fyl = ty * TX + tx, fzc = ty * TX + tx;
      const int zl = m & 1, zr = (m + 1) & 1;
      // Low faces that are material interfaces under the NUMERICAL interface
      // flux: this cell's flux is its EOS's numerical flux between the right
      // star state and its own cell-centred state (SpaceOperator.cpp:2499-2542).
      // Low faces cut by an embedded surface likewise take this cell's flux
      // against its one-sided star state (SpaceOperator.cpp:2462-2478).
      T F2[3][5];
      bool ifc[3] = {false, false, false};
      if constexpr (MULTI) {
        const uint8_t wm = WALLS ? a.wall.mask[off] : 0;
        const bool num = a.iface.mp_flux == 1;  // set only with interface slots (two-material contexts)
        if (num || wm) {
          const int sc = slot4(m), lx = tx + 2, ly = ty + 2;
          const uint8_t me = sm.ids[sc][ly][lx];
          ifc[0] = (wm & 1) || (num && me != sm.ids[sc][ly][lx - 1]);
          ifc[1] = (wm & 2) || (num && me != sm.ids[sc][ly - 1][lx]);
          ifc[2] = (wm & 4) || (num && me != sm.ids[slot4(m - 1)][ly][lx]);
          if (ifc[0] || ifc[1] || ifc[2]) {
            const int islot = num ? a.iface.slot[off] : 0;
            const int wslot = wm ? a.wall.slot[off] : 0;
            for (int d = 0; d < 3; d++) {
              if (!ifc[d]) continue;
              const bool w = (wm >> d) & 1;
              // this cell's side of the face: its cell-centred state, or its
              // reconstructed state on that face (vl) under LINEAR interface
              // reconstruction
              T W[5];
              if (w ? a.wall.linear : a.iface.mp_recon) {
                cell_face(m, tx + 1, ty + 1, d, 0, W);
              } else {
#pragma unroll
                for (int c = 0; c < 5; c++) W[c] = M2C_VV(sc, c, ly, lx);
              }
              const long long base = ((long long)(w ? wslot : islot) * 3 + d) * 5;
              const double* src = w ? a.wall.Vsp : a.iface.Vsp;
              T Sp[5];
#pragma unroll
              for (int c = 0; c < 5; c++) Sp[c] = T(src[base + c]);
              const int err2 = flux_of<T, FLUX>(eos_of<T, MULTI>(a.s, me), d, Sp, W, delta, F2[d]);
              if (err2) report(a.err, err2, -1, where + 2);
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 5; c++) {
        // low faces: the flux this cell sees as the right-hand cell
        // (SpaceOperator.cpp:2555-2556, 2683-2684, 2810-2811)
        const T fl = ifc[0] ? F2[0][c] : sm.fx[c][fxl];
        const T gl = ifc[1] ? F2[1][c] : sm.fy[c][fyl];
        const T hl = ifc[2] ? F2[2][c] : sm.fz[zl][c][fzc];
        double f;
        if constexpr (sizeof(T) == 8) {
          // FP64: the reference's order, 0 - Fl A - Gl A - Hl A + Fr A + Gr A + Hr A
          f = 0.0;
          f = f - fl * ax;
          f = f - gl * ay;
          f = f - hl * az;
          f = f + double(sm.fx[c][fxl + 1]) * ax;
          f = f + double(sm.fy[c][fyl + TX]) * ay;
          f = f + double(sm.fz[zr][c][fzc]) * az;
        } else {
          // mixed: FP32 accumulation of the flux differences (the difference
          // of two nearby FP32 fluxes is exact), one conversion per component
          f = double((sm.fx[c][fxl + 1] - fl) * axf + (sm.fy[c][fyl + TX] - gl) * ayf +
                     (sm.fz[zr][c][fzc] - hl) * azf);
        }
        if (a.visc.fr[0]) {
          // viscous fluxes (ViscosityOperator::AddDiffusionFluxes), added to
          // the flux sum in its cell order: this cell's low x, y, z faces,
          // then the low faces of its +x, +y, +z neighbours
          if (c == 0) {
            f = f + 0.0; f = f + 0.0; f = f + 0.0;
            f = f - 0.0; f = f - 0.0; f = f - 0.0;
          } else {
            const long long S = a.visc.nf[0], cc = (long long)(c - 1) * S;
            const long long fxi = ((long long)m * g.ny + gj) * (g.nx + 1) + gi;
            const long long fyi = ((long long)m * (g.ny + 1) + gj) * g.nx + gi;
            const long long fzi = ((long long)m * g.ny + gj) * g.nx + gi;
            f = f + a.visc.fr[0][cc + fxi];
            f = f + a.visc.fr[1][cc + fyi];
            f = f + a.visc.fr[2][cc + fzi];
            f = f - a.visc.fl[0][cc + fxi + 1];
            f = f - a.visc.fl[1][cc + fyi + g.nx];
            f = f - a.visc.fl[2][cc + fzi + (long long)g.ny * g.nx];
          }
        }
        if (c == 4 && a.visc.fh[0]) {
          // heat fluxes (HeatDiffusionOperator::AddDiffusionFluxes, after the
          // viscous ones), energy only, in the same cell order
          const long long fxi = ((long long)m * g.ny + gj) * (g.nx + 1) + gi;
          const long long fyi = ((long long)m * (g.ny + 1) + gj) * g.nx + gi;
          const long long fzi = ((long long)m * g.ny + gj) * g.nx + gi;
          f = f + a.visc.fh[0][fxi];
          f = f + a.visc.fh[1][fyi];
          f = f + a.visc.fh[2][fzi];
          f = f - a.visc.fh[0][fxi + 1];
          f = f - a.visc.fh[1][fyi + g.nx];
          f = f - a.visc.fh[2][fzi + (long long)g.ny * g.nx];
        }
        const double R = f * inv_mvol;
        if (a.Ro[0]) a.Ro[c][off] = R;
        Unew[c] = Unew[c] + bdt * R;
      }
      if (a.Ro[0]) continue;
      double V[5];
      e.c2p(Unew, V);
      const bool clipped = e.clip(V);
      clipped_local |= clipped ? 1 : 0;
      if (e.bad(V)) report(a.err, ERR_STATE, (int)((long long)m * g.ny * g.nx + (long long)gj * g.nx + gi), where + 3);
      if (a.final_stage) {
#pragma unroll
        for (int c = 0; c < 5; c++) a.Vo[c][off] = V[c];
        if (a.Vfo[0]) {
#pragma unroll
          for (int c = 0; c < 5; c++) a.Vfo[c][off] = float(V[c]);
        }
        const double ee = e.energy(V[0], V[4]);
        const double c2 = e.c2(V[0], ee);
        if (c2 < 0.0) report(a.err, ERR_SOUND, (int)off, where + 4);
        const double cs = sqrt(c2);
        const double lx = fabs(V[1]) + cs, ly = fabs(V[2]) + cs, lz = fabs(V[3]) + cs;
        const double r = smin(dxi / lx, smin(dyj / ly, dzk / lz));
        dtmin_local = smin(dtmin_local, r);
      } else {
#pragma unroll
        for (int c = 0; c < 5; c++) a.Uo[c][off] = Unew[c];
        // the next stage's input: clip(C2P(U_new)), as it would recompute it
#pragma unroll
        for (int c = 0; c < 5; c++) static_cast<T*>(a.Po[c])[off] = T(V[c]);
      }
    }
  }

  if (a.clipped_out && __syncthreads_or(clipped_local)) {
    if (tid == 0) atomicOr(a.clipped_out, 1);
  }
  if (a.final_stage && a.dtmin_bits) {
    double v = dtmin_local;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (tx == 0) sm.red[ty] = v;
    __syncthreads();
    if (tid == 0) {
      double r = sm.red[0];
      for (int q = 1; q < TY; q++) r = smin(r, sm.red[q]);
      if (r < 1.0e300) atomicMin(a.dtmin_bits, (unsigned long long)__double_as_longlong(r));
    }
  }
}

}  // namespace m2c
