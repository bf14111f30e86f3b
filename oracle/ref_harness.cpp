/*
 * CPU oracle driver around the UNMODIFIED reference M2C sources.
 *
 * TEST INFRASTRUCTURE ONLY: this file is compiled together with the reference
 * sources (taken in place from the reference tree by oracle/Makefile, never
 * copied into this repository) and the single-rank MPI/PETSc shims in
 * oracle/ref_shim into oracle/_ref/libm2c_ref.so. Only tests, smoke() and the
 * CPU-baseline legs of bench.py load it, as the checker.
 *
 * It mirrors the set-up and time loop of the reference driver
 * (Main.cpp:106-379 object construction, Main.cpp:514-575 time loop) with
 * the configuration coming from the m2cg_* structs instead of an input file,
 * and exposes an extern "C" API over it. State arrays use the reference's
 * own ghosted local-vector layout [k][j][i][dof] with ghost indices -1..N.
 */
#include <IoData.h>
#include <VarFcnSG.h>
#include <VarFcnNASG.h>
#include <VarFcnDummy.h>
#include <FluxFcnGenRoe.h>
#include <FluxFcnLLF.h>
#include <FluxFcnHLLC.h>
#include <ExactRiemannSolverBase.h>
#include <MeshGenerator.h>
#include <GlobalMeshInfo.h>
#include <SpaceVariable.h>
#include <SpaceOperator.h>
#include <LevelSetOperator.h>
#include <MultiPhaseOperator.h>
#include <TimeIntegrator.h>
#include <Utils.h>
#include <Interpolator.h>
#include <GradientCalculatorCentral.h>
#include <EmbeddedBoundaryDataSet.h>
#include <TriangulatedSurface.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/m2c_gpu.h"
#ifdef M2C_DROPIN
// The drop-in build: the same driver with M2C's RK integrator replaced by
// the GPU one a maintainer would add (m2c_b200/adapter/TimeIntegratorGPU.h).
#include "m2c_b200/adapter/TimeIntegratorGPU.h"
#endif

// Globals the reference expects from its driver (Main.cpp:39-44).
int verbose = 0;
double domain_diagonal = 0.0;
clock_t start_time;
MPI_Comm m2c_comm = 0;
int INACTIVE_MATERIAL_ID = 0;

namespace {

struct RefCase {
  MPI_Comm comm = 0;
  IoData iod;
  std::vector<VarFcnBase*> vf;
  ExactRiemannSolverBase* riemann = nullptr;
  FluxFcnBase* ff = nullptr;
  GlobalMeshInfo* gmi = nullptr;
  DataManagers3D* dms = nullptr;
  SpaceOperator* spo = nullptr;
  std::vector<LevelSetOperator*> lso;
  std::vector<SpaceVariable3D*> Phi;
  MultiPhaseOperator* mpo = nullptr;
  TimeIntegratorBase* integrator = nullptr;
  SpaceVariable3D* V = nullptr;
  SpaceVariable3D* ID = nullptr;
  InterpolatorLinear* interp = nullptr;         // viscous fluxes (Main.cpp:195-205)
  GradientCalculatorCentral* grad = nullptr;
  int NX = 0, NY = 0, NZ = 0;
  double t = 0.0;
  int time_step = 0;
  double advance_seconds = 0.0;  // wall time inside dt + AdvanceOneTimeStep
};

MeshData::BcType to_bc(int b) { return (MeshData::BcType)b; }

void fill_material(MaterialModelData* d, const m2cg_material& m) {
  d->eos = m.eos == M2CG_EOS_NASG ? MaterialModelData::NOBLE_ABEL_STIFFENED_GAS
                                  : MaterialModelData::STIFFENED_GAS;
  d->rhomin = m.rhomin;
  d->pmin = m.pmin;
  d->rhomax = m.rhomax;
  d->pmax = m.pmax;
  d->failsafe_density = m.failsafe_density;
  d->sgModel.specificHeatRatio = m.gamma;
  d->sgModel.pressureConstant = m.p_c;
  d->nasgModel.specificHeatRatio = m.gamma;
  d->nasgModel.pressureConstant = m.p_c;
  d->nasgModel.volumeConstant = m.b;
  d->nasgModel.energyConstant = m.q;
  d->sgModel.cv = m.cv;
  d->sgModel.T0 = m.T0;
  d->sgModel.e0 = m.e0;
  d->sgModel.cp = m.cp;
  d->sgModel.h0 = m.h0;
  d->nasgModel.cv = m.cv;
  if (m.heat_diffusivity != 0.0) {
    d->heat_diffusion.type = HeatDiffusionModelData::CONSTANT;
    d->heat_diffusion.diffusivity = m.heat_diffusivity;
  }
  if (m.mu != 0.0 || m.mu_bulk != 0.0) {
    d->viscosity.type = ViscosityModelData::CONSTANT;
    d->viscosity.dynamicViscosity = m.mu;
    d->viscosity.bulkViscosity = m.mu_bulk;
  }
}

void fill_scheme(IoData& iod, const m2cg_scheme& s) {
  iod.schemes.ns.flux = (SchemeData::Flux)s.flux;
  iod.schemes.ns.delta = s.roe_delta;
  iod.schemes.ns.rec.type = (ReconstructionData::Reconstruction)s.rec_type;
  iod.schemes.ns.rec.limiter = (ReconstructionData::Limiter)s.limiter;
  iod.schemes.ns.rec.generalized_minmod_coeff = s.minmod_coeff;
  iod.schemes.ns.rec.slopeNearInterface = (ReconstructionData::SlopeNearInterface)s.slope_near_interface;
  iod.schemes.ns.rec.varType = (ReconstructionData::VariableType)s.rec_var;
  iod.ts.type = TsData::EXPLICIT;
  iod.ts.expl.type = s.rk_order == 1 ? ExplicitData::FORWARD_EULER
                     : s.rk_order == 2 ? ExplicitData::RUNGE_KUTTA_2 : ExplicitData::RUNGE_KUTTA_3;
  iod.ts.cfl = s.cfl;
  iod.multiphase.flux = (MultiPhaseData::Flux)s.mp_flux;
  iod.multiphase.recon = (MultiPhaseData::ReconstructionAtInterface)s.mp_recon;
  iod.multiphase.phasechange_type = (MultiPhaseData::PhaseChangeType)s.mp_phasechange_type;
  iod.multiphase.phasechange_dir = (MultiPhaseData::PhaseChangeDirection)s.mp_phasechange_dir;
  iod.multiphase.apply_failsafe_density = (MultiPhaseData::OnOff)s.mp_apply_failsafe_density;
  iod.multiphase.riemann_normal = (MultiPhaseData::RiemannNormal)s.mp_riemann_normal;
  iod.ebm.riemann_normal = (EmbeddedBoundaryMethodData::RiemannNormal)s.ebm_riemann_normal;
  iod.ebm.recon = (EmbeddedBoundaryMethodData::ReconstructionAtInterface)s.ebm_recon;
  iod.eqs.dummy_state.density = s.inactive_density;
  iod.eqs.dummy_state.pressure = s.inactive_pressure;
  iod.eqs.dummy_state.internal_energy_per_mass = s.inactive_energy;
  ExactRiemannSolverData& r = iod.exact_riemann;
  r.maxIts_main = s.riem_maxits_main;
  r.maxIts_bracket = s.riem_maxits_bracket;
  r.maxIts_shock = s.riem_maxits_shock;
  r.numSteps_rarefaction = s.riem_nsteps_rarefaction;
  r.tol_main = s.riem_tol_main;
  r.tol_shock = s.riem_tol_shock;
  r.tol_rarefaction = s.riem_tol_rarefaction;
  r.min_pressure = s.riem_min_pressure;
  r.failure_threshold = s.riem_failure_threshold;
  r.pressure_at_failure = s.riem_pressure_at_failure;
}

// Copy between a host array in ghosted layout and a SpaceVariable3D.
void copy_in(SpaceVariable3D& S, const double* h, int dof, int NX, int NY, int NZ, bool insert = true) {
  double*** a = S.GetDataPointer();
  for (int k = -1; k <= NZ; k++)
    for (int j = -1; j <= NY; j++)
      for (int i = -1; i <= NX; i++)
        for (int p = 0; p < dof; p++)
          a[k][j][i * dof + p] = h[(((size_t)(k + 1) * (NY + 2) + (j + 1)) * (NX + 2) + (i + 1)) * dof + p];
  if (insert)
    S.RestoreDataPointerAndInsert();
  else
    S.RestoreDataPointerToLocalVector();
}

void copy_out(SpaceVariable3D& S, double* h, int dof, int NX, int NY, int NZ) {
  double*** a = S.GetDataPointer();
  for (int k = -1; k <= NZ; k++)
    for (int j = -1; j <= NY; j++)
      for (int i = -1; i <= NX; i++)
        for (int p = 0; p < dof; p++)
          h[(((size_t)(k + 1) * (NY + 2) + (j + 1)) * (NX + 2) + (i + 1)) * dof + p] = a[k][j][i * dof + p];
  S.RestoreDataPointerToLocalVector();
}

}  // namespace

extern "C" {

void* m2cref_create(const m2cg_grid* g, const m2cg_scheme* s, const m2cg_material* mats, int nmat,
                    const m2cg_levelset* ls, int nls) {
  RefCase* c = new RefCase;
  IoData& iod = c->iod;
  verbose = 0;

  iod.mesh.x0 = g->x0; iod.mesh.xmax = g->xmax;
  iod.mesh.y0 = g->y0; iod.mesh.ymax = g->ymax;
  iod.mesh.z0 = g->z0; iod.mesh.zmax = g->zmax;
  iod.mesh.Nx = g->nx; iod.mesh.Ny = g->ny; iod.mesh.Nz = g->nz;
  iod.mesh.bc_x0 = to_bc(g->bc[0]); iod.mesh.bc_xmax = to_bc(g->bc[1]);
  iod.mesh.bc_y0 = to_bc(g->bc[2]); iod.mesh.bc_ymax = to_bc(g->bc[3]);
  iod.mesh.bc_z0 = to_bc(g->bc[4]); iod.mesh.bc_zmax = to_bc(g->bc[5]);
  iod.bc.inlet.density = g->inlet[0];
  iod.bc.inlet.velocity_x = g->inlet[1];
  iod.bc.inlet.velocity_y = g->inlet[2];
  iod.bc.inlet.velocity_z = g->inlet[3];
  iod.bc.inlet.pressure = g->inlet[4];
  iod.bc.outlet.density = g->outlet[0];
  iod.bc.outlet.velocity_x = g->outlet[1];
  iod.bc.outlet.velocity_y = g->outlet[2];
  iod.bc.outlet.velocity_z = g->outlet[3];
  iod.bc.outlet.pressure = g->outlet[4];

  for (int m = 0; m < nmat; m++) {
    MaterialModelData* d = new MaterialModelData();
    fill_material(d, mats[m]);
    iod.eqs.materials.dataMap[m] = d;
  }
  fill_scheme(iod, *s);
  for (int l = 0; l < nls; l++) {
    LevelSetSchemeData* d = new LevelSetSchemeData();
    d->materialid = ls[l].material_id;
    d->bc_x0 = (LevelSetSchemeData::BcType)ls[l].bc[0];
    d->bc_xmax = (LevelSetSchemeData::BcType)ls[l].bc[1];
    d->bc_y0 = (LevelSetSchemeData::BcType)ls[l].bc[2];
    d->bc_ymax = (LevelSetSchemeData::BcType)ls[l].bc[3];
    d->bc_z0 = (LevelSetSchemeData::BcType)ls[l].bc[4];
    d->bc_zmax = (LevelSetSchemeData::BcType)ls[l].bc[5];
    d->reinit.frequency = ls[l].reinit_frequency;
    d->reinit.maxIts = ls[l].reinit_maxits;
    d->reinit.cfl = ls[l].reinit_cfl;
    d->reinit.convergence_tolerance = ls[l].reinit_tol;
    d->reinit.firstLayerTreatment = (LevelSetReinitializationData::FirstLayerTreatment)ls[l].reinit_first_layer;
    d->solver = (LevelSetSchemeData::Solver)ls[l].solver;
    d->flux = (LevelSetSchemeData::Flux)ls[l].flux;
    d->delta = ls[l].delta;
    d->rec.type = (ReconstructionData::Reconstruction)ls[l].rec_type;
    d->rec.limiter = (ReconstructionData::Limiter)ls[l].limiter;
    d->rec.generalized_minmod_coeff = ls[l].minmod_coeff;
    iod.schemes.ls.dataMap[l] = d;
  }
  iod.finalize();

  // EOS per material + the dummy "inactive" material (Main.cpp:106-138).
  for (int m = 0; m < nmat; m++) {
    MaterialModelData* d = iod.eqs.materials.dataMap[m];
    if (d->eos == MaterialModelData::STIFFENED_GAS)
      c->vf.push_back(new VarFcnSG(*d));
    else
      c->vf.push_back(new VarFcnNASG(*d));
  }
  c->vf.push_back(new VarFcnDummy(iod.eqs.dummy_state));
  INACTIVE_MATERIAL_ID = (int)c->vf.size() - 1;

  c->riemann = new ExactRiemannSolverBase(c->vf, iod.exact_riemann);
  if (iod.schemes.ns.flux == SchemeData::ROE)
    c->ff = new FluxFcnGenRoe(c->vf, iod);
  else if (iod.schemes.ns.flux == SchemeData::LOCAL_LAX_FRIEDRICHS)
    c->ff = new FluxFcnLLF(c->vf, iod);
  else
    c->ff = new FluxFcnHLLC(c->vf, iod);

  // Mesh (Main.cpp:161-169), or the caller's non-uniform cell centres/widths.
  std::vector<double> xc, dx, yc, dy, zc, dz;
  MeshGenerator meshgen;
  meshgen.ComputeMeshCoordinatesAndDeltas(iod.mesh, xc, yc, zc, dx, dy, dz);
  if (g->xc && g->dx) { xc.assign(g->xc, g->xc + g->nx); dx.assign(g->dx, g->dx + g->nx); }
  if (g->yc && g->dy) { yc.assign(g->yc, g->yc + g->ny); dy.assign(g->dy, g->dy + g->ny); }
  if (g->zc && g->dz) { zc.assign(g->zc, g->zc + g->nz); dz.assign(g->dz, g->dz + g->nz); }
  domain_diagonal = sqrt(pow(iod.mesh.xmax - iod.mesh.x0, 2) + pow(iod.mesh.ymax - iod.mesh.y0, 2) +
                         pow(iod.mesh.zmax - iod.mesh.z0, 2));
  c->gmi = new GlobalMeshInfo(xc, yc, zc, dx, dy, dz);
  c->NX = (int)xc.size(); c->NY = (int)yc.size(); c->NZ = (int)zc.size();
  c->dms = new DataManagers3D(c->comm, c->NX, c->NY, c->NZ);
  c->gmi->GetSubdomainInfo(c->comm, *c->dms);
  c->spo = new SpaceOperator(c->comm, *c->dms, iod, c->vf, *c->ff, *c->riemann, *c->gmi, false);
  bool viscous = false, heat = false;
  for (int m = 0; m < nmat; m++) {
    viscous = viscous || mats[m].mu != 0.0 || mats[m].mu_bulk != 0.0;
    heat = heat || mats[m].heat_diffusivity != 0.0;
  }
  if (viscous || heat) {  // Main.cpp:195-208: linear interpolation + central differences
    c->interp = new InterpolatorLinear(c->comm, *c->dms, c->spo->GetMeshCoordinates(), c->spo->GetMeshDeltaXYZ());
    c->grad = new GradientCalculatorCentral(c->comm, *c->dms, c->spo->GetMeshCoordinates(), c->spo->GetMeshDeltaXYZ(),
                                            *c->interp);
    c->spo->SetupViscosityOperator(c->interp, c->grad, false);
    c->spo->SetupHeatDiffusionOperator(c->interp, c->grad);
  }

  c->V = new SpaceVariable3D(c->comm, &(c->dms->ghosted1_5dof));
  c->ID = new SpaceVariable3D(c->comm, &(c->dms->ghosted1_1dof));

  for (auto it = iod.schemes.ls.dataMap.begin(); it != iod.schemes.ls.dataMap.end(); it++) {
    c->lso.push_back(new LevelSetOperator(c->comm, *c->dms, iod, *it->second, *c->spo));
    c->Phi.push_back(new SpaceVariable3D(c->comm, &(c->dms->ghosted1_1dof)));
  }
  c->mpo = new MultiPhaseOperator(c->comm, *c->dms, iod, c->vf, *c->gmi, *c->spo, c->lso);

#ifdef M2C_DROPIN
  c->integrator = new TimeIntegratorGPU(c->comm, iod, *c->dms, *c->spo, c->lso, *c->mpo, s->precision);
  return c;
#endif
  if (iod.ts.expl.type == ExplicitData::FORWARD_EULER)
    c->integrator = new TimeIntegratorFE(c->comm, iod, *c->dms, *c->spo, c->lso, *c->mpo, nullptr, nullptr, nullptr);
  else if (iod.ts.expl.type == ExplicitData::RUNGE_KUTTA_2)
    c->integrator = new TimeIntegratorRK2(c->comm, iod, *c->dms, *c->spo, c->lso, *c->mpo, nullptr, nullptr, nullptr);
  else
    c->integrator = new TimeIntegratorRK3(c->comm, iod, *c->dms, *c->spo, c->lso, *c->mpo, nullptr, nullptr, nullptr);
  return c;
}

// Set the state; interior values are taken from the host arrays and the
// end-of-initial-condition steps of the reference are applied
// (SpaceOperator.cpp:1088-1089 clip + BCs, level-set BCs,
// MultiPhaseOperator::UpdateMaterialIDAtGhostNodes as in Main.cpp:301).
void m2cref_set_state(void* h, const double* V, const double* ID, const double* phi) {
  RefCase* c = (RefCase*)h;
  copy_in(*c->V, V, 5, c->NX, c->NY, c->NZ);
  if (ID)
    copy_in(*c->ID, ID, 1, c->NX, c->NY, c->NZ);
  else
    c->ID->SetConstantValue(0.0, true);
  for (size_t l = 0; l < c->Phi.size(); l++)
    copy_in(*c->Phi[l], phi + l * (size_t)(c->NX + 2) * (c->NY + 2) * (c->NZ + 2), 1, c->NX, c->NY, c->NZ);
  c->spo->ClipDensityAndPressure(*c->V, *c->ID);
  c->spo->ApplyBoundaryConditions(*c->V);
  for (size_t l = 0; l < c->lso.size(); l++) c->lso[l]->ApplyBoundaryConditions(*c->Phi[l]);
  c->mpo->UpdateMaterialIDAtGhostNodes(*c->ID);
}

// Raw state overwrite (no clipping, no boundary conditions).
void m2cref_set_state_raw(void* h, const double* V, const double* ID, const double* phi) {
  RefCase* c = (RefCase*)h;
  copy_in(*c->V, V, 5, c->NX, c->NY, c->NZ);
  if (ID) copy_in(*c->ID, ID, 1, c->NX, c->NY, c->NZ);
  for (size_t l = 0; l < c->Phi.size(); l++)
    copy_in(*c->Phi[l], phi + l * (size_t)(c->NX + 2) * (c->NY + 2) * (c->NZ + 2), 1, c->NX, c->NY, c->NZ);
}

void m2cref_get_state(void* h, double* V, double* ID, double* phi) {
  RefCase* c = (RefCase*)h;
  if (V) copy_out(*c->V, V, 5, c->NX, c->NY, c->NZ);
  if (ID) copy_out(*c->ID, ID, 1, c->NX, c->NY, c->NZ);
  if (phi)
    for (size_t l = 0; l < c->Phi.size(); l++)
      copy_out(*c->Phi[l], phi + l * (size_t)(c->NX + 2) * (c->NY + 2) * (c->NZ + 2), 1, c->NX, c->NY, c->NZ);
}

// MultiPhaseOperator::UpdateStateVariablesAfterInterfaceMotion with the given
// step-start IDs and no stored Riemann solutions (an empty RiemannSolutions),
// followed by the clip and boundary conditions of
// TimeIntegratorBase::UpdateSolutionAfterTimeStepping (TimeIntegrator.cpp:767-768).
// Returns the number of cells still unresolved.
int m2cref_update_states_after_motion(void* h, const double* IDn) {
  RefCase* c = (RefCase*)h;
  SpaceVariable3D idn(c->comm, &(c->dms->ghosted1_1dof));
  copy_in(idn, IDn, 1, c->NX, c->NY, c->NZ);
  RiemannSolutions rs;
  std::vector<Int3> unresolved;
  int n = c->mpo->UpdateStateVariablesAfterInterfaceMotion(idn, *c->ID, *c->V, rs, nullptr, unresolved);
  c->spo->ClipDensityAndPressure(*c->V, *c->ID);
  c->spo->ApplyBoundaryConditions(*c->V);
  idn.Destroy();
  return n;
}

double m2cref_compute_dt(void* h) {
  RefCase* c = (RefCase*)h;
  double dt = 0.0, cfl = 0.0;
  c->spo->ComputeTimeStepSize(*c->V, *c->ID, dt, cfl);
  return dt;
}

// An embedded surface cutting the listed faces: one EmbeddedBoundaryDataSet
// whose intersector results are written directly, so that
// SpaceOperator::FindEdgeSurfaceIntersections (SpaceOperator.cpp:3435-3501)
// yields the given normal and velocity on each face. Face q = (axis d, i, j,
// k) gets two triangles, 2q (forward: normal nf, node velocity uf) and 2q+1
// (backward), each met at barycentric coordinates (1, 0, 0), so the
// interpolated surface velocity is the given one exactly; XForward /
// XBackward of node (i, j, k), component d, hold 2q and 2q+1.
struct HandSurface {
  TriangulatedSurface surf;
  std::vector<IntersectionPoint> xs;
  SpaceVariable3D* xf = nullptr;
  SpaceVariable3D* xb = nullptr;
  std::vector<std::unique_ptr<EmbeddedBoundaryDataSet>> ebds;
  HandSurface(RefCase* c, int n, const int* faces, const double* nf, const double* uf, const double* nb,
              const double* ub) {
    xf = new SpaceVariable3D(c->comm, &(c->dms->ghosted1_3dof));
    xb = new SpaceVariable3D(c->comm, &(c->dms->ghosted1_3dof));
    xf->SetConstantValue(-1.0, true);
    xb->SetConstantValue(-1.0, true);
    Vec3D*** f = (Vec3D***)xf->GetDataPointer();
    Vec3D*** b = (Vec3D***)xb->GetDataPointer();
    double xi[3] = {1.0, 0.0, 0.0};
    for (int q = 0; q < n; q++) {
      const int d = faces[4 * q], i = faces[4 * q + 1], j = faces[4 * q + 2], k = faces[4 * q + 3];
      for (int side = 0; side < 2; side++) {
        const double* nw = side == 0 ? nf + 3 * q : nb + 3 * q;
        const double* uw = side == 0 ? uf + 3 * q : ub + 3 * q;
        const int base = (int)surf.Udot.size();
        for (int v = 0; v < 3; v++) surf.X.push_back(Vec3D(0.0, 0.0, 0.0));
        surf.Udot.push_back(Vec3D(uw[0], uw[1], uw[2]));
        surf.Udot.push_back(Vec3D(0.0, 0.0, 0.0));
        surf.Udot.push_back(Vec3D(0.0, 0.0, 0.0));
        surf.elems.push_back(Int3(base, base + 1, base + 2));
        surf.elemNorm.push_back(Vec3D(nw[0], nw[1], nw[2]));
        const int tid = 2 * q + side;
        xs.push_back(IntersectionPoint(i, j, k, d, side == 0 ? 0.25 : 0.75, tid, xi));
        (side == 0 ? f : b)[k][j][i][d] = (double)tid;
      }
    }
    xf->RestoreDataPointerAndInsert();
    xb->RestoreDataPointerAndInsert();
    ebds.push_back(std::make_unique<EmbeddedBoundaryDataSet>());
    ebds[0]->surface_ptr = &surf;
    ebds[0]->XForward_ptr = xf;
    ebds[0]->XBackward_ptr = xb;
    ebds[0]->intersections_ptr = &xs;
  }
  ~HandSurface() {
    xf->Destroy();
    xb->Destroy();
    delete xf;
    delete xb;
  }
};

// R for the current state with an embedded surface cutting the listed faces.
void m2cref_compute_residual_walls(void* h, int n, const int* faces, const double* nf, const double* uf,
                                   const double* nb, const double* ub, double* R) {
  RefCase* c = (RefCase*)h;
  HandSurface hs(c, n, faces, nf, uf, nb, ub);
  SpaceVariable3D Rv(c->comm, &(c->dms->ghosted1_5dof));
  c->spo->ComputeResidual(*c->V, *c->ID, Rv, nullptr, nullptr, nullptr, &hs.ebds);
  copy_out(Rv, R, 5, c->NX, c->NY, c->NZ);
  Rv.Destroy();
}

// nsteps CFL steps of one material with an embedded surface cutting the
// listed faces: the statements of TimeIntegratorRK2 / RK3::
// AdvanceOneTimeStep (TimeIntegrator.cpp:291-428, 496-690) without level
// sets (UpdateSolutionAfterTimeStepping then does nothing), with the
// surface's data set passed to every ComputeResidual, as the reference's
// integrator does with its EmbeddedBoundaryOperator's. Returns steps taken.
int m2cref_run_walls(void* h, int n, const int* faces, const double* nf, const double* uf, const double* nb,
                     const double* ub, int nsteps, double* t_out) {
  RefCase* c = (RefCase*)h;
  if (!c->Phi.empty()) return -1;
  const int rk = c->iod.ts.expl.type == ExplicitData::RUNGE_KUTTA_3 ? 3 : 2;
  HandSurface hs(c, n, faces, nf, uf, nb, ub);
  auto* E = &hs.ebds;
  SpaceVariable3D R(c->comm, &(c->dms->ghosted1_5dof)), Un(c->comm, &(c->dms->ghosted1_5dof)),
      U1(c->comm, &(c->dms->ghosted1_5dof)), V1(c->comm, &(c->dms->ghosted1_5dof)),
      V2(c->comm, &(c->dms->ghosted1_5dof));
  SpaceVariable3D& V = *c->V;
  SpaceVariable3D& ID = *c->ID;
  SpaceOperator& spo = *c->spo;
  int done = 0;
  for (; done < nsteps; done++) {
    double dt = 0.0, cfl = 0.0;
    spo.ComputeTimeStepSize(V, ID, dt, cfl);
    c->time_step++;
    c->t += dt;
    spo.ComputeResidual(V, ID, R, nullptr, nullptr, nullptr, E);
    spo.PrimitiveToConservative(V, ID, Un);
    U1.AXPlusBY(0.0, 1.0, Un);
    U1.AXPlusBY(1.0, dt, R);
    spo.ConservativeToPrimitive(U1, ID, V1);
    if (spo.ClipDensityAndPressure(V1, ID)) spo.PrimitiveToConservative(V1, ID, U1);
    spo.ApplyBoundaryConditions(V1);
    spo.ComputeResidual(V1, ID, R, nullptr, nullptr, nullptr, E);
    if (rk == 2) {
      U1.AXPlusBY(0.5, 0.5, Un);
      U1.AXPlusBY(1.0, 0.5 * dt, R);
    } else {
      U1.AXPlusBY(0.25, 0.75, Un);
      U1.AXPlusBY(1.0, 0.25 * dt, R);
      spo.ConservativeToPrimitive(U1, ID, V2);
      if (spo.ClipDensityAndPressure(V2, ID)) spo.PrimitiveToConservative(V2, ID, U1);
      spo.ApplyBoundaryConditions(V2);
      spo.ComputeResidual(V2, ID, R, nullptr, nullptr, nullptr, E);
      U1.AXPlusBY(2.0 / 3.0, 1.0 / 3.0, Un);
      U1.AXPlusBY(1.0, 2.0 / 3.0 * dt, R);
    }
    spo.ConservativeToPrimitive(U1, ID, V);
    spo.ClipDensityAndPressure(V, ID);
    spo.ApplyBoundaryConditions(V);
  }
  R.Destroy();
  Un.Destroy();
  U1.Destroy();
  V1.Destroy();
  V2.Destroy();
  if (t_out) *t_out = c->t;
  return done;
}

// R for the current state (ghosted layout, 5 dof).
void m2cref_compute_residual(void* h, double* R) {
  RefCase* c = (RefCase*)h;
  SpaceVariable3D Rv(c->comm, &(c->dms->ghosted1_5dof));
  c->spo->ComputeResidual(*c->V, *c->ID, Rv);
  copy_out(Rv, R, 5, c->NX, c->NY, c->NZ);
  Rv.Destroy();
}

// One step with the given dt; time is the reference's updated time t+dt.
void m2cref_advance(void* h, double dt) {
  RefCase* c = (RefCase*)h;
  c->time_step++;
  c->t += dt;
  c->integrator->AdvanceOneTimeStep(*c->V, *c->ID, c->Phi, nullptr, nullptr, nullptr, c->t, dt,
                                    c->time_step, 0, dt);
}

// The reference time loop (Main.cpp:514-575): dt from the CFL condition,
// last step shortened to end at t_max. Returns steps taken.
int m2cref_run(void* h, int nsteps, double t_max, double* t_out) {
  RefCase* c = (RefCase*)h;
  int done = 0;
  auto t0 = std::chrono::steady_clock::now();
  while (done < nsteps && c->t < t_max) {
    double dt = 0.0, cfl = 0.0;
    c->spo->ComputeTimeStepSize(*c->V, *c->ID, dt, cfl);
    if (c->t + dt > t_max) dt = t_max - c->t;
    m2cref_advance(h, dt);
    done++;
  }
  auto t1 = std::chrono::steady_clock::now();
  c->advance_seconds += std::chrono::duration<double>(t1 - t0).count();
  if (t_out) *t_out = c->t;
  return done;
}

double m2cref_seconds(void* h) { return ((RefCase*)h)->advance_seconds; }
double m2cref_time(void* h) { return ((RefCase*)h)->t; }

void m2cref_destroy(void* h) {
  RefCase* c = (RefCase*)h;
  c->integrator->Destroy();
  delete c->integrator;
  c->mpo->Destroy();
  delete c->mpo;
  for (size_t l = 0; l < c->lso.size(); l++) {
    c->Phi[l]->Destroy(); delete c->Phi[l];
    c->lso[l]->Destroy(); delete c->lso[l];
  }
  c->V->Destroy(); delete c->V;
  c->ID->Destroy(); delete c->ID;
  c->spo->Destroy();
  delete c->spo;
  if (c->grad) { c->grad->Destroy(); delete c->grad; }
  if (c->interp) { c->interp->Destroy(); delete c->interp; }
  c->dms->DestroyAllDataManagers();
  delete c->dms;
  delete c->gmi;
  delete c->ff;
  delete c->riemann;
  for (auto* v : c->vf) delete v;
  delete c;
}

// ---------------------------------------------------------------------------
// Point-wise entry points (no mesh): EOS, numerical flux, exact Riemann.
// ---------------------------------------------------------------------------
struct RefPoint {
  IoData iod;
  std::vector<VarFcnBase*> vf;
  FluxFcnBase* ff = nullptr;
  ExactRiemannSolverBase* riemann = nullptr;
};

void* m2cref_point_create(const m2cg_scheme* s, const m2cg_material* mats, int nmat) {
  RefPoint* p = new RefPoint;
  for (int m = 0; m < nmat; m++) {
    MaterialModelData* d = new MaterialModelData();
    fill_material(d, mats[m]);
    p->iod.eqs.materials.dataMap[m] = d;
    if (d->eos == MaterialModelData::STIFFENED_GAS)
      p->vf.push_back(new VarFcnSG(*d));
    else
      p->vf.push_back(new VarFcnNASG(*d));
  }
  fill_scheme(p->iod, *s);
  p->vf.push_back(new VarFcnDummy(p->iod.eqs.dummy_state));
  INACTIVE_MATERIAL_ID = (int)p->vf.size() - 1;
  if (s->flux == M2CG_FLUX_ROE)
    p->ff = new FluxFcnGenRoe(p->vf, p->iod);
  else if (s->flux == M2CG_FLUX_LLF)
    p->ff = new FluxFcnLLF(p->vf, p->iod);
  else
    p->ff = new FluxFcnHLLC(p->vf, p->iod);
  p->riemann = new ExactRiemannSolverBase(p->vf, p->iod.exact_riemann);
  return p;
}

void m2cref_point_flux(void* h, int n, int dir, const double* Vm, const double* Vp, const int* id, double* F) {
  RefPoint* p = (RefPoint*)h;
  for (int q = 0; q < n; q++) {
    double a[5], b[5];
    memcpy(a, Vm + 5 * q, sizeof a);
    memcpy(b, Vp + 5 * q, sizeof b);
    p->ff->ComputeNumericalFluxAtCellInterface(dir, a, b, id[q], F + 5 * q);
  }
}

void m2cref_point_c2p(void* h, int n, const double* U, const int* id, double* V) {
  RefPoint* p = (RefPoint*)h;
  for (int q = 0; q < n; q++) {
    double u[5];
    memcpy(u, U + 5 * q, sizeof u);
    p->vf[id[q]]->ConservativeToPrimitive(u, V + 5 * q);
  }
}

void m2cref_point_p2c(void* h, int n, const double* V, const int* id, double* U) {
  RefPoint* p = (RefPoint*)h;
  for (int q = 0; q < n; q++) {
    double v[5];
    memcpy(v, V + 5 * q, sizeof v);
    p->vf[id[q]]->PrimitiveToConservative(v, U + 5 * q);
  }
}

int m2cref_point_riemann(void* h, int n, const double* dir, const double* VL, const int* idl,
                         const double* VR, const int* idr, double* Vs, int* id, double* Vsm, double* Vsp,
                         int* err) {
  RefPoint* p = (RefPoint*)h;
  int nerr = 0;
  for (int q = 0; q < n; q++) {
    double d[3], a[5], b[5];
    memcpy(d, dir + 3 * q, sizeof d);
    memcpy(a, VL + 5 * q, sizeof a);
    memcpy(b, VR + 5 * q, sizeof b);
    int midid = 0;
    err[q] = p->riemann->ComputeRiemannSolution(d, a, idl[q], b, idr[q], Vs + 5 * q, midid, Vsm + 5 * q,
                                                Vsp + 5 * q);
    id[q] = midid;
    nerr += err[q] != 0;
  }
  return nerr;
}

// ExactRiemannSolverBase::ComputeOneSidedRiemannSolution on each problem;
// Vs is zeroed first (the reference leaves it untouched where id = -1).
int m2cref_point_riemann_wall(void* h, int n, const double* dir, const double* Vm, const int* idm,
                              const double* uwall, double* Vs, int* id, double* Vsm, int* err) {
  RefPoint* p = (RefPoint*)h;
  int nerr = 0;
  for (int q = 0; q < n; q++) {
    double d[3], a[5], w[3];
    memcpy(d, dir + 3 * q, sizeof d);
    memcpy(a, Vm + 5 * q, sizeof a);
    memcpy(w, uwall + 3 * q, sizeof w);
    for (int c = 0; c < 5; c++) Vs[5 * q + c] = 0.0;
    int midid = 0;
    err[q] = p->riemann->ComputeOneSidedRiemannSolution(d, a, idm[q], w, Vs + 5 * q, midid, Vsm + 5 * q);
    id[q] = midid;
    nerr += err[q] != 0;
  }
  return nerr;
}

void m2cref_point_destroy(void* h) {
  RefPoint* p = (RefPoint*)h;
  delete p->ff;
  delete p->riemann;
  for (auto* v : p->vf) delete v;
  delete p;
}

}  // extern "C"
