// TimeIntegratorGPU: the drop-in a maintainer adds to M2C so that its own
// driver advances the flow on a B200 through the C-ABI of m2c_gpu.h.
//
// It is a TimeIntegratorBase (TimeIntegrator.h:22-80) like TimeIntegratorRK2
// and TimeIntegratorRK3 (TimeIntegrator.cpp:291-690): Main.cpp constructs it
// where it now constructs those (Main.cpp:368-379) and keeps calling
// ComputeTimeStepSize (Main.cpp:524) and AdvanceOneTimeStep (Main.cpp:570)
// unchanged. Each step uploads V, ID and phi from the reference's own
// ghosted local vectors (SpaceVariable3D::GetDataPointer), advances them by
// one explicit RK step on the GPU (m2cg_advance) and writes them back, ghost
// layers included. The scope is the GPU path's: one structured subdomain
// (a single-rank run), at most one level set (finite-difference or
// finite-volume), MUSCL in any of the reference's variable types.
//
// Built against the reference's headers (IoData.h, TimeIntegrator.h,
// MeshGenerator.h) and linked with libm2c_gpu.so.
#pragma once
#include <IoData.h>
#include <MeshGenerator.h>
#include <SpaceOperator.h>
#include <TimeIntegrator.h>
#include <Utils.h>

#include <vector>

#include "../../include/m2c_gpu.h"

class TimeIntegratorGPU : public TimeIntegratorBase {
  m2cg_ctx* ctx = nullptr;

  static void fail(m2cg_status st) {
    print_error("*** Error: GPU time integrator (status %d): %s\n", (int)st, m2cg_last_error());
    exit_mpi();
  }

  // Base of a single-subdomain ghosted local array: node (-1,-1,-1), dof 0.
  static double* ghosted_base(SpaceVariable3D& S, int dof) {
    double*** a = S.GetDataPointer();
    return &a[-1][-1][-dof];
  }

 public:
  // precision: M2CG_PREC_FP64 or M2CG_PREC_MIXED
  TimeIntegratorGPU(MPI_Comm& comm_, IoData& iod_, DataManagers3D& dms_, SpaceOperator& spo_,
                    vector<LevelSetOperator*>& lso_, MultiPhaseOperator& mpo_, int precision = M2CG_PREC_FP64)
      : TimeIntegratorBase(comm_, iod_, dms_, spo_, lso_, mpo_, nullptr, nullptr, nullptr) {
    // mesh: the reference's own generator, passed as explicit centres/widths
    std::vector<double> xc, yc, zc, dx, dy, dz;
    MeshGenerator meshgen;
    meshgen.ComputeMeshCoordinatesAndDeltas(iod.mesh, xc, yc, zc, dx, dy, dz);
    m2cg_grid g;
    g.nx = (int)xc.size(); g.ny = (int)yc.size(); g.nz = (int)zc.size();
    g.x0 = iod.mesh.x0; g.xmax = iod.mesh.xmax;
    g.y0 = iod.mesh.y0; g.ymax = iod.mesh.ymax;
    g.z0 = iod.mesh.z0; g.zmax = iod.mesh.zmax;
    g.xc = xc.data(); g.dx = dx.data(); g.yc = yc.data(); g.dy = dy.data(); g.zc = zc.data(); g.dz = dz.data();
    const MeshData::BcType bcs[6] = {iod.mesh.bc_x0, iod.mesh.bc_xmax, iod.mesh.bc_y0,
                                     iod.mesh.bc_ymax, iod.mesh.bc_z0, iod.mesh.bc_zmax};
    for (int q = 0; q < 6; q++) g.bc[q] = (int)bcs[q];  // MeshData::BcType values 0..5 are the C-ABI's
    const StateVariable& in = iod.bc.inlet;
    const StateVariable& out = iod.bc.outlet;
    const double inl[5] = {in.density, in.velocity_x, in.velocity_y, in.velocity_z, in.pressure};
    const double outl[5] = {out.density, out.velocity_x, out.velocity_y, out.velocity_z, out.pressure};
    for (int p = 0; p < 5; p++) { g.inlet[p] = inl[p]; g.outlet[p] = outl[p]; }
    // materials
    std::vector<m2cg_material> mats;
    for (auto it = iod.eqs.materials.dataMap.begin(); it != iod.eqs.materials.dataMap.end(); it++) {
      const MaterialModelData& d = *it->second;
      m2cg_material m;
      m2cg_default_material(&m);
      const bool nasg = d.eos == MaterialModelData::NOBLE_ABEL_STIFFENED_GAS;
      m.eos = nasg ? M2CG_EOS_NASG : M2CG_EOS_SG;
      m.gamma = nasg ? d.nasgModel.specificHeatRatio : d.sgModel.specificHeatRatio;
      m.p_c = nasg ? d.nasgModel.pressureConstant : d.sgModel.pressureConstant;
      m.b = nasg ? d.nasgModel.volumeConstant : 0.0;
      m.q = nasg ? d.nasgModel.energyConstant : 0.0;
      m.rhomin = d.rhomin; m.pmin = d.pmin; m.rhomax = d.rhomax; m.pmax = d.pmax;
      m.failsafe_density = d.failsafe_density;
      // viscosity and heat diffusion (ViscosityModelData / HeatDiffusionModelData
      // CONSTANT) with the EOS's temperature law; other models are refused
      if (d.viscosity.type == ViscosityModelData::CONSTANT) {
        m.mu = d.viscosity.dynamicViscosity;
        m.mu_bulk = d.viscosity.bulkViscosity;
      } else if (d.viscosity.type != ViscosityModelData::NONE) {
        print_error("*** Error: the GPU integrator implements the CONSTANT viscosity model only.\n");
        exit_mpi();
      }
      if (d.heat_diffusion.type == HeatDiffusionModelData::CONSTANT) m.heat_diffusivity = d.heat_diffusion.diffusivity;
      m.cv = nasg ? d.nasgModel.cv : d.sgModel.cv;
      m.T0 = nasg ? 0.0 : d.sgModel.T0;
      m.e0 = nasg ? 0.0 : d.sgModel.e0;
      m.cp = nasg ? 0.0 : d.sgModel.cp;
      m.h0 = nasg ? 0.0 : d.sgModel.h0;
      if (m.heat_diffusivity != 0.0 && !nasg && d.sgModel.cv > 0 && d.sgModel.rho0 > 0) {
        print_error("*** Error: the GPU integrator does not implement the rho0 temperature law.\n");
        exit_mpi();
      }
      mats.push_back(m);
    }
    // scheme (SchemeData, ReconstructionData, TsData, MultiPhaseData, ExactRiemannSolverData)
    m2cg_scheme s;
    m2cg_default_scheme(&s);
    s.flux = (int)iod.schemes.ns.flux;
    s.roe_delta = iod.schemes.ns.delta;
    s.rec_type = (int)iod.schemes.ns.rec.type;
    s.limiter = (int)iod.schemes.ns.rec.limiter;
    s.minmod_coeff = iod.schemes.ns.rec.generalized_minmod_coeff;
    s.slope_near_interface = (int)iod.schemes.ns.rec.slopeNearInterface;
    s.rec_var = (int)iod.schemes.ns.rec.varType;
    s.rk_order = 1 + (int)iod.ts.expl.type;  // FORWARD_EULER, RUNGE_KUTTA_2, RUNGE_KUTTA_3
    s.cfl = iod.ts.cfl;
    s.precision = precision;
    s.mp_flux = (int)iod.multiphase.flux;
    s.mp_recon = (int)iod.multiphase.recon;
    s.mp_phasechange_type = (int)iod.multiphase.phasechange_type;
    s.mp_phasechange_dir = (int)iod.multiphase.phasechange_dir;
    s.mp_apply_failsafe_density = (int)iod.multiphase.apply_failsafe_density;
    s.mp_riemann_normal = (int)iod.multiphase.riemann_normal;
    s.ebm_riemann_normal = (int)iod.ebm.riemann_normal;  // EmbeddedBoundaryMethodData
    s.ebm_recon = (int)iod.ebm.recon;
    s.inactive_density = iod.eqs.dummy_state.density;  // VarFcnDummy (Main.cpp:137)
    s.inactive_pressure = iod.eqs.dummy_state.pressure;
    s.inactive_energy = iod.eqs.dummy_state.internal_energy_per_mass;
    const ExactRiemannSolverData& r = iod.exact_riemann;
    s.riem_maxits_main = r.maxIts_main;
    s.riem_maxits_bracket = r.maxIts_bracket;
    s.riem_maxits_shock = r.maxIts_shock;
    s.riem_nsteps_rarefaction = r.numSteps_rarefaction;
    s.riem_tol_main = r.tol_main;
    s.riem_tol_shock = r.tol_shock;
    s.riem_tol_rarefaction = r.tol_rarefaction;
    s.riem_min_pressure = r.min_pressure;
    s.riem_failure_threshold = r.failure_threshold;
    s.riem_pressure_at_failure = r.pressure_at_failure;
    // level set (at most one)
    m2cg_levelset ls;
    m2cg_default_levelset(&ls);
    const int nls = (int)iod.schemes.ls.dataMap.size();
    if (nls == 1) {
      const LevelSetSchemeData& d = *iod.schemes.ls.dataMap.begin()->second;
      ls.material_id = d.materialid;
      const LevelSetSchemeData::BcType lb[6] = {d.bc_x0, d.bc_xmax, d.bc_y0, d.bc_ymax, d.bc_z0, d.bc_zmax};
      for (int q = 0; q < 6; q++) ls.bc[q] = (int)lb[q];
      ls.reinit_frequency = d.reinit.frequency;
      ls.reinit_maxits = d.reinit.maxIts;
      ls.reinit_cfl = d.reinit.cfl;
      ls.reinit_tol = d.reinit.convergence_tolerance;
      ls.reinit_first_layer = (int)d.reinit.firstLayerTreatment;
      ls.solver = (int)d.solver;
      ls.flux = (int)d.flux;
      ls.delta = d.delta;
      ls.rec_type = (int)d.rec.type;
      ls.limiter = (int)d.rec.limiter;
      ls.minmod_coeff = d.rec.generalized_minmod_coeff;
    }
    m2cg_status st = m2cg_create(&g, &s, mats.data(), (int)mats.size(), nls ? &ls : nullptr, nls, &ctx);
    if (st != M2CG_OK) fail(st);
  }

  ~TimeIntegratorGPU() { m2cg_destroy(ctx); }

  void AdvanceOneTimeStep(SpaceVariable3D& V, SpaceVariable3D& ID, vector<SpaceVariable3D*>& Phi,
                          [[maybe_unused]] SpaceVariable3D* L, [[maybe_unused]] SpaceVariable3D* Xi,
                          [[maybe_unused]] SpaceVariable3D* LocalDt, double time, double dt, int time_step,
                          [[maybe_unused]] int subcycle, [[maybe_unused]] double dts) override {
    double* v = ghosted_base(V, 5);
    double* id = ghosted_base(ID, 1);
    double* phi = Phi.empty() ? nullptr : ghosted_base(*Phi[0], 1);
    // `time` is the time at the end of the step, as the reference passes it
    m2cg_status st = m2cg_upload_state(ctx, v, id, phi);
    if (st == M2CG_OK) st = m2cg_advance(ctx, time, dt, time_step);
    if (st == M2CG_OK) st = m2cg_download_state(ctx, v, id, phi);
    V.RestoreDataPointerAndInsert();
    ID.RestoreDataPointerAndInsert();
    if (phi) Phi[0]->RestoreDataPointerAndInsert();
    if (st != M2CG_OK) fail(st);  // the reference aborts on the same conditions
  }

  void Destroy() override {
    m2cg_destroy(ctx);
    ctx = nullptr;
    TimeIntegratorBase::Destroy();
  }
};
