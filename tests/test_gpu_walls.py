"""Faces cut by an embedded surface (walls) against the reference's
embedded-boundary branch of SpaceOperator::ComputeAdvectionFluxes
(SpaceOperator.cpp:2438-2484 and the y/z analogues): on each cut face the low
cell's flux against its one-sided Riemann star state
(ExactRiemannSolverBase::ComputeOneSidedRiemannSolution, the surface seen
forward) and the high cell's against its own (seen backward).

The reference side runs SpaceOperator::ComputeResidual with one
EmbeddedBoundaryDataSet whose intersector results are written so that
FindEdgeSurfaceIntersections yields the same normal and velocity on the same
faces (oracle/ref_harness.cpp, m2cref_compute_residual_walls). Bar: the FP64
residual within 1e-12 relative (max norm per variable); the mixed path
tracks FP64 in L1.
"""
import numpy as np
import pytest

from m2c_b200 import abi, cases
from tests.helpers import inner, l1_rel, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def wall_faces(g, n, seed, speed=0.4):
    """n distinct interior faces of every axis (the low neighbour interior
    too), unit normals near each face normal, velocities uniform in
    +-speed per component."""
    rng = np.random.default_rng(seed)
    dims = (g.nx, g.ny, g.nz)
    out = set()
    while len(out) < n:
        d = int(rng.integers(0, 3))
        ijk = [int(rng.integers(0, m)) for m in dims]
        ijk[d] = int(rng.integers(1, dims[d]))
        out.add((d, *ijk))
    faces = np.array(sorted(out), np.int32)
    def normals():
        v = rng.normal(scale=0.4, size=(n, 3))
        v[np.arange(n), faces[:, 0]] += rng.choice([-1.0, 1.0], n)
        return v / np.linalg.norm(v, axis=1)[:, None]
    nf, nb = normals(), normals()
    uf = rng.uniform(-speed, speed, (n, 3))
    ub = rng.uniform(-speed, speed, (n, 3))
    return faces, nf, uf, nb, ub


@pytest.mark.parametrize("normal", [abi.EBM_NORMAL_MESH, abi.EBM_NORMAL_SURFACE, abi.EBM_NORMAL_AVERAGE])
@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_ROE])
def test_wall_residual_matches_reference(gpu, ref, normal, flux):
    g, s, mats, V = cases.random_box(14, 11, 9, seed=5, flux=flux)
    s.ebm_riemann_normal = normal
    W = wall_faces(g, 120, seed=normal)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.set_wall_faces(*W)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    Rg, Rr = inner(sol.residual()), inner(rc.residual_walls(*W))
    assert rel_err(Rg, Rr) <= TOL
    # the walls matter: the residual without them differs
    assert rel_err(inner(rc.residual()), Rr) > 1e-6
    # each residual evaluation solves two one-sided problems per cut face
    c = sol.counters()
    assert c["wall_riemann_calls"] == 2 * len(W[0])
    # removing the walls restores the plain residual
    sol.set_wall_faces(np.zeros((0, 4), np.int32))
    assert rel_err(inner(sol.residual()), inner(rc.residual())) <= TOL
    sol.close()


@pytest.mark.parametrize("normal", [abi.EBM_NORMAL_MESH, abi.EBM_NORMAL_AVERAGE])
def test_wall_residual_linear_reconstruction_matches_reference(gpu, ref, normal):
    """EmbeddedBoundaryMethodData::recon LINEAR: the one-sided problems and
    the fluxes take the limited face states (vr of the low cell, vl of the
    high cell, SpaceOperator.cpp:2452-2456, 2474-2478), which a face pass of
    the stage kernel writes; every limiter branch of the random box."""
    g, s, mats, V = cases.random_box(14, 11, 9, seed=5)
    s.ebm_recon = 1
    s.ebm_riemann_normal = normal
    W = wall_faces(g, 120, seed=7)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.set_wall_faces(*W)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    Rr = inner(rc.residual_walls(*W))
    assert rel_err(inner(sol.residual()), Rr) <= TOL
    s0 = abi.scheme(**{f: getattr(s, f) for f, _ in abi.Scheme._fields_})
    s0.ebm_recon = 0
    rc0 = ref.RefCase(g, s0, mats)
    rc0.set_state(V)
    assert rel_err(inner(rc0.residual_walls(*W)), Rr) > 1e-8  # LINEAR differs from CONSTANT
    sol.close()


def test_wall_residual_of_receding_and_fast_walls_matches_reference(gpu, ref):
    """Walls moving away faster than the fluid can follow (the one-sided
    rarefaction reports failure and the reference keeps the input state
    with the wall's normal velocity) and walls driven into the fluid
    (strong shocks)."""
    g, s, mats, V = cases.random_box(12, 10, 8, seed=9)
    W = wall_faces(g, 90, seed=4, speed=12.0)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.set_wall_faces(*W)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert rel_err(inner(sol.residual()), inner(rc.residual_walls(*W))) <= TOL
    assert sol.counters()["riemann_errors"] > 0
    sol.close()


@pytest.mark.parametrize("linear", [False, True])
def test_wall_residual_two_materials_matches_reference(gpu, ref, linear):
    """A surface through the bubble case: cut faces between two cells of the
    same material and across the material interface (the wall branch is
    taken there, as in the reference), water and air; with linear=True LINEAR
    reconstruction at both the material interface and the surface (one face
    pass writes both sets of face states)."""
    if not ref.available("crpow"):
        pytest.skip("reference oracle with correctly rounded pow not built (make -C oracle refcr)")
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(16, reinit_frequency=-1, radius=4.0e-3)
    V[1:-1, 1:-1, 1:-1, 1:4] += np.array([20.0, -10.0, 5.0])
    faces = [(0, 10, j, k) for j in range(3, 13) for k in range(3, 13)]
    faces += [(1, i, 8, k) for i in range(5, 11) for k in range(5, 11)]
    faces = np.array(faces, np.int32)
    n = len(faces)
    rng = np.random.default_rng(3)
    en = np.zeros((n, 3))
    en[np.arange(n), faces[:, 0]] = 1.0
    uf = rng.uniform(-30.0, 30.0, (n, 3))
    W = (faces, en, uf, en, uf)
    if linear:
        s.mp_recon = 1
        s.ebm_recon = 1
    sol = gpu.Solver(g, s, mats, ls)
    sol.upload(V, ID, PHI)
    sol.set_wall_faces(*W)
    rc = ref.RefCaseCR(g, s, mats, ls)
    rc.set_state(V, ID, PHI)
    idg = inner(ID)
    lo = np.array([idg[k, j, i - 1] if d == 0 else idg[k, j - 1, i] for d, i, j, k in faces])
    hi = np.array([idg[k, j, i] for d, i, j, k in faces])
    assert (lo != hi).sum() > 0 and (lo == hi).sum() > 0
    assert rel_err(inner(sol.residual()), inner(rc.residual_walls(*W))) <= TOL
    sol.close()


@pytest.mark.parametrize("rk,linear", [(3, False), (2, False), (3, True)])
def test_wall_steps_match_reference(gpu, ref, rk, linear):
    """Whole CFL steps with cut faces: the reference side takes the
    statements of TimeIntegratorRK2 / RK3::AdvanceOneTimeStep with the
    surface's data set in every ComputeResidual (oracle/ref_harness.cpp,
    m2cref_run_walls)."""
    g, s, mats, V = cases.random_box(14, 11, 9, seed=5, rk=rk)
    s.ebm_recon = int(linear)
    W = wall_faces(g, 120, seed=2)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.set_wall_faces(*W)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    n, t = sol.run(6)
    nr, tr = rc.run_walls(*W, 6)
    assert n == nr == 6 and t == tr
    assert rel_err(inner(sol.download()[0]), inner(rc.get_state()[0])) <= TOL
    sol.close()


def test_wall_residual_with_heat_diffusion_matches_reference(gpu, ref):
    """Heat diffusion ignores the surface in the reference
    (HeatDiffusionOperator::AddDiffusionFluxes takes the data set but does
    not use it): the heat fluxes are added as without cut faces."""
    g, s, _, V = cases.random_box(14, 11, 9, seed=5)
    mats = [abi.material(1.4, 0.0, heat_diffusivity=0.02, cv=2.5, T0=1.0, e0=0.5)]
    W = wall_faces(g, 120, seed=3)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.set_wall_faces(*W)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V)
    assert rel_err(inner(sol.residual()), inner(rc.residual_walls(*W))) <= TOL
    sol.close()


@pytest.mark.parametrize("linear", [False, True])
def test_wall_steps_mixed_track_fp64(gpu, linear):
    out = []
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        g, s, mats, V = cases.random_box(14, 11, 9, seed=5, precision=prec)
        s.ebm_recon = int(linear)
        W = wall_faces(g, 120, seed=1)
        sol = gpu.Solver(g, s, mats)
        sol.upload(V)
        sol.set_wall_faces(*W)
        sol.run(8)
        out.append(inner(sol.download()[0]))
        assert sol.counters()["wall_riemann_calls"] == 8 * 3 * 2 * len(W[0])
        sol.close()
    assert l1_rel(out[1], out[0]) <= 1e-5


def test_wall_faces_refused(gpu):
    g, s, mats, V = cases.random_box(10, 8, 6, seed=5)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    with pytest.raises(gpu.M2CError, match="inside the subdomain"):
        sol.set_wall_faces([(0, 0, 3, 3)])  # the face on the x0 boundary
    with pytest.raises(gpu.M2CError, match="twice"):
        sol.set_wall_faces([(1, 2, 3, 3), (1, 2, 3, 3)])
    with pytest.raises(gpu.M2CError, match="outside"):
        sol.set_wall_faces([(2, 2, 3, 6)])
    sol.close()
    s.ebm_recon = 2
    sol = gpu.Solver(g, s, mats)
    with pytest.raises(gpu.M2CError, match="ebm_recon"):
        sol.set_wall_faces([(0, 3, 3, 3)])
    sol.close()
    visc = gpu.Solver(g, abi.scheme(), [abi.material(1.4, 0.0, mu=1e-3)])
    with pytest.raises(gpu.M2CError, match="viscous"):
        visc.set_wall_faces([(0, 3, 3, 3)])
    visc.close()


def enclosed_block(g, V, lo=(4, 3, 3), hi=(9, 8, 6), speed=0.0, seed=0):
    """A closed box-shaped surface around the cells lo <= (i, j, k) < hi:
    those cells become inactive (material ID = nmat = 1, the dummy state),
    and the faces of the block's boundary are cut, each seen from outside
    with the outward normal and from inside with the inward one."""
    rng = np.random.default_rng(seed)
    ID = np.zeros(V.shape[:3])
    V = V.copy()
    sl = np.s_[lo[2] + 1:hi[2] + 1, lo[1] + 1:hi[1] + 1, lo[0] + 1:hi[0] + 1]
    ID[sl] = 1
    V[sl] = (1.0e-6, 0.0, 0.0, 0.0, 0.0)
    faces, nf, nb = [], [], []
    for d in range(3):
        for side, plane in ((0, lo[d]), (1, hi[d])):
            ranges = [range(lo[a], hi[a]) if a != d else [plane] for a in range(3)]
            for i in ranges[0]:
                for j in ranges[1]:
                    for k in ranges[2]:
                        faces.append((d, i, j, k))
                        n = np.zeros(3)
                        n[d] = -1.0 if side == 0 else 1.0  # the block's outward normal
                        nf.append(n)  # seen from the low cell
                        nb.append(n)
    faces = np.array(faces, np.int32)
    u = rng.uniform(-speed, speed, (len(faces), 3))
    return ID, V, (faces, np.array(nf), u, np.array(nb), u)


@pytest.mark.parametrize("linear,normal", [(False, abi.EBM_NORMAL_MESH), (True, abi.EBM_NORMAL_SURFACE)])
def test_enclosed_inactive_region_matches_reference(gpu, ref, linear, normal):
    """A closed surface around a block of inactive cells (the reference's
    INACTIVE_MATERIAL_ID with VarFcnDummy's fixed state): no slope toward an
    inactive neighbour, constant reconstruction and no checks inside, zero
    fluxes on the inactive side of every cut face, no CFL contribution;
    residual and 6 whole steps."""
    g, s, mats, V = cases.random_box(14, 11, 9, seed=5, rk=3)
    s.ebm_recon = int(linear)
    s.ebm_riemann_normal = normal
    ID, V, W = enclosed_block(g, V, speed=0.2, seed=1)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V, ID)
    sol.set_wall_faces(*W)
    rc = ref.RefCase(g, s, mats)
    rc.set_state(V, ID)
    Rr = inner(rc.residual_walls(*W))
    assert rel_err(inner(sol.residual()), Rr) <= TOL
    n, t = sol.run(6)
    nr, tr = rc.run_walls(*W, 6)
    assert n == nr == 6 and t == tr
    Vg, IDg, _ = sol.download()
    Vr, IDr, _ = rc.get_state()
    assert rel_err(inner(Vg), inner(Vr)) <= TOL
    inside = inner(ID) == 1
    assert np.array_equal(inner(Vg)[inside], np.tile([1.0e-6, 0.0, 0.0, 0.0, 0.0], (inside.sum(), 1)))
    sol.close()


def test_inactive_ids_allowed_only_where_supported(gpu):
    """ID = nmat marks an inactive cell in a context of one material without
    diffusion; elsewhere, and beyond nmat anywhere, the upload is refused."""
    g, s, mats, V = cases.random_box(10, 8, 6, seed=5)
    ID = np.zeros(V.shape[:3])
    ID[3, 3, 3] = 1
    sol = gpu.Solver(g, s, mats)
    sol.upload(V, ID)  # accepted
    ID[3, 3, 4] = 2
    with pytest.raises(gpu.M2CError, match="material ID"):
        sol.upload(V, ID)
    sol.close()
    heat = gpu.Solver(g, s, [abi.material(1.4, 0.0, heat_diffusivity=0.02, cv=2.5)])
    ID[3, 3, 4] = 0
    with pytest.raises(gpu.M2CError, match="material ID"):
        heat.upload(V, ID)
    heat.close()
