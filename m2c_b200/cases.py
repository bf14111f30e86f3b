"""Seeded synthetic workloads with the shapes, sizes and value distributions
of the benchmark configurations (no dataset exists for this path; every
field here is generated from a fixed seed).

Host arrays use the reference's ghosted layout: V[(nz+2),(ny+2),(nx+2),5].
"""
import ctypes as C

import numpy as np

from . import abi


def empty_state(g):
    return np.zeros(abi.ghosted_shape(g, 5))


def sod(n=400, flux=abi.FLUX_HLLC, limiter=abi.LIM_VANALBADA, rk=2, cfl=0.5, precision=abi.PREC_FP64):
    """Sod shock tube: gamma 1.4, [0,1], diaphragm at 0.5, left (1,0,1), right
    (0.125,0,0.1); MUSCL + van Albada, HLLC, RK2, CFL 0.5, t_end 0.2.
    Transmissive ends are Dirichlet INLET/OUTLET ghosts holding the initial
    end states (identical while waves stay inside the tube)."""
    g = abi.grid(n, 1, 1, bc=(abi.BC_INLET, abi.BC_OUTLET) + (abi.BC_SYMMETRY,) * 4,
                 inlet=(1.0, 0.0, 0.0, 0.0, 1.0), outlet=(0.125, 0.0, 0.0, 0.0, 0.1))
    s = abi.scheme(flux=flux, limiter=limiter, rk_order=rk, cfl=cfl, precision=precision)
    mats = [abi.material(1.4, 0.0)]
    V = empty_state(g)
    x = abi.cell_centres(g)[0]
    V[1:-1, 1:-1, 1:-1, 0] = np.where(x < 0.5, 1.0, 0.125)
    V[1:-1, 1:-1, 1:-1, 4] = np.where(x < 0.5, 1.0, 0.1)
    return g, s, mats, V


def fourier_box(n, seed=2024, nmodes=16, kmax=8, amp=0.01, mach_rms=0.3, bc=abi.BC_PERIODIC,
                flux=abi.FLUX_ROE, limiter=abi.LIM_GENMINMOD, minmod=1.0, rk=3, cfl=0.4, precision=abi.PREC_FP64,
                shape=None):
    """3D single-material box on [0,1)^3, ideal gas gamma 1.4: rho = 1 and
    p = 1/1.4 (c = 1) each perturbed by `nmodes` seeded Fourier modes with
    integer wave vectors 1 <= |k| <= kmax (units of 2 pi), relative amplitude
    `amp`; velocity = sum of seeded solenoidal modes scaled to RMS |u| = mach_rms.
    Roe flux (delta 0.2) with generalized minmod (alpha = 1), RK3, CFL 0.4."""
    nx, ny, nz = shape if shape else (n, n, n)
    g = abi.grid(nx, ny, nz, bc=(bc,) * 6)
    s = abi.scheme(flux=flux, limiter=limiter, minmod_coeff=minmod, rk_order=rk, cfl=cfl, precision=precision)
    mats = [abi.material(1.4, 0.0)]
    rng = np.random.default_rng(seed)
    xc, yc, zc = abi.cell_centres(g)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")

    def wavevectors(m):
        out = []
        while len(out) < m:
            k = rng.integers(-kmax, kmax + 1, size=3)
            if 1 <= np.linalg.norm(k) <= kmax:
                out.append(k)
        return out

    def scalar_field():
        f = np.zeros_like(X)
        for k in wavevectors(nmodes):
            ph = rng.uniform(0, 2 * np.pi)
            f += np.cos(2 * np.pi * (k[0] * X + k[1] * Y + k[2] * Z) + ph)
        return f / np.sqrt(nmodes / 2.0)

    rho = 1.0 * (1.0 + amp * scalar_field())
    p = (1.0 / 1.4) * (1.0 + amp * scalar_field())
    u = np.zeros((3,) + X.shape)
    for k in wavevectors(nmodes):
        a = rng.normal(size=3)
        b = np.cross(k, a)  # k x a is orthogonal to k: divergence-free mode
        ph = rng.uniform(0, 2 * np.pi)
        phase = np.cos(2 * np.pi * (k[0] * X + k[1] * Y + k[2] * Z) + ph)
        for d in range(3):
            u[d] += b[d] * phase
    rms = np.sqrt(np.mean(np.sum(u * u, axis=0)))
    u *= mach_rms / rms
    V = empty_state(g)
    V[1:-1, 1:-1, 1:-1, 0] = rho
    V[1:-1, 1:-1, 1:-1, 1] = u[0]
    V[1:-1, 1:-1, 1:-1, 2] = u[1]
    V[1:-1, 1:-1, 1:-1, 3] = u[2]
    V[1:-1, 1:-1, 1:-1, 4] = p
    return g, s, mats, V


def stretched_widths(n, span, kind, seed=0):
    """Cell widths of a non-uniform mesh of n cells over `span`: "grow"
    (geometric, ratio 1.05), "shrink" (ratio 1/1.04) or "jitter" (seeded
    +-25% around uniform)."""
    if kind == "grow":
        w = 1.05 ** np.arange(n)
    elif kind == "shrink":
        w = (1.0 / 1.04) ** np.arange(n)
    else:
        w = 1.0 + np.random.default_rng(seed).uniform(-0.25, 0.25, n)
    return w * (span / w.sum())


def stretch(g, kinds=("grow", "shrink", "jitter"), seed=0):
    """Non-uniform widths on every axis of g with more than one cell."""
    for axis, (n, a, b) in enumerate(((g.nx, g.x0, g.xmax), (g.ny, g.y0, g.ymax), (g.nz, g.z0, g.zmax))):
        if n > 1:
            abi.set_mesh(g, axis, stretched_widths(n, b - a, kinds[axis], seed + axis))
    return g


def random_box(nx, ny, nz, seed=7, bc=(abi.BC_SYMMETRY,) * 6, flux=abi.FLUX_HLLC, limiter=abi.LIM_VANALBADA,
               rk=3, cfl=0.5, precision=abi.PREC_FP64, water=False, nasg=False, mesh=None):
    """Small box with smooth seeded fields plus a density/pressure jump: a
    parity workload that exercises every limiter branch and both wave
    directions. water=True uses the stiffened-gas water of the bubble case
    (gamma 6.12, p_inf 3.43e8 Pa); nasg=True the same states with a
    Noble-Abel stiffened-gas liquid water (gamma 1.19, p_c 7.028e8 Pa,
    b 6.61e-4 m^3/kg, q -1.177788e6 J/kg). mesh: None (uniform) or a
    function applied to the grid before the fields are laid out (e.g.
    stretch)."""
    g = abi.grid(nx, ny, nz, bc=bc, inlet=(1.2, 0.3, 0.0, 0.0, 1.1), outlet=(0.9, 0.0, 0.0, 0.0, 0.8))
    if mesh is not None:
        mesh(g)
    s = abi.scheme(flux=flux, limiter=limiter, rk_order=rk, cfl=cfl, precision=precision)
    rng = np.random.default_rng(seed)
    xc, yc, zc = abi.cell_centres(g)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    if water or nasg:
        mats = [abi.material(6.12, 3.43e8)] if not nasg else \
            [abi.material(1.19, 7.028e8, eos=abi.EOS_NASG, b=6.61e-4, q=-1.177788e6)]
        rho0, p0, u0 = 1000.0, 1.0e5, 50.0
        if g.bc[0] == abi.BC_INLET:
            g.inlet = (C.c_double * 5)(1100.0, 60.0, 0.0, 0.0, 2.0e8)
            g.outlet = (C.c_double * 5)(1000.0, 0.0, 0.0, 0.0, 1.0e5)
    else:
        mats = [abi.material(1.4, 0.0)]
        rho0, p0, u0 = 1.0, 1.0, 0.3
    V = empty_state(g)
    jump = np.where(X + 0.3 * Y + 0.2 * Z < 0.55, 1.0, 0.25)
    smooth = lambda: 0.05 * np.sin(2 * np.pi * (rng.uniform(0.5, 2) * X + rng.uniform(0.5, 2) * Y +
                                                rng.uniform(0.5, 2) * Z) + rng.uniform(0, 6.28))
    V[1:-1, 1:-1, 1:-1, 0] = rho0 * (jump + smooth() + 0.1)
    V[1:-1, 1:-1, 1:-1, 1] = u0 * (0.5 + smooth() * 10)
    V[1:-1, 1:-1, 1:-1, 2] = u0 * (smooth() * 10 - 0.2)
    V[1:-1, 1:-1, 1:-1, 3] = u0 * (smooth() * 10)
    V[1:-1, 1:-1, 1:-1, 4] = p0 * (jump * (1.0 + smooth()) + 0.05)
    if water or nasg:
        V[1:-1, 1:-1, 1:-1, 4] = np.where(jump > 0.5, 1.0e9, 1.0e5) * (1.0 + smooth())
    return g, s, mats, V


def tile_periodic(g, V, reps):
    """Copy of a periodic box tiled reps=(rx,ry,rz) times, with symmetry
    ghosts: the reference (which has no periodic boundary) run on the tiled
    copy reproduces the periodic evolution in the central tile for as many
    steps as the wave of boundary influence needs to cross one tile
    (2 cells per stage)."""
    rx, ry, rz = reps
    G = abi.grid(g.nx * rx, g.ny * ry, g.nz * rz, x=(0.0, (g.xmax - g.x0) * rx), y=(0.0, (g.ymax - g.y0) * ry),
                 z=(0.0, (g.zmax - g.z0) * rz), bc=(abi.BC_SYMMETRY,) * 6)
    inner = V[1:-1, 1:-1, 1:-1]
    T = np.tile(inner, (rz, ry, rx, 1))
    W = np.zeros((G.nz + 2, G.ny + 2, G.nx + 2, 5))
    W[1:-1, 1:-1, 1:-1] = T
    return G, W


def interior(A):
    return A[1:-1, 1:-1, 1:-1]


def stiffened_gas_pair(rng):
    """One seeded stiffened-gas material: gamma in [1.2, 7], p_inf = 0 with
    probability 1/4, else log-uniform in [1e6, 1e9] Pa."""
    gam = rng.uniform(1.2, 7.0)
    pinf = 0.0 if rng.uniform() < 0.25 else 10.0 ** rng.uniform(6.0, 9.0)
    return abi.material(gam, pinf)


def riemann_problems(n, seed=3, nmat_pairs=None):
    """Seeded two-material interface Riemann problems with the state
    distribution of the batched-tube workload: densities log-uniform in
    1..1000 kg/m^3, pressures log-uniform in 1e4..1e9 Pa, velocities uniform
    in +-200 m/s, material 0 on the left and 1 on the right, unit normal x.
    Returns (materials, VL, idl, VR, idr, dirs)."""
    rng = np.random.default_rng(seed)
    mats = [stiffened_gas_pair(rng), stiffened_gas_pair(rng)]
    VL = np.zeros((n, 5))
    VR = np.zeros((n, 5))
    for V in (VL, VR):
        V[:, 0] = 10.0 ** rng.uniform(0.0, 3.0, n)
        V[:, 1] = rng.uniform(-200.0, 200.0, n)
        V[:, 2] = rng.uniform(-20.0, 20.0, n)
        V[:, 3] = rng.uniform(-20.0, 20.0, n)
        V[:, 4] = 10.0 ** rng.uniform(4.0, 9.0, n)
    dirs = np.zeros((n, 3))
    dirs[:, 0] = 1.0
    idl = np.zeros(n, np.int32)
    idr = np.ones(n, np.int32)
    return mats, VL, idl, VR, idr, dirs


def wall_problems(n, seed=7):
    """Seeded one-sided (wall) Riemann problems: the riemann_problems state
    distribution on the fluid side (material 0 or 1 of a stiffened-gas pair),
    a wall velocity uniform in +-300 m/s per component, and a random unit
    normal (so shocks, rarefactions, transonic fans and receding walls all
    occur); about 2% of the problems have the wall's normal velocity equal
    to the fluid's (the trivial branch). Returns (materials, Vm, idm, uwall,
    dirs)."""
    rng = np.random.default_rng(seed)
    mats = [stiffened_gas_pair(rng), stiffened_gas_pair(rng)]
    Vm = np.zeros((n, 5))
    Vm[:, 0] = 10.0 ** rng.uniform(0.0, 3.0, n)
    Vm[:, 1:4] = rng.uniform(-200.0, 200.0, (n, 3))
    Vm[:, 4] = 10.0 ** rng.uniform(4.0, 9.0, n)
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    uwall = rng.uniform(-300.0, 300.0, (n, 3))
    same = rng.random(n) < 0.02
    uwall[same] = Vm[same, 1:4]
    idm = rng.integers(0, 2, n).astype(np.int32)
    return mats, Vm, idm, uwall, dirs


def tube_states(n, rng):
    """Left/right primitive states of n tubes: densities log-uniform in
    1..1000 kg/m^3, velocities uniform in +-200 m/s (along the tube),
    pressures log-uniform in 1e4..1e9 Pa."""
    VL = np.zeros((n, 5))
    VR = np.zeros((n, 5))
    for V in (VL, VR):
        V[:, 0] = 10.0 ** rng.uniform(0.0, 3.0, n)
        V[:, 1] = rng.uniform(-200.0, 200.0, n)
        V[:, 4] = 10.0 ** rng.uniform(4.0, 9.0, n)
    return VL, VR


def tubes(ntubes=4096, seed=11, lmin=100, lmax=2000, reject=None):
    """The batched-tube workload: ntubes independent 1D two-material shock
    tubes on [0, 1] with seeded lengths uniform in lmin..lmax cells, a
    stiffened-gas pair per tube (gamma in [1.2, 7], p_inf 0 with probability
    1/4 else log-uniform in 1e6..1e9 Pa) and the tube_states distribution.
    `reject(mats, VL, VR) -> bool array` flags tubes to redraw (e.g. those
    whose initial Riemann problem the solver cannot bracket); redraws come
    from the same seeded stream. Returns (lens, mats, VL, VR, redrawn)."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(lmin, lmax + 1, ntubes).astype(np.int32)
    mats = []
    for _ in range(ntubes):
        mats += [stiffened_gas_pair(rng), stiffened_gas_pair(rng)]
    VL, VR = tube_states(ntubes, rng)
    redrawn = 0
    for _ in range(20):
        if reject is None:
            break
        bad = np.nonzero(reject(mats, VL, VR))[0]
        if len(bad) == 0:
            break
        redrawn += len(bad)
        for t in bad:
            mats[2 * t] = stiffened_gas_pair(rng)
            mats[2 * t + 1] = stiffened_gas_pair(rng)
        nl, nr = tube_states(len(bad), rng)
        VL[bad], VR[bad] = nl, nr
    return lens, mats, VL, VR, redrawn


def tube_scheme(**kw):
    """Scheme of the batched tubes: HLLC, MUSCL with the van Albada limiter,
    exact interface Riemann solve (MultiPhase flux NUMERICAL, constant
    reconstruction at the interface), RK2, CFL 0.5."""
    d = dict(flux=abi.FLUX_HLLC, limiter=abi.LIM_VANALBADA, rk_order=2, cfl=0.5)
    d.update(kw)
    return abi.scheme(**d)


def tube_case(n, VL, VR):
    """One tube as a reference/3D-path case: an n x 1 x 1 grid on [0, 1],
    INLET ghost holding VL, OUTLET ghost holding VR, symmetry in y and z,
    phi = 0.5 - x, material 1 where phi < 0. Returns (g, ls, V, ID, PHI)."""
    g = abi.grid(n, 1, 1, bc=(abi.BC_INLET, abi.BC_OUTLET) + (abi.BC_SYMMETRY,) * 4,
                 inlet=tuple(VL), outlet=tuple(VR))
    ls = abi.levelset(material_id=1)
    x = abi.cell_centres(g)[0]
    phi = 0.5 - x
    right = phi < 0
    V = empty_state(g)
    V[1, 1, 1:-1] = np.where(right[:, None], np.asarray(VR)[None, :], np.asarray(VL)[None, :])
    ID = np.zeros(abi.ghosted_shape(g))
    ID[1, 1, 1:-1] = right.astype(np.float64)
    PHI = np.zeros(abi.ghosted_shape(g))
    PHI[1, 1, 1:-1] = phi
    return g, ls, V, ID, PHI


WATER = dict(gamma=6.12, p_c=3.43e8)
AIR = dict(gamma=1.4, p_c=0.0)


def post_shock_sg(rho0, p0, p1, gamma, p_c):
    """State behind a right-moving shock of pressure p1 entering still
    stiffened gas (rho0, p0): the Rankine-Hugoniot root of
    e(rho1,p1) - e(rho0,p0) + (p0+p1)/2 (1/rho1 - 1/rho0) = 0 in closed form,
    and u1 = sqrt((p1-p0)(1/rho0 - 1/rho1))."""
    a = (gamma + 1.0) * (p1 + p_c) + (gamma - 1.0) * (p0 + p_c)
    b = (gamma - 1.0) * (p1 + p_c) + (gamma + 1.0) * (p0 + p_c)
    rho1 = rho0 * a / b
    u1 = np.sqrt((p1 - p0) * (1.0 / rho0 - 1.0 / rho1))
    return rho1, u1


def bubble_case(n, nbubbles=1, seed=5, rk=3, cfl=0.4, precision=abi.PREC_FP64, reinit_frequency=10,
                radius=2.0e-3, radii=(0.5e-3, 1.5e-3), shape=None, shock_front=0.005, tile=None, mesh=None):
    """Shock-induced collapse of air bubble(s) in water in a 2 cm cube:
    water is stiffened gas (gamma 6.12, p_inf 3.43e8 Pa, rho 1000, p 1e5),
    air is gamma 1.4 (rho 1.2, p 1e5); a planar shock from the post-shock
    water state at p = 1e9 Pa occupies x < 5 mm; INLET (post-shock) at x0,
    OUTLET (ambient water) at xmax, SYMMETRY on y and z; HLLC + van Albada,
    exact interface Riemann problems, FD3 level set with reinitialisation
    every `reinit_frequency` steps, RK3, CFL 0.4. nbubbles = 1: one bubble of
    radius 2 mm at the centre; otherwise seeded non-overlapping bubbles with
    radii uniform in `radii`, at least two cells apart, fully inside.
    The level set is the signed distance to the nearest bubble surface
    (material 1, air, where phi < 0).

    shock_front: x of the shock front in metres, or "contact": the moment
    the front, coming from x = 5 mm through still water, reaches the
    nearest bubble. Ahead of the front the water is uniform and at rest, so
    that moment's state is this initial state with the front two cells
    upstream of the nearest bubble surface.

    tile: None, or (shape, origin) of a sub-box of the grid in cells, e.g.
    ((48, 48, 48), (i0, j0, k0)): the same state restricted to those cells
    (same cell size), with the domain's boundary conditions on faces that
    lie on the domain boundary and symmetry walls on the others. Used to
    run bounded samples of a large case on the CPU reference.

    mesh: None (uniform) or a function applied to the grid before the
    fields are laid out (e.g. stretch)."""
    L = 0.02
    nx, ny, nz = shape if shape else (n, n, n)
    rho1, u1 = post_shock_sg(1000.0, 1.0e5, 1.0e9, **WATER)
    post = (rho1, u1, 0.0, 0.0, 1.0e9)
    bc = [abi.BC_INLET, abi.BC_OUTLET] + [abi.BC_SYMMETRY] * 4
    lo, hi = (0.0, 0.0, 0.0), (L, L, L)
    cells = (nx, ny, nz)
    if tile is not None:
        ext, org = tile
        h3 = (L / nx, L / ny, L / nz)
        lo = tuple(org[a] * h3[a] for a in range(3))
        hi = tuple((org[a] + ext[a]) * h3[a] for a in range(3))
        for a, full in enumerate((nx, ny, nz)):
            if org[a] > 0:
                bc[2 * a] = abi.BC_SYMMETRY
            if org[a] + ext[a] < full:
                bc[2 * a + 1] = abi.BC_SYMMETRY
        cells = tuple(ext)
    g = abi.grid(*cells, x=(lo[0], hi[0]), y=(lo[1], hi[1]), z=(lo[2], hi[2]), bc=tuple(bc), inlet=post,
                 outlet=(1000.0, 0.0, 0.0, 0.0, 1.0e5))
    if mesh is not None:
        mesh(g)
    s = abi.scheme(flux=abi.FLUX_HLLC, limiter=abi.LIM_VANALBADA, rk_order=rk, cfl=cfl, precision=precision)
    mats = [abi.material(**WATER), abi.material(**AIR)]
    ls = abi.levelset(material_id=1, reinit_frequency=reinit_frequency)
    xc, yc, zc = abi.cell_centres(g)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    h = L / nx
    if nbubbles == 1:
        centres = [(L / 2, L / 2, L / 2)]
        rads = [radius]
    else:
        rng = np.random.default_rng(seed)
        centres, rads = [], []
        tries = 0
        while len(centres) < nbubbles and tries < 100000:
            tries += 1
            r = rng.uniform(*radii)
            c = rng.uniform(0.0075 + r + 2 * h, L - r - 2 * h, size=3)  # downstream of the shock front
            c[1] = rng.uniform(r + 2 * h, L - r - 2 * h)
            c[2] = rng.uniform(r + 2 * h, L - r - 2 * h)
            if all(np.linalg.norm(c - np.array(c2)) >= r + r2 + 2 * h for c2, r2 in zip(centres, rads)):
                centres.append(tuple(c))
                rads.append(r)
    phi = np.full(X.shape, np.inf)
    for c, r in zip(centres, rads):
        phi = np.minimum(phi, np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r)
    V = empty_state(g)
    ID = np.zeros(abi.ghosted_shape(g))
    PHI = np.zeros(abi.ghosted_shape(g))
    inner = np.s_[1:-1, 1:-1, 1:-1]
    if shock_front == "contact":
        shock_front = min(c[0] - r for c, r in zip(centres, rads)) - 2 * h
    shocked = X < shock_front
    V[inner + (0,)] = np.where(shocked, rho1, 1000.0)
    V[inner + (1,)] = np.where(shocked, u1, 0.0)
    V[inner + (4,)] = np.where(shocked, 1.0e9, 1.0e5)
    air = phi < 0
    V[inner + (0,)] = np.where(air, 1.2, V[inner + (0,)])
    V[inner + (1,)] = np.where(air, 0.0, V[inner + (1,)])
    V[inner + (4,)] = np.where(air, 1.0e5, V[inner + (4,)])
    ID[inner] = np.where(air, 1.0, 0.0)
    PHI[inner] = phi
    return g, s, mats, ls, V, ID, PHI
