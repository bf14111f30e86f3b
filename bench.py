"""Benchmark: cell-updates/s per RK step of the explicit finite-volume step.

Headline workload (one GPU holds it): the 384^3 two-material bubble cluster.
A 2 cm cube of water (stiffened gas, gamma 6.12, p_inf 3.43e8 Pa, 1000
kg/m^3, 1e5 Pa) holds 16 seeded air bubbles (gamma 1.4, 1.2 kg/m^3, radii
0.5-1.5 mm); a planar shock carrying the post-shock water state at 1e9 Pa
runs in from x = 0 (INLET post-shock, OUTLET ambient water, symmetry on the
other faces). HLLC + van Albada MUSCL, exact two-material Riemann problems at
the interface faces, FD3 level set with reinitialisation every 10 steps,
RK3, CFL 0.4. The timed window starts when the shock front reaches the
nearest bubble (the front coming from x = 5 mm meets only still water on its
way there, so that moment's state is the initial one with the front two
cells upstream of the nearest bubble surface): the timed steps solve the
interface Riemann problems of the bubbles the shock is hitting. The headline
runs the mixed path (FP32 reconstruction/flux; FP64 state, water pressure
recovery and Riemann solves); the FP64 path runs the same steps from the
same state and the mixed path's error against it is reported.

A "step" is one full RK3 step (3 interface Riemann pre-passes, 3 fused
stage launches, 3 level-set stages, ID and state update, amortised
reinitialisation, device clock). Inputs are larger than L2 (5 x 453 MB per
state array), so no explicit flush is needed between steps.

Multi-GPU: the path does not shard; --gpus N runs N independent replicas
(one per GPU, "scaling": "weak"), value = all cells updated / max time over
ranks.

--impl reference: the reference's own CPU implementation (the unmodified
sources built with single-rank shims under oracle/_ref), run on the host
cores as independent processes, each advancing one 48^3 tile of the same
384^3 state (same cell size and physics; the domain's boundary rule on
faces on the domain boundary, symmetry walls on the others) by one RK3 step
per benchmark step; the tiles are a seeded sample of the 512 tiles.

Extras (rank 0 at N = 1, skipped by --only-headline), under "extras": the
256^3 single-material periodic box (mixed vs FP64, with its own roofline,
CPU figure and end-to-end figure), the 192^3 single bubble over 500 steps,
the 4096 batched two-material tubes (CUDA-graph replay, autotuned tiles,
with and without the learned warm start), a 192^3 box cut by a resting
plane (one-sided Riemann problems at the cut faces), and the learned warm
start's evaluations and iterations saved on held-out interface problems and
on the cluster (network in m2c_b200/data/warmstart_mlp.npz).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per RK step (RK3, 384^3 two-material bubble cluster, mixed FP32/FP64)"
UNIT = "cell-updates/s"
CLUSTER_N = 384
CLUSTER_BUBBLES = 16
TILE = 48
BOX_SAMPLE_N = 48

# DRAM bytes (read + write) per cell of one launch of the two-material FP32
# stage kernel, from an ncu capture of the same kernel on the 192^3 cluster
# (stage-1 launch, 138 B per cell; the capture and its command are under
# profiles/).
STAGE_MULTI_TRAFFIC_B_PER_CELL = 138.0
# The same for the single-material FP32 stage kernel (stage-2 launch, 160^3
# periodic box).
STAGE_SINGLE_TRAFFIC_B_PER_CELL = 164.9
# Algorithmic bytes of one stage launch: the FP64 conserved state of an RK3
# step (8 five-vectors, 320 B per cell) over its three stages, plus, with two
# materials, the material-ID byte the stage reads.
ALG_STAGE_SINGLE = 320.0 / 3.0
ALG_STAGE_MULTI = 320.0 / 3.0 + 1.0
# Algorithmic bytes of a two-material RK3 step per cell: 320 B state, 64 B
# level set (8 phi values), 3 ID bytes.
ALG_STEP_MULTI = 387.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=CLUSTER_N, help="cluster grid size (cells per axis)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64 leg of the headline")
    p.add_argument("--only-headline", action="store_true",
                   help="skip the extra workloads (periodic box, single bubble, batched tubes, warm start)")
    p.add_argument("--bubble", type=int, default=0, metavar="N",
                   help="run only the cluster workload at N^3, mixed then FP64, and print its JSON (profiling)")
    p.add_argument("--box", type=int, default=0, metavar="N",
                   help="run only the periodic-box workload at N^3 and print its JSON (profiling)")
    p.add_argument("--plane", type=int, default=0, metavar="N",
                   help="run only the box cut by a resting plane at N^3 and print its JSON (profiling)")
    return p.parse_args()


def config(n, world):
    return {"workload": f"bubble cluster {n}^3: 16 air bubbles (0.5-1.5 mm) in water, 2 cm cube, 1 GPa planar "
                        f"shock timed from its first contact with a bubble; HLLC + van Albada, exact interface "
                        f"Riemann, FD3 level set, reinitialisation every 10 steps, RK3, CFL 0.4",
            "cells": n ** 3, "flush": "inputs larger than L2 (no explicit flush)",
            "parallelism": f"replicas x{world}"}


def cluster_case(n, precision, tile=None):
    from m2c_b200 import cases
    return cases.bubble_case(n, nbubbles=CLUSTER_BUBBLES, precision=precision, shock_front="contact", tile=tile)


# --------------------------------------------------------------------------
# CPU reference legs (the reference arm and the cpu_baseline): independent
# processes, spawned before any GPU work
# --------------------------------------------------------------------------
def _quiet():
    # the reference prints mesh statistics on stdout: keep the JSON line alone there
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, ROOT)


def cluster_tiles(n, count, seed=7):
    """A seeded sample of `count` of the (n/48)^3 tiles of the cluster grid
    (origins in cells)."""
    import numpy as np
    m = n // TILE
    order = np.random.default_rng(seed).permutation(m ** 3)[:count]
    return [(int(t % m) * TILE, int((t // m) % m) * TILE, int(t // (m * m)) * TILE) for t in order]


def _cpu_cluster_worker(args):
    n, origin, steps = args
    _quiet()
    from m2c_b200 import abi
    from oracle import ref
    g, s, mats, ls, V, ID, PHI = cluster_case(n, abi.PREC_FP64, tile=((TILE,) * 3, origin))
    c = ref.RefCase(g, s, mats, ls)
    c.set_state(V, ID, PHI)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        c.run(1)
        times.append(time.perf_counter() - t0)
    interface = bool(((ID[1:-1, 1:-1, 1:-1] > 0).any()))
    p = V[1:-1, 1:-1, 1:-1, 4]
    shocked = bool((p > 1.0e8).any() and (p < 1.0e8).any())
    return times, interface, shocked


def cpu_reference_cluster(n, steps, warmup, cores=None):
    """The reference on `cores` tiles of the cluster state, one process per
    tile; per benchmark step the slowest process's step time. Returns
    (per-step seconds, cells per step, cores, sample text)."""
    import multiprocessing as mp
    cores = cores or min(os.cpu_count() or 1, 64)
    tiles = cluster_tiles(n, cores)
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_cpu_cluster_worker, [(n, t, warmup + steps) for t in tiles])
    per_step = [max(r[0][warmup + w] for r in res) for w in range(steps)]
    nif = sum(1 for r in res if r[1])
    nsh = sum(1 for r in res if r[2])
    sample = (f"{cores} processes x one {TILE}^3 tile of the {n}^3 cluster state (seeded sample of "
              f"{(n // TILE) ** 3} tiles; {nif} hold bubble cells, {nsh} the shock front), {steps} RK3 steps "
              f"each after {warmup}, FP64, reinitialisation every 10 steps")
    return per_step, cores * TILE ** 3, cores, sample


def _cpu_box_worker(args):
    n, steps, seed = args
    _quiet()
    from m2c_b200 import abi, cases
    from oracle import ref
    g, s, mats, V = cases.fourier_box(n, seed=seed, bc=abi.BC_SYMMETRY)
    c = ref.RefCase(g, s, mats)
    c.set_state(V)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        c.run(1)
        times.append(time.perf_counter() - t0)
    return times


def cpu_reference_box(steps, warmup, cores=None):
    import multiprocessing as mp
    cores = cores or min(os.cpu_count() or 1, 64)
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_cpu_box_worker, [(BOX_SAMPLE_N, warmup + steps, 100 + r) for r in range(cores)])
    per_step = [max(r[w + warmup] for r in res) for w in range(steps)]
    return {"value": cores * BOX_SAMPLE_N ** 3 * steps / sum(per_step), "unit": UNIT, "cores": cores,
            "kind": "reference",
            "sample": f"{cores} processes x one {BOX_SAMPLE_N}^3 box (symmetry walls), {steps} RK3 steps each "
                      f"after {warmup}"}


# --------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# --------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) > 8:
                for q, name in enumerate(names):
                    if "Active" in r[5 + q] and "Not" not in r[5 + q]:
                        reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _l1(a, b):
    import numpy as np
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


# --------------------------------------------------------------------------
# the headline: the bubble cluster, mixed, in its contact window
# --------------------------------------------------------------------------
def cluster_run(n, steps, warmup, with_fp64=True, clocks=None, dist=None):
    """Mixed path on the cluster: `warmup` steps, then `steps` timed steps,
    then 2 steps with the stage launches timed one by one. With with_fp64,
    the FP64 path runs the same steps from the same state (timed alike) and
    the two are compared. Returns a dict (and keeps the mixed solver open
    under "_solver" with the case arrays under "_case" for the e2e leg)."""
    import numpy as np
    from m2c_b200 import abi, gpu
    cells = n ** 3
    case = cluster_case(n, abi.PREC_MIXED)
    g, s, mats, ls, V, ID, PHI = case
    sol = gpu.Solver(g, s, mats, ls)
    sol.upload(V, ID, PHI)
    sol.time_steps(warmup)
    c0 = sol.counters()
    if dist:
        dist.barrier()
    if clocks:
        clocks.start()
    ms, launches = sol.time_steps(steps)
    clk = clocks.stop() if clocks else None
    c1 = sol.counters()
    stage_ms, nstage, _ = sol.profile_stages(2)
    peak, _ = measured_peak()
    d = {k: (c1[k] - c0[k]) / steps for k in c1}
    out = {"ms": ms, "launches": launches, "clocks": clk,
           "per_step": {"riemann_calls": d["riemann_calls"], "riemann_nontrivial": d["riemann_nontrivial"],
                        "riemann_iterations": d["riemann_iterations"],
                        "riemann_evaluations": d["riemann_evaluations"],
                        "cells_changed_material_unresolved": d["unresolved_cells"],
                        "reinitialisations": d["reinit_calls"], "kernel_launches": launches / steps},
           "stage_avg_ms": stage_ms / nstage, "stage_launches_profiled": nstage,
           "hbm_frac_step": ALG_STEP_MULTI * cells * steps / (ms / 1e3) / 1e9 / peak}
    if with_fp64:
        s64 = abi.scheme(**{f: getattr(s, f) for f, _ in abi.Scheme._fields_})
        s64.precision = abi.PREC_FP64
        b = gpu.Solver(g, s64, mats, ls)
        b.upload(V, ID, PHI)
        b.time_steps(warmup)
        ms64, _ = b.time_steps(steps)
        st64, n64, _ = b.profile_stages(2)  # the same step count as the mixed leg
        Vm, Im, Pm = sol.download()
        Vf, If, Pf = b.download()
        b.close()
        inner = np.s_[1:-1, 1:-1, 1:-1]
        vm, vf = Vm[inner].reshape(-1, 5), Vf[inner].reshape(-1, 5)
        vel = float(np.linalg.norm(vm[:, 1:4] - vf[:, 1:4], axis=1).sum() /
                    np.linalg.norm(vf[:, 1:4], axis=1).sum())
        linf = lambda a, c: float(np.abs(a - c).max() / np.abs(c).max())
        out["fp64"] = {"value": cells * steps / (ms64 / 1e3), "ms_per_step": ms64 / steps,
                       "hbm_frac_step": ALG_STEP_MULTI * cells * steps / (ms64 / 1e3) / 1e9 / peak,
                       "stage_avg_ms": st64 / n64,
                       "stage_hbm_frac": ALG_STAGE_MULTI * cells / (st64 / n64 / 1e3) / 1e9 / peak,
                       "mixed_speedup": ms64 / ms,
                       "mixed_vs_fp64_rel_L1": {"rho": _l1(vm[:, 0], vf[:, 0]), "velocity": vel,
                                                "p": _l1(vm[:, 4], vf[:, 4]),
                                                "phi": _l1(Pm[inner].ravel(), Pf[inner].ravel())},
                       "mixed_vs_fp64_rel_Linf": {"rho": linf(vm[:, 0], vf[:, 0]), "p": linf(vm[:, 4], vf[:, 4])},
                       "material_id_mismatch": int((Im[inner] != If[inner]).sum()),
                       "phi_sign_mismatch": int(((Pm[inner] < 0) != (Pf[inner] < 0)).sum()),
                       "after_steps": warmup + steps + 2}
        del Vm, Im, Pm, Vf, If, Pf
    out["_solver"] = sol
    out["_case"] = case
    return out


def cluster_e2e(sol, case, steps, dist=None):
    """The same metric through the public C-ABI: the host state in the
    reference's ghosted AoS layout (V, material ID and phi) in pinned memory,
    m2cg_upload_state + m2cg_run(1) + m2cg_download_state per step."""
    import torch
    g, s, mats, ls, V, ID, PHI = case
    pin = lambda a: torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
    Vh, Ih, Ph = pin(V), pin(ID), pin(PHI)
    Vh[...] = V
    Ih[...] = ID
    Ph[...] = PHI
    Vo, Io, Po = pin(V), pin(ID), pin(PHI)
    sol.upload(Vh, Ih, Ph)
    sol.run(1)
    sol.download(out_V=Vo, out_ID=Io, out_phi=Po)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        sol.upload(Vh, Ih, Ph)
        sol.run(1)
        sol.download(out_V=Vo, out_ID=Io, out_phi=Po)
    te = time.perf_counter() - t0
    return te, int(Vh.nbytes + Ih.nbytes + Ph.nbytes)


# --------------------------------------------------------------------------
# extra workloads (rank 0, one GPU): the other configurations of the path
# --------------------------------------------------------------------------
def extra_box(n=256, steps=20, warmup=3, cpu=True):
    """The 256^3 single-material periodic box (ideal gas, Roe + generalized
    minmod, RK3, CFL 0.4), mixed vs FP64, with its stage kernel's roofline,
    a reference-CPU figure and an end-to-end figure."""
    import numpy as np
    import torch
    from m2c_b200 import abi, cases, gpu
    cells = n ** 3
    g, s, mats, V = cases.fourier_box(n, precision=abi.PREC_MIXED, seed=2024)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.time_steps(warmup)
    ms, _ = sol.time_steps(steps)
    stage_ms, nstage, _ = sol.profile_stages(3)
    avg = stage_ms / nstage
    peak, peak_kind = measured_peak()
    achieved = ALG_STAGE_SINGLE * cells / (avg / 1e3) / 1e9
    s64 = abi.scheme(**{f: getattr(s, f) for f, _ in abi.Scheme._fields_})
    s64.precision = abi.PREC_FP64
    b = gpu.Solver(g, s64, mats)
    b.upload(V)
    b.time_steps(warmup)
    ms64, _ = b.time_steps(steps)
    st64, n64, _ = b.profile_stages(3)
    b.close()
    a = gpu.Solver(g, s, mats)
    a.upload(V)
    c = gpu.Solver(g, s64, mats)
    c.upload(V)
    a.run(steps)
    c.run(steps)
    Va, _, _ = a.download()
    Vb, _, _ = c.download()
    a.close()
    c.close()
    ia, ib = Va[1:-1, 1:-1, 1:-1].reshape(-1, 5), Vb[1:-1, 1:-1, 1:-1].reshape(-1, 5)
    l1 = (np.abs(ia - ib).sum(0) / np.abs(ib).sum(0)).tolist()
    Vh = torch.empty(V.shape, dtype=torch.float64, pin_memory=True).numpy()
    Vh[...] = V
    Vo = torch.empty(V.shape, dtype=torch.float64, pin_memory=True).numpy()
    sol.upload(Vh)
    sol.run(1)
    sol.download(out_V=Vo, with_id=False)
    ne = 5
    t0 = time.perf_counter()
    for _ in range(ne):
        sol.upload(Vh)
        sol.run(1)
        sol.download(out_V=Vo, with_id=False)
    te = time.perf_counter() - t0
    sol.close()
    out = {"workload": f"periodic box {n}^3, ideal gas, Roe + generalized minmod, RK3, CFL 0.4",
           "mixed": {"cell_updates_per_s": cells * steps / (ms / 1e3), "ms_per_step": ms / steps},
           "fp64": {"cell_updates_per_s": cells * steps / (ms64 / 1e3), "ms_per_step": ms64 / steps,
                    "stage_avg_ms": st64 / n64,
                    "stage_hbm_frac": ALG_STAGE_SINGLE * cells / (st64 / n64 / 1e3) / 1e9 / peak},
           "mixed_speedup": ms64 / ms,
           "mixed_vs_fp64_rel_L1": dict(zip(["rho", "u", "v", "w", "p"], l1)),
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_kind": peak_kind,
                        "traffic": STAGE_SINGLE_TRAFFIC_B_PER_CELL * cells,
                        "kernel": "m2c::stage_kernel<float,16,ROE,single>", "avg_launch_ms": avg,
                        "alg_bytes_per_launch": ALG_STAGE_SINGLE * cells},
           "e2e": {"value": cells * ne / te, "unit": UNIT, "h2d_bytes_per_step": int(Vh.nbytes),
                   "d2h_bytes_per_step": int(Vo.nbytes), "steps": ne}}
    if cpu:
        out["cpu_reference"] = cpu_reference_box(6, 1)
    return out


def extra_walls(n=192, steps=20, warmup=3):
    """A flat surface across the periodic box (ideal gas, Roe + generalized
    minmod, RK3): every x face of the plane i = n/2 cut, the surface at rest
    (m2cg_set_wall_faces; per stage two one-sided exact Riemann problems per
    cut face, then the wall branch of the face fluxes). Time per step with
    and without the surface, mixed and FP64."""
    import numpy as np
    from m2c_b200 import abi, cases, gpu
    jj, kk = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    faces = np.stack([np.zeros(n * n, np.int32), np.full(n * n, n // 2, np.int32), jj.ravel().astype(np.int32),
                      kk.ravel().astype(np.int32)], axis=1)
    out = {"workload": f"periodic box {n}^3 cut by a resting plane (x faces at i = {n // 2}, {n * n} cut faces), "
                       f"Roe + generalized minmod, RK3"}
    for prec, name in ((abi.PREC_MIXED, "mixed"), (abi.PREC_FP64, "fp64")):
        g, s, mats, V = cases.fourier_box(n, precision=prec, seed=2024)
        r = {}
        for walls in (False, True):
            sol = gpu.Solver(g, s, mats)
            sol.upload(V)
            if walls:
                sol.set_wall_faces(faces)
            sol.time_steps(warmup)
            c0 = sol.counters()
            ms, _ = sol.time_steps(steps)
            c1 = sol.counters()
            sol.close()
            key = "with_plane" if walls else "without"
            r[key] = {"ms_per_step": ms / steps, "cell_updates_per_s": n ** 3 * steps / (ms / 1e3)}
            if walls:
                r[key]["wall_riemann_calls_per_step"] = (c1["wall_riemann_calls"] - c0["wall_riemann_calls"]) / steps
                r[key]["wall_riemann_errors"] = c1["riemann_errors"] - c0["riemann_errors"]
        r["plane_cost_ms_per_step"] = r["with_plane"]["ms_per_step"] - r["without"]["ms_per_step"]
        out[name] = r
    return out


def extra_bubble(n=192, nbubbles=1, steps=500, warmup=3):
    """Single bubble (192^3, 500 steps), mixed vs FP64: cell-updates/s, HBM
    fraction of the algorithmic bytes, and the mixed path's error against the
    FP64 path after the same steps."""
    import numpy as np
    from m2c_b200 import abi, cases, gpu
    res = {}
    for prec in (abi.PREC_MIXED, abi.PREC_FP64):
        g, s, mats, ls, V, ID, PHI = cases.bubble_case(n, nbubbles=nbubbles, precision=prec)
        sol = gpu.Solver(g, s, mats, ls)
        sol.upload(V, ID, PHI)
        del V, ID, PHI
        sol.time_steps(warmup)
        c0 = sol.counters()
        ms, _ = sol.time_steps(steps)
        c1 = sol.counters()
        Vd, IDd, Pd = sol.download()
        res[prec] = (ms, Vd[1:-1, 1:-1, 1:-1].reshape(-1, 5), IDd[1:-1, 1:-1, 1:-1].ravel(),
                     Pd[1:-1, 1:-1, 1:-1].ravel(), {k: c1[k] - c0[k] for k in c1})
        sol.close()
        del Vd, IDd, Pd
    cells = n ** 3
    (mm, Vm, Im, Pm, cm), (mf, Vf, If, Pf, cf) = res[abi.PREC_MIXED], res[abi.PREC_FP64]
    vel = float(np.linalg.norm(Vm[:, 1:4] - Vf[:, 1:4], axis=1).sum() / np.linalg.norm(Vf[:, 1:4], axis=1).sum())
    alg = ALG_STEP_MULTI * cells * steps
    peak, _ = measured_peak()
    return {"workload": f"single bubble {n}^3, radius 2 mm at the centre, HLLC + van Albada, exact interface "
                        f"Riemann, FD3 level set with reinitialisation every 10 steps, RK3, CFL 0.4",
            "steps": steps, "after_warmup_steps": warmup,
            "mixed": {"cell_updates_per_s": cells * steps / (mm / 1e3), "ms_per_step": mm / steps,
                      "hbm_frac": alg / (mm / 1e3) / 1e9 / peak},
            "fp64": {"cell_updates_per_s": cells * steps / (mf / 1e3), "ms_per_step": mf / steps,
                     "hbm_frac": alg / (mf / 1e3) / 1e9 / peak},
            "mixed_speedup": mf / mm,
            "mixed_vs_fp64_rel_L1": {"rho": _l1(Vm[:, 0], Vf[:, 0]), "velocity": vel, "p": _l1(Vm[:, 4], Vf[:, 4])},
            "material_id_mismatch": int((Im != If).sum()), "phi_sign_mismatch": int(((Pm < 0) != (Pf < 0)).sum()),
            "riemann_calls_per_step_mixed": cm["riemann_calls"] / steps,
            "riemann_nontrivial_per_step_mixed": cm["riemann_nontrivial"] / steps}


def extra_tubes(ntubes=4096, steps=200, mlp=None):
    """Batched 1D two-material tubes (one graph-replayed step sequence,
    autotuned tiles); tubes whose initial interface problem fails are
    redrawn (counted)."""
    from m2c_b200 import cases, gpu
    s = cases.tube_scheme()
    lens, mats, VL, VR, redrawn = cases.tubes(ntubes, seed=11, reject=gpu.tube_rejects(s))
    out = {"workload": f"{ntubes} two-material shock tubes, 100-2000 cells, HLLC + van Albada, exact interface "
                       f"Riemann, RK2, CFL 0.5, {steps} steps", "cells": int(lens.sum()),
           "redrawn_at_t0": int(redrawn)}
    peak, _ = measured_peak()
    # after the first steps most interface problems are near-acoustic, where
    # the acoustic estimate already starts within one iteration; gate 0.03
    # ignores proposals that close to it
    for label, net, gate in (("cold", None, 0.0), ("warm_start", mlp, 0.0), ("warm_start_gate_0.03", mlp, 0.03)):
        if label != "cold" and net is None:
            continue
        s.riem_warm_gate = gate
        b = gpu.Batch(s, lens, mats, VL, VR)
        if net is not None:
            b.set_mlp(net)
        ms = b.time_steps(steps, check_errors=False)
        c = b.counters()
        # RK2: 5 FP64 five-vectors (200 B) + 5 phi values (40 B) per cell and step
        out[label] = {"cell_updates_per_s": b.ncell * steps / (ms / 1e3), "ms_per_step": ms / steps,
                      "hbm_frac": 240.0 * b.ncell * steps / (ms / 1e3) / 1e9 / peak,
                      "tuning": b.tuning(), "failed_tubes": int((b.tube_errors() != 0).sum()),
                      "riemann_calls": c["riemann_calls"], "riemann_iterations": c["riemann_iterations"],
                      "riemann_evaluations": c["riemann_evaluations"]}
        b.close()
    return out


def load_warmstart():
    """The trained warm-start network committed with the package (trained on
    the GPU by m2c_b200.warmstart), or None."""
    from m2c_b200 import warmstart
    p = os.path.join(ROOT, "m2c_b200", "data", "warmstart_mlp.npz")
    return warmstart.load(p) if os.path.exists(p) else None


def extra_warm_start(net, n=100_000):
    """Star-state evaluations and secant iterations of the exact interface
    solve with and without the learned warm start, on held-out problems of
    the tube distribution; the converged states must agree to the solver's
    tolerance."""
    import numpy as np
    from m2c_b200 import abi, warmstart
    s = abi.scheme()
    mats, VL, VR, dirs = warmstart.sample_problems(n, seed=123)
    cold = warmstart.solve(s, mats, VL, VR, dirs)
    t0 = time.perf_counter()
    warm = net.predict_pairs(mats, VL, VR, dirs)
    t_inf = time.perf_counter() - t0
    hot = warmstart.solve(s, mats, VL, VR, dirs, warm=warm)
    both = (cold["err"] == 0) & (hot["err"] == 0)
    g = mats["gamma"]
    pc = mats["p_c"]
    sh = np.minimum(pc[0::2], pc[1::2])  # the proposal's error on the shifted scale p + min(pinf)
    ok = both & (cold["Vsm"][:, 4] + sh > 0) & np.isfinite(warm) & (warm + sh > 0)
    rel = np.abs(np.log((warm[ok] + sh[ok]) / (cold["Vsm"][ok, 4] + sh[ok])))
    cl = np.sqrt(g[0::2] * (VL[:, 4] + pc[0::2]) / VL[:, 0])
    cr = np.sqrt(g[1::2] * (VR[:, 4] + pc[1::2]) / VR[:, 0])
    du = (np.abs(hot["Vsm"][:, 1] - cold["Vsm"][:, 1]) / np.maximum(cl, cr))[both]
    # what a proposal of a given accuracy would save: the cold solution's p*
    # perturbed by a log-normal error of width eps, through the same solver
    curve = {}
    okc = (cold["err"] == 0) & (cold["Vsm"][:, 4] > 0)
    rng = np.random.default_rng(5)
    for eps in (0.0, 1e-5, 1e-4, 1e-3, 6e-3):
        prop = np.where(okc, cold["Vsm"][:, 4] * np.exp(eps * rng.normal(size=n)), np.nan)
        r = warmstart.solve(s, mats, VL, VR, dirs, warm=prop)
        m = okc & (r["err"] == 0)
        curve[f"{eps:g}"] = {"iteration_ratio": float(cold["iters"][m].mean() / r["iters"][m].mean()),
                             "evaluation_ratio": float(cold["evals"][m].mean() / r["evals"][m].mean())}
    return {"problems": n, "solved_both": int(both.sum()),
            "proposal_error_vs_gain": curve,
            "evaluations_cold": float(cold["evals"][both].mean()), "evaluations_warm": float(hot["evals"][both].mean()),
            "evaluation_ratio": float(cold["evals"][both].mean() / hot["evals"][both].mean()),
            "iterations_cold": float(cold["iters"][both].mean()), "iterations_warm": float(hot["iters"][both].mean()),
            "iteration_ratio": float(cold["iters"][both].mean() / hot["iters"][both].mean()),
            "prediction_abs_shifted_log_error_median": float(np.median(rel)),
            "star_velocity_diff_over_c_p99": float(np.percentile(du, 99)),
            "inference_s_host_call": t_inf}


def extra_cluster_warm_start(net, n=CLUSTER_N, steps=10):
    """The headline workload (the cluster in its shock-bubble window) with
    and without the learned warm start on the interface Riemann problems of
    every stage (m2cg_set_mlp): per-step secant iterations and star-state
    evaluations, time per step, and the largest relative state difference to
    the cold run after `steps` steps. With gate 0 every proposal is used;
    with gate 0.03 proposals within 3% (shifted log distance) of the
    acoustic estimate are ignored."""
    import numpy as np
    from m2c_b200 import abi, gpu
    out, ref = {}, None
    for name, gate in (("cold", None), ("warm", 0.0), ("warm_gate_0.03", 0.03)):
        g, s, mats, ls, V, ID, PHI = cluster_case(n, abi.PREC_MIXED)
        if gate is not None:
            s.riem_warm_gate = gate
        sol = gpu.Solver(g, s, mats, ls)
        sol.upload(V, ID, PHI)
        if gate is not None:
            sol.set_mlp(net)
        c0 = sol.counters()
        ms, _ = sol.time_steps(steps)
        c1 = sol.counters()
        Vr, Ir, Pr = sol.download()
        sol.close()
        d = {k: (c1[k] - c0[k]) / steps for k in ("riemann_calls", "riemann_nontrivial", "riemann_iterations",
                                                   "riemann_evaluations")}
        d["ms_per_step"] = ms / steps
        inner = np.s_[1:-1, 1:-1, 1:-1]
        if ref is None:
            ref = (Vr[inner].copy(), Ir[inner].copy())
        else:
            scale = np.abs(ref[0]).reshape(-1, 5).max(axis=0)
            d["max_state_diff_over_scale"] = [float(x) for x in
                                              (np.abs(Vr[inner] - ref[0]).reshape(-1, 5).max(axis=0) / scale)]
            d["material_id_mismatch"] = int((Ir[inner] != ref[1]).sum())
        out[name] = d
        del Vr, Ir, Pr
    return {"workload": f"bubble cluster {n}^3, {steps} steps from first shock-bubble contact", **out}


def max_over_ranks(x, dist, device):
    """The slowest rank's time (the replicas' job ends with it)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(cells_per_rank, world, steps, ms_max):
    """Whole-job cell-updates/s of `world` replicas: all cells updated over
    the slowest rank's time."""
    return world * cells_per_rank * steps / (ms_max / 1000.0)


def reference_arm(args, world):
    per_step, ccells, cores, sample = cpu_reference_cluster(args.n, args.steps, args.warmup)
    tot = sum(per_step)
    v = ccells * len(per_step) / tot
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * tot / len(per_step), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded bubble cluster)",
        "config": config(args.n, world), "impl": "reference",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, world)
        return

    if args.box:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(extra_box(n=args.box, steps=args.steps, warmup=args.warmup, cpu=False)))
        return
    if args.plane:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(extra_walls(n=args.plane, steps=args.steps, warmup=args.warmup)))
        return

    # CPU baseline first (spawned processes, before any GPU work), rank 0, N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.bubble:
        try:
            per_step, ccells, cores, sample = cpu_reference_cluster(args.n, 12, 1)
            cpu = {"value": ccells * len(per_step) / sum(per_step), "unit": UNIT, "cores": cores,
                   "kind": "reference", "sample": sample}
        except Exception as e:  # the oracle build is missing on this host
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    from m2c_b200 import gpu
    gpu.set_device(local if world > 1 else 0)
    n = args.bubble or args.n
    cells = n ** 3

    clocks = Clocks(local if world > 1 else 0)
    torch.cuda.synchronize()
    r = cluster_run(n, args.steps, args.warmup, with_fp64=(rank == 0 and not args.no_fp64), clocks=clocks,
                    dist=dist)
    ms = r["ms"]
    if dist:
        ms = max_over_ranks(ms, dist, "cuda")
        dist.barrier()
    value = replica_value(cells, world, args.steps, ms)
    peak, peak_kind = measured_peak()
    achieved = ALG_STAGE_MULTI * cells / (r["stage_avg_ms"] / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": STAGE_MULTI_TRAFFIC_B_PER_CELL * cells, "peak_kind": peak_kind,
                "kernel": "m2c::stage_kernel<float,16,HLLC,two materials>", "avg_launch_ms": r["stage_avg_ms"],
                "alg_bytes_per_launch": ALG_STAGE_MULTI * cells,
                "step_hbm_frac": r["hbm_frac_step"],
                "traffic_source": "ncu dram__bytes_read+write per cell of the two-material stage kernel "
                                  "(192^3 cluster), scaled to the launch's cells"}
    if args.bubble:
        out = {k: v for k, v in r.items() if not k.startswith("_")}
        out.update({"value": value, "roofline": roofline, "ms_per_step": ms / args.steps})
        r["_solver"].close()
        print(json.dumps(out))
        return

    e2e = None
    if not args.no_e2e:
        ne = 3
        te, nbytes = cluster_e2e(r["_solver"], r["_case"], ne, dist)
        if dist:
            te = max_over_ranks(te, dist, "cuda")
        e2e = {"value": world * cells * ne / te, "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": ne,
               "note": "m2cg_upload_state(V, ID, phi) + m2cg_run(1) + m2cg_download_state(V, ID, phi) per step, "
                       "ghosted AoS host state in pinned memory"}
    r["_solver"].close()
    del r["_solver"], r["_case"]

    extras = None
    if rank == 0 and world == 1 and not args.only_headline:
        extras = {}
        net = load_warmstart()
        for name, fn in (("periodic_box_256", lambda: extra_box(cpu=not args.no_cpu_baseline)),
                         ("single_bubble_192", lambda: extra_bubble()),
                         ("batched_tubes", lambda: extra_tubes(mlp=net)),
                         ("embedded_plane_192", lambda: extra_walls()),
                         ("learned_warm_start", lambda: extra_warm_start(net) if net is not None else
                          {"unavailable": "m2c_b200/data/warmstart_mlp.npz not present"}),
                         ("learned_warm_start_cluster", lambda: extra_cluster_warm_start(net) if net is not None else
                          {"unavailable": "m2c_b200/data/warmstart_mlp.npz not present"})):
            try:
                extras[name] = fn()
            except Exception as e:  # an extra must not cost the headline line
                extras[name] = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 flux / f64 state", "data": "synthetic (seeded bubble cluster)",
            "config": config(n, world),
            "gpu_launches": int(r["launches"]),
            "roofline": roofline,
            "clocks": r["clocks"],
            "interface_work_per_step": r["per_step"],
            "fp64": r.get("fp64"),
            "cpu_baseline": cpu,
            "e2e": e2e,
            "extras": extras,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
