"""Benchmark: cell-updates/s per RK step of the explicit finite-volume step.

Workload (one GPU holds it): the 3D single-material periodic box, 256^3
cells, ideal gas gamma 1.4, rho = 1 and p = 1/1.4 perturbed by 16 seeded
Fourier modes (|k| in 1..8, 1%), solenoidal velocity with RMS Mach 0.3,
generalized Roe flux with generalized minmod MUSCL (alpha 1), RK3, CFL 0.4.
The headline runs the mixed path (FP32 reconstruction/flux, FP64 state);
the FP64 path is timed on the same state and the L1 difference between the
two is reported.

A "step" is one full RK3 step (3 fused stage launches + the device clock).
Inputs are larger than L2 (5 x 128 MiB per state array), so no explicit
flush is needed between steps.

Multi-GPU: the north-star path does not shard; --gpus N runs N independent
replicas (one per GPU, "scaling": "weak"), value = all cells updated / max
time over ranks.

--impl reference: the reference's own CPU implementation (the unmodified
sources built with single-rank shims under oracle/_ref), run on the host
cores as independent processes, each advancing a bounded 48^3 sample of the
same physics (symmetry walls instead of periodic: the reference has no
periodic boundary) by one RK3 step per benchmark step.

Extras (rank 0 at N = 1, skipped by --only-headline), under "extras": the
384^3 sixteen-bubble cluster (mixed vs FP64, error of mixed against FP64,
material-ID and level-set sign mismatches), the 4096 batched two-material
tubes (CUDA-graph replay, autotuned tiles, with and without the learned
warm start), and the learned warm start's evaluations and iterations saved
on held-out interface problems (network in m2c_b200/data/warmstart_mlp.npz).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per RK step (RK3, 256^3 periodic box, mixed FP32/FP64)"
UNIT = "cell-updates/s"
CPU_SAMPLE_N = 48


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--only-headline", action="store_true",
                   help="skip the extra workloads (bubble cluster, batched tubes, learned warm start)")
    p.add_argument("--bubble", type=int, default=0, metavar="N",
                   help="run only the bubble-cluster workload at N^3 (for profiling) and print its JSON")
    return p.parse_args()


# --------------------------------------------------------------------------
# CPU reference leg (also the cpu_baseline): independent processes
# --------------------------------------------------------------------------
def _cpu_worker(args):
    n, steps, seed = args
    # the reference prints mesh statistics on stdout: keep the JSON line alone there
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, ROOT)
    from m2c_b200 import abi, cases
    from oracle import ref
    g, s, mats, V = cases.fourier_box(CPU_SAMPLE_N if n is None else n, seed=seed, bc=abi.BC_SYMMETRY)
    c = ref.RefCase(g, s, mats)
    c.set_state(V)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        c.run(1)
        times.append(time.perf_counter() - t0)
    return times


def _cpu_bubble_worker(args):
    n, nbubbles, steps, seed = args
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, ROOT)
    from m2c_b200 import cases
    from oracle import ref
    g, s, mats, ls, V, ID, PHI = cases.bubble_case(n, nbubbles=nbubbles, seed=seed)
    c = ref.RefCase(g, s, mats, ls)
    c.set_state(V, ID, PHI)
    t0 = time.perf_counter()
    c.run(steps)
    return time.perf_counter() - t0


def cpu_reference_bubble(n=48, nbubbles=16, steps=12, cores=None):
    """The reference on the bubble-cluster physics at n^3 (the 384^3 case does
    not fit its memory model on the host): `cores` independent processes,
    `steps` steps each (reinitialisation every 10 steps); cell-updates/s of
    all processes together."""
    import multiprocessing as mp
    cores = cores or min(os.cpu_count() or 1, 64)
    with mp.get_context("spawn").Pool(cores) as pool:
        times = pool.map(_cpu_bubble_worker, [(n, nbubbles, steps, 5 + r) for r in range(cores)])
    return {"value": cores * n ** 3 * steps / max(times), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{cores} processes x one {n}^3 cluster of {nbubbles} bubbles (same physics), {steps} RK3 "
                      f"steps each (reinitialisation every 10 steps)"}


def cpu_reference(steps, warmup, cores=None):
    """Run the reference on `cores` processes; returns per-step wall times
    (max over processes) and the cell count per step (all processes)."""
    import multiprocessing as mp
    cores = cores or min(os.cpu_count() or 1, 64)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(CPU_SAMPLE_N, warmup + steps, 100 + r) for r in range(cores)])
    per_step = [max(r[w + warmup] for r in res) for w in range(steps)]
    cells = cores * CPU_SAMPLE_N ** 3
    return per_step, cells, cores


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


def profiled_traffic():
    """DRAM bytes (read + write) per cell per stage launch of the mixed stage
    kernel, from the committed ncu summary (one stage-2 launch at 160^3), or
    None."""
    import re
    p = os.path.join(ROOT, "profiles", "stage_kernel_mixed_160cube.md")
    if os.path.exists(p):
        m = re.search(r"traffic_bytes_per_cell_per_launch:\s*([0-9.]+)", open(p).read())
        if m:
            return {"bytes_per_cell_per_launch": float(m.group(1))}
    return None


# --------------------------------------------------------------------------
# extra workloads (rank 0, one GPU): the other configurations of the path
# --------------------------------------------------------------------------
def extra_bubble(n=384, nbubbles=16, steps=10, warmup=2):
    """Two-material bubble cluster in water, mixed vs FP64: cell-updates/s,
    HBM fraction of the algorithmic bytes (RK3: 8 FP64 5-vectors, 8 phi
    values and 3 ID bytes per cell and step), and the mixed path's error
    against the FP64 path after the same steps."""
    import numpy as np
    from m2c_b200 import abi, cases, gpu
    res = {}
    for prec in (abi.PREC_MIXED, abi.PREC_FP64):
        g, s, mats, ls, V, ID, PHI = cases.bubble_case(n, nbubbles=nbubbles, precision=prec)
        sol = gpu.Solver(g, s, mats, ls)
        sol.upload(V, ID, PHI)
        del V, ID, PHI
        sol.time_steps(warmup)
        ms, _ = sol.time_steps(steps)
        Vd, IDd, Pd = sol.download()
        res[prec] = (ms, Vd[1:-1, 1:-1, 1:-1].reshape(-1, 5), IDd[1:-1, 1:-1, 1:-1].ravel(),
                     Pd[1:-1, 1:-1, 1:-1].ravel(), sol.counters())
        sol.close()
        del Vd, IDd, Pd
    cells = n ** 3
    (mm, Vm, Im, Pm, cm), (mf, Vf, If, Pf, cf) = res[abi.PREC_MIXED], res[abi.PREC_FP64]
    l1 = lambda a, b: float(np.abs(a - b).sum() / np.abs(b).sum())
    vel = float(np.linalg.norm(Vm[:, 1:4] - Vf[:, 1:4], axis=1).sum() / np.linalg.norm(Vf[:, 1:4], axis=1).sum())
    alg = 387.0 * cells * steps
    peak, kind = measured_peak()
    kind = "single bubble" if nbubbles == 1 else "bubble cluster"
    out = {"workload": f"{kind} {n}^3, {nbubbles} air bubble(s) in water, HLLC + van Albada, exact interface "
                       f"Riemann, FD3 level set with reinitialisation every 10 steps, RK3, CFL 0.4",
           "steps": steps, "after_warmup_steps": warmup,
           "mixed": {"cell_updates_per_s": cells * steps / (mm / 1e3), "ms_per_step": mm / steps,
                     "hbm_frac": alg / (mm / 1e3) / 1e9 / peak},
           "fp64": {"cell_updates_per_s": cells * steps / (mf / 1e3), "ms_per_step": mf / steps,
                    "hbm_frac": alg / (mf / 1e3) / 1e9 / peak},
           "mixed_speedup": mf / mm,
           "mixed_vs_fp64_rel_L1": {"rho": l1(Vm[:, 0], Vf[:, 0]), "velocity": vel, "p": l1(Vm[:, 4], Vf[:, 4])},
           "material_id_mismatch": int((Im != If).sum()), "phi_sign_mismatch": int(((Pm < 0) != (Pf < 0)).sum()),
           "riemann_calls_per_step_mixed": cm["riemann_calls"] / (steps + warmup),
           "peak_kind": kind}
    return out


def extra_tubes(ntubes=4096, steps=200, mlp=None):
    """Batched 1D two-material tubes (one graph-replayed step sequence, autotuned
    tiles); tubes whose initial interface problem fails or that fail during a
    screening run are redrawn (counted)."""
    import numpy as np
    from m2c_b200 import cases, gpu
    s = cases.tube_scheme()
    lens, mats, VL, VR, redrawn = cases.tubes(ntubes, seed=11, reject=gpu.tube_rejects(s))
    rng = np.random.default_rng(99)
    failed_total = 0
    for _ in range(4):
        b = gpu.Batch(s, lens, mats, VL, VR)
        b.time_steps(steps, check_errors=False)
        bad = np.nonzero(b.tube_errors())[0]
        b.close()
        if len(bad) == 0:
            break
        failed_total += len(bad)
        for t in bad:
            while True:
                mats[2 * t], mats[2 * t + 1] = cases.stiffened_gas_pair(rng), cases.stiffened_gas_pair(rng)
                a, c = cases.tube_states(1, rng)
                VL[t], VR[t] = a[0], c[0]
                if not gpu.tube_rejects(s)([mats[2 * t], mats[2 * t + 1]], VL[t:t + 1], VR[t:t + 1])[0]:
                    break
    out = {"workload": f"{ntubes} two-material shock tubes, 100-2000 cells, HLLC + van Albada, exact interface "
                       f"Riemann, RK2, CFL 0.5, {steps} steps", "cells": int(lens.sum()),
           "redrawn_at_t0": int(redrawn), "redrawn_after_failing_run": int(failed_total)}
    for label, net in (("cold", None), ("warm_start", mlp)):
        if label == "warm_start" and net is None:
            continue
        b = gpu.Batch(s, lens, mats, VL, VR)
        if net is not None:
            b.set_mlp(net)
        ms = b.time_steps(steps, check_errors=False)
        c = b.counters()
        out[label] = {"cell_updates_per_s": b.ncell * steps / (ms / 1e3), "ms_per_step": ms / steps,
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
    ok = both & (cold["Vsm"][:, 4] > 0) & np.isfinite(warm)
    rel = np.abs(np.log(warm[ok] / cold["Vsm"][ok, 4]))
    g = mats["gamma"]
    pc = mats["p_c"]
    cl = np.sqrt(g[0::2] * (VL[:, 4] + pc[0::2]) / VL[:, 0])
    cr = np.sqrt(g[1::2] * (VR[:, 4] + pc[1::2]) / VR[:, 0])
    du = (np.abs(hot["Vsm"][:, 1] - cold["Vsm"][:, 1]) / np.maximum(cl, cr))[both]
    return {"problems": n, "solved_both": int(both.sum()),
            "evaluations_cold": float(cold["evals"][both].mean()), "evaluations_warm": float(hot["evals"][both].mean()),
            "evaluation_ratio": float(cold["evals"][both].mean() / hot["evals"][both].mean()),
            "iterations_cold": float(cold["iters"][both].mean()), "iterations_warm": float(hot["iters"][both].mean()),
            "iteration_ratio": float(cold["iters"][both].mean() / hot["iters"][both].mean()),
            "prediction_abs_log_error_median": float(np.median(rel)),
            "star_velocity_diff_over_c_p99": float(np.percentile(du, 99)),
            "inference_s_host_call": t_inf}


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


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    n = args.n
    cells = n ** 3

    if args.bubble:
        print(json.dumps(extra_bubble(n=args.bubble, steps=args.steps, warmup=args.warmup)))
        return

    if args.impl == "reference":
        if rank != 0:
            return
        per_step, ccells, cores = cpu_reference(args.steps, args.warmup)
        tot = sum(per_step)
        v = ccells * len(per_step) / tot
        sample = f"{cores} processes x one {CPU_SAMPLE_N}^3 box (symmetry walls), 1 RK3 step each per benchmark step"
        print(json.dumps({
            "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * tot / len(per_step), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Fourier modes)",
            "config": {"workload": f"periodic box {n}^3 RK3 Roe/minmod, sampled on CPU as {CPU_SAMPLE_N}^3 boxes",
                       "flush": "inputs larger than L2"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    # CPU baseline first (spawned processes, before any GPU work), rank 0, N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            per_step, ccells, cores = cpu_reference(12, 1)
            cpu = {"value": ccells * len(per_step) / sum(per_step), "unit": UNIT, "cores": cores,
                   "kind": "reference",
                   "sample": f"{cores} processes x one {CPU_SAMPLE_N}^3 box, 12 RK3 steps each (after 1 warm-up)"}
        except Exception as e:  # the oracle build is missing on this host
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    import numpy as np
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    from m2c_b200 import abi, cases, gpu
    gpu.set_device(local if world > 1 else 0)

    g, s, mats, V = cases.fourier_box(n, precision=abi.PREC_MIXED, seed=2024 + rank)
    sol = gpu.Solver(g, s, mats)
    sol.upload(V)
    sol.time_steps(args.warmup)

    clocks = Clocks(local if world > 1 else 0)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms, launches = sol.time_steps(args.steps)
    clk = clocks.stop()
    torch.cuda.synchronize()
    if dist:
        ms = max_over_ranks(ms, dist, "cuda")
        dist.barrier()
    value = replica_value(cells, world, args.steps, ms)

    # roofline of the dominant kernel (the fused stage): algorithmic bytes
    # 320 B/cell per RK3 step (8 FP64 5-vectors) over the 3 stage launches
    prof_steps = 3
    stage_ms, nlaunch, _ = sol.profile_stages(prof_steps)
    avg_launch_ms = stage_ms / nlaunch
    alg_bytes_per_launch = 320.0 * cells / 3.0
    achieved = alg_bytes_per_launch / (avg_launch_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peak()
    tr = profiled_traffic()
    traffic = tr["bytes_per_cell_per_launch"] * cells if tr else None

    # FP64 path on the same state, and the L1 difference to it
    fp64 = None
    if rank == 0:
        s64 = abi.scheme(**{f: getattr(s, f) for f, _ in abi.Scheme._fields_})
        s64.precision = abi.PREC_FP64
        sol64 = gpu.Solver(g, s64, mats)
        sol64.upload(V)
        sol64.time_steps(args.warmup)
        ms64, _ = sol64.time_steps(args.steps)
        # L1 after the same number of steps from the same initial state
        a = gpu.Solver(g, s, mats)
        a.upload(V)
        b = gpu.Solver(g, s64, mats)
        b.upload(V)
        a.run(args.steps)
        b.run(args.steps)
        Va, _, _ = a.download()
        Vb, _, _ = b.download()
        ia, ib = Va[1:-1, 1:-1, 1:-1].reshape(-1, 5), Vb[1:-1, 1:-1, 1:-1].reshape(-1, 5)
        l1 = (np.abs(ia - ib).sum(0) / np.abs(ib).sum(0)).tolist()
        linf = (np.abs(ia - ib).max(0) / np.abs(ib).max(0)).tolist()
        fp64 = {"value": cells * args.steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps,
                "mixed_speedup": ms64 / ms, "mixed_vs_fp64_rel_L1": dict(zip(["rho", "u", "v", "w", "p"], l1)),
                "mixed_vs_fp64_rel_Linf": dict(zip(["rho", "u", "v", "w", "p"], linf)),
                "after_steps": args.steps}
        del a, b, sol64

    # end to end through the public API: host state in pinned memory,
    # upload + one step + download per step
    e2e = None
    if not args.no_e2e:
        Vh = torch.empty(V.shape, dtype=torch.float64, pin_memory=True).numpy()
        Vh[...] = V
        Vo = torch.empty(V.shape, dtype=torch.float64, pin_memory=True).numpy()
        ne = max(3, min(args.steps, 10))
        sol.upload(Vh)
        sol.run(1)
        sol.download(out_V=Vo, with_id=False)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ne):
            sol.upload(Vh)
            sol.run(1)
            sol.download(out_V=Vo, with_id=False)
        te = time.perf_counter() - t0
        if dist:
            te = max_over_ranks(te, dist, "cuda")
        e2e = {"value": world * cells * ne / te, "unit": UNIT, "h2d_bytes_per_step": int(Vh.nbytes),
               "d2h_bytes_per_step": int(Vo.nbytes), "steps": ne,
               "note": "m2cg_upload_state + m2cg_run(1) + m2cg_download_state per step, ghosted AoS host state"}

    extras = None
    if rank == 0 and world == 1 and not args.only_headline:
        extras = {}
        net = load_warmstart()
        for name, fn in (("bubble_cluster", lambda: extra_bubble()),
                         ("bubble_cluster_cpu_reference", lambda: cpu_reference_bubble()
                          if not args.no_cpu_baseline else {"skipped": "--no-cpu-baseline"}),
                         ("single_bubble_192", lambda: extra_bubble(n=192, nbubbles=1, steps=500, warmup=3)),
                         ("batched_tubes", lambda: extra_tubes(mlp=net)),
                         ("learned_warm_start", lambda: extra_warm_start(net) if net is not None else
                          {"unavailable": "m2c_b200/data/warmstart_mlp.npz not present"})):
            try:
                extras[name] = fn()
            except Exception as e:  # an extra must not cost the headline line
                extras[name] = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 flux / f64 state", "data": "synthetic (seeded Fourier modes)",
            "config": {"workload": f"periodic box {n}^3, ideal gas, Roe + generalized minmod, RK3, CFL 0.4, mixed",
                       "cells": cells, "flush": "inputs larger than L2 (no explicit flush)",
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "m2c::stage_kernel<float,16>", "avg_launch_ms": avg_launch_ms,
                         "alg_bytes_per_launch": alg_bytes_per_launch,
                         "traffic_source": "ncu dram__bytes_read+write of one stage-2 launch at 160^3, "
                                           "scaled per cell (profiles/stage_kernel_mixed_160cube.md)"},
            "clocks": clk,
            "fp64": fp64,
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
