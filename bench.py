#!/usr/bin/env python
"""SMAC pressure-projection throughput on B200.

Metric: 256^3 pressure solves/s to a 1e-8 FP64 true relative residual,
mixed precision (headline `value`) beside plain FP64, plus the HBM fraction
of the dominant kernel.  A step is one projection of the 256^3 single-phase
workload: divergence of a seeded U[-1,1) face field -> MG-PCG solve to
1e-8 -> velocity correction.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One process per GPU (torchrun for N>1); every rank projects its own replica
(the path does not shard: "replicas only"), value = all ranks' solves / the
slowest rank's time.  --impl reference times the reference algorithm's CPU
restatement (oracle, all host threads) on the same workload (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "256^3 pressure solves/s to 1e-8 FP64 resid (mixed; FP64 plain alongside)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--workload", choices=["plain", "vof", "ibm"], default="plain")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own GPU projection (oracle/_ref) beside the bench line")
    ap.add_argument("--cpu-budget", type=float, default=25.0, help="seconds of oracle work for cpu_baseline")
    ap.add_argument("--kernel-only", type=int, default=None,
                    help="set up the workload and launch one kernel (smac_time_kernel id) a few times: a small, "
                         "self-contained command for ncu captures")
    ap.add_argument("--around", default=None,
                    choices=["predict_vstar", "vstar_boundary", "pressure_ghost", "velocity_ghost", "face_gradp",
                             "update_properties", "predict_vstar_two_way", "mass_flux", "mass_flux_two_way",
                             "poisson_beta_two_way"],
                    help="set up the workload and launch one of the calls around the projection --reps times "
                         "(for ncu captures)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--breakdown", action="store_true",
                    help="two warm-up and three timed projections per precision (mixed, FP64) of the workload, "
                         "event-timed: a small, fixed launch list for ncu")
    ap.add_argument("--sweep-kernel", type=int, default=0,
                    help="smac_sweep_kernel of the solvers: 0 auto, 1 TMA ring, 2 z-march, 3 shared tiles")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """NVML clock / throttle-reason sampling on a thread during the timed region."""

    REASONS = {
        "hw_slowdown": 0x0000000000000008,
        "sw_power_cap": 0x0000000000000004,
        "hw_thermal_slowdown": 0x0000000000000040,
        "sw_thermal_slowdown": 0x0000000000000020,
        "hw_power_brake_slowdown": 0x0000000000000080,
    }

    def __init__(self, index):
        self.samples = []
        self.reasons = set()
        self._stop = threading.Event()
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # noqa: BLE001
            self.err = str(e)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "error": getattr(self, "err", "")}
        med = statistics.median(self.samples) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(name="k_rbgs_zm_fp32_256.md"):
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of
    the dominant kernel, from the line `traffic_bytes_per_launch: N` of the
    committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if "traffic_bytes_per_launch:" in line:
                try:
                    return float(line.split("traffic_bytes_per_launch:")[1].strip().strip("`").split()[0])
                except (ValueError, IndexError):
                    return None
    return None


def bench_config(args, world):
    """The workload both arms measure (the same dict in both lines)."""
    return {"workload": f"{args.workload} {args.n}^3 projection (divergence + MG-PCG to {args.tol:g} + correction), "
                        f"replicas per GPU", "grid": args.n, "tol": args.tol,
            "l2": "working set > L2 (coefficients alone 3x139 MB at 256^3)", "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------------------
def build_case(args, solid_fraction=None):
    from mydemcfd_b200 import workloads as W
    if args.workload == "plain":
        return W.plain_case(args.n, seed=2)
    if args.workload == "vof":
        return W.vof_case(args.n, seed=3, ratio=1000.0)
    return W.ibm_case(args.n, seed=4, nsph=200, solid_fraction=solid_fraction)


def cpu_projection(case, tol):
    """One whole projection of the reference algorithm on the host (the
    oracle's restatement: divergence, Jacobi-MG-PCG solve_pureneumann_gmgpcg
    to ||r||/||b|| < tol checked every 5 iterations, correction), all host
    threads.  Returns (seconds, PCG iterations)."""
    from oracle import oracle as O
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _cases import ref_grid
    g = ref_grid(case)
    t0 = time.perf_counter()
    pd, _, st = O.solve(g, tol=tol, stop_rule=O.STOP_REL_RECURSIVE, max_iter=2000)
    O.correct(g, pd)
    return time.perf_counter() - t0, st["iterations"]


def cpu_baseline(args, case, budget):
    """The reference algorithm on all host threads: whole projections of the
    same workload (as many as fit in `budget` seconds, at least one)."""
    from oracle import oracle as O
    cores = O.num_threads()
    secs, iters = [], 0
    t_start = time.perf_counter()
    while not secs or (time.perf_counter() - t_start) + statistics.mean(secs) <= budget:
        sec, iters = cpu_projection(case, args.tol)
        secs.append(sec)
    t = statistics.median(secs)
    return {
        "value": 1.0 / t, "unit": "solves/s", "cores": cores, "kind": "port",
        "sample": (f"{len(secs)} whole projections (divergence, Jacobi-MG-PCG to ||r||/||b|| < {args.tol:g} in "
                   f"{iters} iterations, correction) of the {case.N[0]}^3 {args.workload} workload by the oracle's "
                   f"restatement of the reference algorithm; median"),
        "seconds_per_solve": t, "iterations": iters,
    }


# Algorithmic bytes per fine cell of one PCG iteration of the reference's
# solve_pureneumann_gmgpcg (CFD/pressure_solver/G_PCGSolver.cu:845-918, V-cycle
# G_GMGSolver.cu:925-998), by the byte model of this library's kernels (every
# array a kernel must touch, once; 8-byte values): A dir with p.Ap (dir + 7
# stencil arrays read, Ap written; dir.Ap to a temporary, summed) 72 + 24 + 8;
# dp += a dir, r -= a Ap 48; mean removal of r (sum, subtract) 24; V-cycle on
# the fine grid: clear 8, 8 Jacobi sweeps x (x, rhs, 6 weights + inverse
# diagonal, x out) 80, residual 80, restriction 9, prolongation 17; r.z
# (product, sum) 32; dir = z + b dir 24.  The coarse grids add 1/7.
REF_ITER_BYTES_PER_CELL = (72 + 24 + 8 + 48 + 24 + 8 + 8 * 80 + 80 + 9 + 17 + 32 + 24) * 8.0 / 7.0


class _QuietStdout:
    """Sends the process's C-level stdout to /dev/null for the duration (the
    reference's driver prints its progress there), flushing the C buffers
    before the descriptor is restored."""

    def __enter__(self):
        import ctypes
        self._libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self._libc.fflush(None)
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        self._libc.fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def reference_gpu_baseline(case, peak):
    """The reference's own GPU projection (solve_poisson + correct_vof_velocity,
    built from its sources under oracle/_ref) on the same input, timed by CUDA
    events inside its driver; its tolerance (max|r| dt, tested every 5
    iterations) is the loosest of 1e-2 * 4^-i whose output meets the 1e-8
    relative residual, measured with this library's FP64 operator.  None when
    the reference build is absent."""
    import torch

    from mydemcfd_b200 import _native as nat
    from mydemcfd_b200 import workloads as W
    from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid
    from oracle import ref as REF
    if not REF.available():
        return None
    g = DeviceGrid.from_case(case)
    probe = B200PressureSolver(case.N, case.h, precision=nat.PRECISION_FP64, tol=1e-8)
    probe.set_coefficients(g)
    fluid = torch.from_numpy(W.interior(case.ct) == W.C_INTERIOR).cuda()

    def rel(pd, rhs):
        x = torch.from_numpy(pd).cuda()
        y = torch.zeros_like(x)
        probe.apply_A(x, y)
        b = torch.from_numpy(rhs).cuda()[1:-1, 1:-1, 1:-1][fluid]
        b = b - b.mean()
        r = b - y[1:-1, 1:-1, 1:-1][fluid]
        r = r - r.mean()
        return float(torch.linalg.norm(r) / torch.linalg.norm(b))

    tol, found = 1e-2, None
    with _QuietStdout():
        for _ in range(12):
            out = REF.solve(case, solver_type=nat.PURENEUMANN_GMG_PCG, tol=tol, levels=6, do_correct=True)
            r = rel(out["p_delta"], out["rhs"])
            if r <= 1e-8:
                found = (tol, out, r)
                break
            tol *= 0.25
        probe.close()
        if found is None:
            return None
        tol, out, r = found
        runs = [out] + [REF.solve(case, solver_type=nat.PURENEUMANN_GMG_PCG, tol=tol, levels=6, do_correct=True)
                        for _ in range(2)]
    ms = min(o["solve_ms"] + o["correct_ms"] for o in runs)
    cells = float(np.prod(case.N))
    alg = cells * (out["iterations"] * REF_ITER_BYTES_PER_CELL + 7 * 8 + 10 * 8)  # + RHS, correction
    return {"solves_per_s": 1e3 / ms, "ms_per_projection": ms, "solve_ms": min(o["solve_ms"] for o in runs),
            "iterations": out["iterations"], "tol_max_r_dt": tol, "rel_residual": r,
            "alg_bytes_per_projection": alg, "achieved_GBps": alg / (ms / 1e3) / 1e9,
            "frac_of_peak": alg / (ms / 1e3) / 1e9 / peak,
            "what": "the reference's solve_poisson + correct_vof_velocity built from its sources (oracle/_ref), "
                    "same input, its GMG-PCG with 6 levels; bytes by this library's byte model"}


def run_reference(args, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    case = build_case(args, solid_fraction=lambda N, h, o, s: O.solid_fraction_spheres(N, h, o, s))
    # every step is one whole projection of the workload on the host
    vals, iters = [], 0
    for i in range(args.warmup + args.steps):
        sec, iters = cpu_projection(case, args.tol)
        if i >= args.warmup:
            vals.append(sec)
    sec = statistics.mean(vals)
    v = 1.0 / sec
    cores = O.num_threads()
    out = {
        "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SplitMix64 U[-1,1) faces)",
        "config": bench_config(args, args.gpus),
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": (f"every step one whole projection (divergence, Jacobi-MG-PCG to ||r||/||b|| < "
                                    f"{args.tol:g} in {iters} iterations, correction) by the oracle's restatement "
                                    f"of the reference algorithm on {cores} host threads")},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
def run_ours(args, ranks):
    import torch

    from mydemcfd_b200 import _native as nat
    from mydemcfd_b200 import replicas
    from mydemcfd_b200 import workloads as W
    from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid, ibm_solid_fraction_device

    rank, world = ranks.rank, ranks.world
    torch.cuda.set_device(ranks.local_rank)
    dev = torch.device("cuda", ranks.local_rank)
    replicas.init(ranks, "nccl", device=dev)

    case = build_case(args, solid_fraction=lambda N, h, o, s: ibm_solid_fraction_device(N, h, o, s).cpu().numpy())
    g = DeviceGrid.from_case(case, device=dev)
    sh = W.shapes(case.N)
    stream = torch.cuda.current_stream()

    def solver(precision):
        s = B200PressureSolver(case.N, case.h, precision=precision, tol=args.tol, sweep_kernel=args.sweep_kernel)
        s.set_coefficients(g)
        return s

    s_mixed = solver(nat.PRECISION_MIXED)
    s_plain = solver(nat.PRECISION_FP64)
    out_v = [torch.zeros(sh[k], dtype=torch.float64, device=dev) for k in "xyz"]
    pd = torch.zeros(sh["cell"], dtype=torch.float64, device=dev)

    def step(s):
        return s.project(g.f_vx_star_, g.f_vy_star_, g.f_vz_star_, case.dt, pd, *out_v)

    def timed(fn, k):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        replicas.barrier(ranks)
        torch.cuda.synchronize()
        ev0.record(stream)
        stats = [fn() for _ in range(k)]
        ev1.record(stream)
        torch.cuda.synchronize()
        replicas.barrier(ranks)
        return replicas.max_over_ranks(ranks, ev0.elapsed_time(ev1), device=dev), stats

    for _ in range(args.warmup):
        step(s_mixed)
        step(s_plain)
    torch.cuda.synchronize()

    with ClockSampler(torch.cuda.current_device()) as clk:
        ms_mixed, st_mixed = timed(lambda: step(s_mixed), args.steps)
    ms_plain, st_plain = timed(lambda: step(s_plain), args.steps)
    sps_mixed = replicas.throughput(ranks, args.steps, ms_mixed)
    sps_plain = replicas.throughput(ranks, args.steps, ms_plain)

    # end to end through the C ABI with host buffers: pinned u* in, u and
    # p_delta out, every projection's copies inside the timed region.  The
    # projections go through the queued host-buffer entry points
    # (smac_async_*), which overlap one projection's copies with its
    # neighbours' solves; the timed region ends when the last outputs are in
    # host memory.
    e2e = None
    if not args.no_e2e:
        from mydemcfd_b200.solver import AsyncProjector
        host_in = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (case.vxs, case.vys, case.vzs)]
        host_out = [[torch.empty(sh[k], dtype=torch.float64).pin_memory() for k in ("x", "y", "z", "cell")]
                    for _ in range(2)]
        proj = AsyncProjector(s_mixed)

        def e2e_run(k):
            tickets = []
            for i in range(k):
                o = host_out[i % 2]
                tickets.append(proj.submit(*host_in, case.dt, o[3], o[0], o[1], o[2]))
            return [proj.wait(t) for t in tickets]

        e2e_run(max(2, args.warmup // 2))
        ms_e2e, st_e2e = timed(lambda: e2e_run(args.steps), 1)
        proj.close()
        e2e = {"value": replicas.throughput(ranks, args.steps, ms_e2e), "unit": "solves/s",
               "h2d_bytes_per_step": int(sum(t.numel() * 8 for t in host_in)),
               "d2h_bytes_per_step": int(sum(t.numel() * 8 for t in host_out[0])),
               "api": "smac_async_submit / smac_async_wait (host buffers, copies overlapped with neighbouring solves)"}

    # roofline of the dominant kernel: the fused red-black sweep of the fine
    # grid in FP32 (k_rbgs_zm<float>, the z-march), timed with CUDA events on
    # the solver's stream right after the timed region
    peak, peak_kind = measured_peaks()
    step(s_mixed)
    ms_k, bytes_k = s_mixed.time_kernel(3, reps=20)
    achieved = bytes_k / (ms_k / 1e3) / 1e9
    traffic = ncu_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "k_rbgs_zm<float,4,2,6,0,false>: fused red-black sweep, register z-march "
                                              "over whole rows, 256^3 grid",
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "alg_bytes_per_launch": bytes_k, "ms_per_launch": ms_k}
    kernel_table = {}
    for kid, name in ((0, "matvec_f64"), (1, "matvec_f32"), (2, "rbgs_sweep_f64"), (3, "rbgs_sweep_f32"),
                      (4, "true_residual_f64"), (5, "rbgs_halfsweeps_f64"), (6, "rbgs_halfsweeps_f32"),
                      (7, "dir_matvec_f32"), (8, "dir_matvec_f64"), (9, "update_f32"), (10, "update_f64")):
        ms, b = s_mixed.time_kernel(kid, reps=10)
        kernel_table[name] = {"ms": ms, "GB/s": b / (ms / 1e3) / 1e9}
    # the same sweeps by the TMA-ring kernel, for comparison
    s_mixed.set_options(sweep_kernel=nat.SWEEP_TMA)
    for kid, name in ((2, "rbgs_sweep_f64_tma"), (3, "rbgs_sweep_f32_tma")):
        ms, b = s_mixed.time_kernel(kid, reps=10)
        kernel_table[name] = {"ms": ms, "GB/s": b / (ms / 1e3) / 1e9}
    s_mixed.set_options(sweep_kernel=args.sweep_kernel)

    # the solve alone (RHS in place; MG-PCG and the export of p_delta), beside
    # the whole projection
    solve_only = {}
    for name, s in (("mixed", s_mixed), ("plain_fp64", s_plain)):
        s.divergence(g, case.dt)
        s.solve_rhs(pd)
        ms_s, _ = timed(lambda: s.solve_rhs(pd), args.steps)
        solve_only[name] = {"value": replicas.throughput(ranks, args.steps, ms_s), "unit": "solves/s",
                            "ms_per_solve": ms_s / args.steps}

    post_pass = post_pass_timings(case, g, pd, out_v, dev, stream)

    # error of each result against an FP64 solve to 1e-12 of the same input
    # (relative 2-norm over the fluid cells, fluid mean removed)
    fluid = torch.from_numpy(W.interior(case.ct) == W.C_INTERIOR).to(dev)

    def pressure(s):
        step(s)
        torch.cuda.synchronize()
        return pd[1:-1, 1:-1, 1:-1][fluid].clone()

    p_mixed, p_plain = pressure(s_mixed), pressure(s_plain)
    s_tight = B200PressureSolver(case.N, case.h, precision=nat.PRECISION_FP64, tol=1e-12)
    s_tight.set_coefficients(g)
    p_tight = pressure(s_tight)
    s_tight.close()

    def err(p):
        a, b = p - p.mean(), p_tight - p_tight.mean()
        return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))

    launches = int(sum(s["kernel_launches"] for s in st_mixed))
    res = {
        "metric": METRIC, "value": sps_mixed, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic (seeded SplitMix64 U[-1,1) faces)",
        "config": bench_config(args, world),
        "plain_fp64": {"value": sps_plain, "ms_per_step": ms_plain / args.steps,
                       "iterations": st_plain[-1]["iterations"], "rel_residual": st_plain[-1]["rel_residual"],
                       "error_vs_fp64_1e-12": err(p_plain)},
        "mixed": {"iterations": st_mixed[-1]["iterations"], "reliable_updates": st_mixed[-1]["reliable_updates"],
                  "rel_residual": st_mixed[-1]["rel_residual"], "levels": st_mixed[-1]["num_levels"],
                  "alg_bytes_per_solve": st_mixed[-1]["alg_bytes"],
                  "alg_GBps": st_mixed[-1]["alg_bytes"] * args.steps / (ms_mixed / 1e3) / 1e9,
                  "error_vs_fp64_1e-12": err(p_mixed)},
        "speedup_mixed_vs_plain": sps_mixed / sps_plain,
        "solve_only": solve_only,
        "post_pass": post_pass,
        "e2e": e2e,
        "gpu_launches": launches,
        "roofline": roofline,
        "kernels": kernel_table,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        res["cpu_baseline"] = cpu_baseline(args, case, args.cpu_budget)
        res["cpu_baseline"].pop("seconds_per_solve", None)
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        res["reference_gpu"] = reference_gpu_baseline(case, peak)
    if rank == 0:
        print(json.dumps(res), flush=True)
    s_mixed.close()
    s_plain.close()
    replicas.finish(ranks)


def around_calls(case, g, p, v, dev):
    """The calls either side of the projection on the bench grid, as
    closures, and the algorithmic bytes of each: before it the momentum
    predictor and update_vstar_boundary, after it update_boundary_ghost +
    make_face_gradp, the VoF property update, the mass-flux update and the
    two-way-coupled calls.  Inputs: pressure p and velocity v (device
    tensors), no-slip walls with an outlet on x+; the property update takes
    alpha = (p + 1) / 2, rho 1 / 1000, mu 1e-3 / 1e-1; the two-way calls take
    the void fractions eps = 0.7 + 0.2 alpha and f_inv_rho = f_b; the mass
    flux takes F_accum = 0.01 v."""
    import torch

    from mydemcfd_b200 import workloads as W
    from mydemcfd_b200.solver import (BoundaryConditions, face_gradp_device, predict_vstar_device,
                                      mass_flux_device, poisson_beta_two_way_device, update_pressure_ghost_device,
                                      update_properties_device, update_velocity_ghost_device,
                                      update_vstar_boundary_device)
    N, h = case.N, case.h
    sh = W.shapes(N)
    bcid = [torch.zeros(sh[k], dtype=torch.uint8, device=dev) for k in "xyz"]
    marks = [torch.from_numpy(m).to(dev) for m in W.outlet_marks(N, ("x+",))]
    bc = BoundaryConditions(np.zeros(1, np.uint8), np.zeros(1), np.zeros(1), np.zeros(1))
    gp = [torch.empty(sh[k], dtype=torch.float64, device=dev) for k in "xyz"]
    vs = (g.f_vx_star_, g.f_vy_star_, g.f_vz_star_)
    fb = (g.f_bx_, g.f_by_, g.f_bz_)
    vs_copy = [t.clone() for t in vs]
    # momentum-predictor fields: the projected velocity as both u and the
    # advecting flux, face viscosities 1e-3, rho_old 1, f_b from the grid
    mom = {"mu": torch.full(sh["cell"], 1e-3, dtype=torch.float64, device=dev),
           "rho_old": torch.ones(sh["cell"], dtype=torch.float64, device=dev), "p": p}
    for k, ax in enumerate("xyz"):
        mom["f" + ax + "t"] = (g.f_xtype_, g.f_ytype_, g.f_ztype_)[k]
        mom["f" + ax + "bcid"] = bcid[k]
        mom["v" + ax] = v[k]
        mom["mf" + ax] = v[k]
        mom["mu" + ax] = torch.full(sh["xyz"[k]], 1e-3, dtype=torch.float64, device=dev)
        mom["fb" + ax] = fb[k]
    vs_pred = [t.clone() for t in vs]
    alpha = (p + 1.0) * 0.5
    props = {k: torch.zeros(sh["cell"], dtype=torch.float64, device=dev) for k in ("rho", "inv_rho", "mu")}
    for ax in "xyz":
        for k in ("fb", "fir", "rho", "mu"):
            props[k + ax] = torch.zeros(sh[ax], dtype=torch.float64, device=dev)
    ft = (g.f_xtype_, g.f_ytype_, g.f_ztype_)
    eps = 0.7 + 0.2 * alpha
    two_way = {"eps_old": eps, "eps_new": eps, "inv_rhox": fb[0], "inv_rhoy": fb[1], "inv_rhoz": fb[2]}
    vs_pred2 = [t.clone() for t in vs]
    flux_in = {}
    for k, ax in enumerate("xyz"):
        flux_in["f" + ax + "t"] = ft[k]
        flux_in["f" + ax + "bcid"] = bcid[k]
        flux_in["v" + ax] = v[k]
        flux_in["F" + ax] = 0.01 * v[k]
    mf_out = [torch.zeros_like(t) for t in v]
    fb_out = [torch.zeros_like(t) for t in fb]
    calls = {
        "predict_vstar": lambda: predict_vstar_device(N, h, bc, mom, case.dt, (0.0, 0.0, -9.8), vs_pred),
        "vstar_boundary": lambda: update_vstar_boundary_device(N, h, bc, (g.f_xtype_, g.f_ytype_, g.f_ztype_), bcid,
                                                               marks, None, vs_copy),
        "pressure_ghost": lambda: update_pressure_ghost_device(N, h, g.celltype_, None, (0.0, 0.0, -9.8), p),
        "velocity_ghost": lambda: update_velocity_ghost_device(N, h, bc, bcid, marks, None, vs, fb, p, case.dt, v),
        "face_gradp": lambda: face_gradp_device(N, h, p, gp),
        "update_properties": lambda: update_properties_device(N, h, 1.0, 1000.0, 1e-3, 1e-1, alpha, g.celltype_, ft,
                                                              props),
        "predict_vstar_two_way": lambda: predict_vstar_device(N, h, bc, mom, case.dt, (0.0, 0.0, -9.8), vs_pred2,
                                                              two_way=two_way),
        "mass_flux": lambda: mass_flux_device(N, h, bc, flux_in, 1.0, 1000.0, case.dt, mf_out),
        "mass_flux_two_way": lambda: mass_flux_device(N, h, bc, flux_in, 1.0, 1000.0, case.dt, mf_out, eps_half=eps),
        "poisson_beta_two_way": lambda: poisson_beta_two_way_device(N, h, eps, fb, fb_out),
    }
    nx, ny, nz = N
    ncell = (nx + 2) * (ny + 2) * (nz + 2)
    nghost = ncell - nx * ny * nz
    nface = sum(int(np.prod(sh[k])) for k in "xyz")
    ring = sum(2 * (N[a] + 1) * (N[b] + N[c] + 2) for a, b, c in ((0, 1, 2), (1, 0, 2), (2, 0, 1)))
    nwall = 2 * ((ny * nz) + (nx * nz) + (nx * ny))
    alg = {
        # per cell, for the three families together: u, flux, face viscosity,
        # f_b (8 B each) and the type (1 B) of each family's face; mu, rho_old
        # and p; the three u* written
        "predict_vstar": ncell * (3 * (4 * 8 + 1) + 3 * 8 + 3 * 8),
        # face types scanned; per wall face its id read and u* written
        "vstar_boundary": nface + nwall * (1 + 8),
        # cell types scanned; per ghost cell: its source's p and type read, p written
        "pressure_ghost": ncell + nghost * (8 + 1 + 8),
        # marks scanned; per outlet face v*, f_b, p_delta read, v written; per
        # ghost face two velocities, the id and the face written
        "velocity_ghost": nface + ny * nz * 32 + ring * (8 + 8 + 1 + 8),
        # p read once, three face arrays written on the (N+1)^3 box
        "face_gradp": 8 * (ncell + 3 * (nx + 1) * (ny + 1) * (nz + 1)),
        # per cell its type and alpha read, rho, 1/rho and mu written; per face
        # its type read, 1/rho (f_b and f_inv_rho), rho and mu written
        "update_properties": ncell * (1 + 8 + 3 * 8) + nface * (1 + 4 * 8),
        # as predict_vstar plus eps_old and eps_new per cell
        "predict_vstar_two_way": ncell * (3 * (4 * 8 + 1) + 3 * 8 + 3 * 8 + 2 * 8),
        # per face its type, u and F read, mf written (the ids of the few wall faces not counted)
        "mass_flux": nface * (1 + 8 + 8 + 8),
        "mass_flux_two_way": nface * (1 + 8 + 8 + 8) + ncell * 8,
        # eps per cell; per face of the (N+1)^3 box f_inv_rho read and f_b written
        "poisson_beta_two_way": ncell * 8 + 3 * (nx + 1) * (ny + 1) * (nz + 1) * 16,
    }
    return calls, alg


def post_pass_timings(case, g, p, v, dev, stream):
    """Device time of each call of around_calls (its launches replayed from a
    CUDA graph, CUDA events, median of 10, each after an L2 flush) and the
    algorithmic bytes it moves; p, v the projected pressure and velocity."""
    import torch
    calls, alg = around_calls(case, g, p, v, dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, fn in calls.items():
        fn()
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            fn()
        ts = []
        for _ in range(10):
            flush.fill_(1)
            e0.record(stream)
            graph.replay()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = sorted(ts)[len(ts) // 2]
        out[name] = {"us": ms * 1e3, "alg_bytes": alg[name], "GB/s": alg[name] / (ms / 1e3) / 1e9}
    return out


def run_around(args):
    """Set up the bench grid and launch one call of around_calls --reps
    times: a small, self-contained command for ncu captures.  p is a seeded
    U[-1,1) field, v the seeded u*."""
    import torch

    from mydemcfd_b200 import workloads as W
    from mydemcfd_b200.solver import DeviceGrid
    case = build_case(args)
    g = DeviceGrid.from_case(case)
    sh = W.shapes(case.N)
    p = torch.from_numpy(W.uniform_pm1(77, int(np.prod(sh["cell"]))).reshape(sh["cell"])).cuda()
    v = (g.f_vx_star_, g.f_vy_star_, g.f_vz_star_)
    calls, alg = around_calls(case, g, p, [t.clone() for t in v], torch.device("cuda"))
    for _ in range(args.reps):
        calls[args.around]()
    torch.cuda.synchronize()
    print(json.dumps({"call": args.around, "n": args.n, "reps": args.reps, "alg_bytes": alg[args.around]}))


def run_kernel_only(args):
    import torch

    from mydemcfd_b200 import _native as nat
    from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid
    case = build_case(args)
    g = DeviceGrid.from_case(case)
    s = B200PressureSolver(case.N, case.h, precision=nat.PRECISION_MIXED, tol=args.tol,
                           sweep_kernel=args.sweep_kernel)
    s.set_coefficients(g)
    s.divergence(g, case.dt)
    ms, b = s.time_kernel(args.kernel_only, reps=args.reps)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_id": args.kernel_only, "n": args.n, "ms_per_launch": ms, "alg_bytes": b,
                      "GB/s": b / (ms / 1e3) / 1e9}))
    s.close()


def run_breakdown(args):
    import torch

    from mydemcfd_b200 import _native as nat
    from mydemcfd_b200 import workloads as W
    from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid, ibm_solid_fraction_device
    case = build_case(args, solid_fraction=lambda N, h, o, s: ibm_solid_fraction_device(N, h, o, s).cpu().numpy())
    g = DeviceGrid.from_case(case)
    sh = W.shapes(case.N)
    ov = [torch.zeros(sh[k], dtype=torch.float64, device="cuda") for k in "xyz"]
    pd = torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")
    for prec in (nat.PRECISION_MIXED, nat.PRECISION_FP64):
        s = B200PressureSolver(case.N, case.h, precision=prec, tol=args.tol, sweep_kernel=args.sweep_kernel)
        s.set_coefficients(g)
        for _ in range(2):
            s.project(g.f_vx_star_, g.f_vy_star_, g.f_vz_star_, case.dt, pd, *ov)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            st = s.project(g.f_vx_star_, g.f_vy_star_, g.f_vz_star_, case.dt, pd, *ov)
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"precision": "mixed" if prec == nat.PRECISION_MIXED else "fp64",
                          "ms_per_projection": e0.elapsed_time(e1) / 3, "launches": st["kernel_launches"],
                          "iterations": st["iterations"]}), flush=True)
        s.close()


def main():
    args = parse()
    if args.breakdown:
        run_breakdown(args)
        return
    if args.kernel_only is not None:
        run_kernel_only(args)
        return
    if args.around is not None:
        run_around(args)
        return
    from mydemcfd_b200 import replicas
    ranks = replicas.from_env()
    if args.impl == "reference":
        run_reference(args, ranks.rank)
        return
    run_ours(args, ranks)


if __name__ == "__main__":
    main()
