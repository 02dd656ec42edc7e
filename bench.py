"""Benchmark: ms to the SOR stopping rule per domain, on one B200 per rank.

One step = one full lambda solve of a synthetic city (400 x 400 x 100 cells,
dx = dy = 2 m, z stretched 1 m x 1.03^k, 60 cuboid buildings, power-law
inflow): R, red-black SOR from lambda = 0 until max|dlambda| (FP64) <= 1e-3
or 10 000 iterations, then the velocity correction. The reference's own
tolerance (1e-9) is never reached in FP32, so the benchmark uses 1e-3, the
same rule for every arm.

  value          device time per solve with inputs resident in HBM (CUDA events
                 on the solver's stream, max over ranks) divided by the domains
                 all ranks solved in it; lower is better.
  e2e            the same through the host API: pinned host inputs copied in
                 (qesb_set_inputs) and u, v, w copied out (qesb_solve) every step.
  roofline       the fused SOR kernel alone: algorithmic bytes (36 B per updated
                 cell per iteration) over its measured launch time.
  cpu_baseline   the reference's Solver_CPU_RB (oracle/_ref) on this host's cores,
                 a bounded sample of iterations scaled by the iterations the
                 reference needs to reach the same rule (tests/golden/ref_iters.json).

--impl reference runs only the reference CPU solver (rank 0), same metric.
Multi-GPU (torchrun): each rank solves its own city (seed = rank); no data
crosses ranks ("scaling": "weak").
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "qes-public_b200"))
sys.path.insert(0, ROOT)

TOL = 1e-3
ITERMAX = 10000
WORKLOAD = "city400"
METRIC = "ms to SOR tolerance per domain (plain SOR from lambda=0, tol 1e-3 on FP64 max|dlambda|)"
BYTES_PER_CELL_ITER = 36  # 6 coefficients + R read (28 B), lambda read + write (8 B)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=-1, help="sweep variant for --sweeps-only (-1: autotune)")
    ap.add_argument("--profile-solve", type=int, default=0,
                    help="profiling driver: one solve of this many iterations (tol 0) with --variant, exit")
    ap.add_argument("--sweeps-only", type=int, default=0,
                    help="profiling driver: set up the workload, run this many fused-sweep launches, exit")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_city(workload, seed):
    import qesb

    if workload == "cuboid100":
        return qesb.cuboid100()
    w, _ = qesb.random_city(workload, seed)
    return w


def pinned_copy(torch, a):
    t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1]).dtype, pin_memory=True)
    arr = t.numpy()
    arr[...] = a
    return t, arr


def ref_iterations(workload, solver="Solver_CPU_RB"):
    path = os.path.join(ROOT, "tests", "golden", "ref_iters.json")
    try:
        return json.load(open(path))[workload][solver]["iterations"]
    except (OSError, KeyError):
        return None


def reference_cpu_measure(workload, seconds, threads):
    """Reference Solver_CPU_RB (oracle/_ref), `threads` OpenMP threads, timed on a
    bounded sample of iterations, scaled to the reference's iterations to the
    stopping rule. tol < 0 makes the loop run exactly `sample` iterations, so the
    reference's racy max_error reset (Solver_CPU_RB.cpp:166) cannot end it early."""
    from oracle import oracle as O

    O.ref_set_threads(threads)
    w = make_city(workload, 0)
    d = w.domain
    # calibrate on a few iterations, then time a sample sized to `seconds`
    _, _, _, _, t_cal = _quiet(lambda: O.ref_solve(d, w, -1.0, 3, kind=1, want_lambda=False))
    per_it = max(t_cal / 3, 1e-6)
    sample = int(max(5, min(ITERMAX, seconds / per_it)))
    _, _, _, _, t = _quiet(lambda: O.ref_solve(d, w, -1.0, sample, kind=1, want_lambda=False))
    ms_it = 1e3 * t / sample
    iters = ref_iterations(workload)
    return ms_it, sample, iters


def _quiet(fn):
    """Runs fn with the process's stdout sent to /dev/null (the reference prints)."""
    fd = sys.stdout.fileno()
    sys.stdout.flush()
    saved = os.dup(fd)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, fd)
    try:
        return fn()
    finally:
        sys.stdout.flush()
        os.dup2(saved, fd)
        os.close(saved)
        os.close(null)


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    ms_it, sample, iters = reference_cpu_measure(args.workload, args.cpu_seconds, threads)
    steps = []
    for _ in range(args.steps):
        ms_it_s, _, _ = reference_cpu_measure(args.workload, max(2.0, args.cpu_seconds / max(args.steps, 1)), threads)
        steps.append(ms_it_s)
    ms_it = statistics.median(steps) if steps else ms_it
    value = ms_it * iters if iters else None
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload} seed 0", "solver": "Solver_CPU_RB (reference, OpenMP)",
                   "tol": TOL, "itermax": ITERMAX},
        "cpu_baseline": {"value": value, "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": f"{sample} red-black iterations per step timed, x {iters} iterations "
                                   f"the reference needs to reach tol {TOL}"},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ms_per_iteration": ms_it,
    }
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch

    import qesb

    rank, local, world = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    w = make_city(args.workload, rank)
    d = w.domain
    Nx, Ny, Nz = d.base
    updated = (Nx - 2) * (Ny - 2) * (Nz - 1)

    solver = qesb.Solver_B200(d, TOL, device=dev)
    solver.set_stream(stream.cuda_stream)
    solver.set_inputs(w)
    # autotuner: picks the sweep variant for this grid shape (untimed set-up,
    # cached for the process like a library's algorithm search)
    variant, variant_us = solver.autotune()

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident solves -------------------------------------------------
    du = torch.empty(d.numFaceCentered(), dtype=torch.float32, device=f"cuda:{dev}")
    dv, dw = torch.empty_like(du), torch.empty_like(du)

    def step():
        solver.resetLambda()
        return solver.solve_device(ITERMAX, du.data_ptr(), dv.data_ptr(), dw.data_ptr())

    for _ in range(args.warmup):
        st = step()
    barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            stats.append(step())
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = max_over_ranks(ms)
    iters = stats[-1]["iterations"]
    launches = sum(s["launches"] for s in stats)

    # ---- end to end through the host API ----------------------------------------
    host_in = [pinned_copy(torch, a) for a in w.inputs()]
    ins = [arr for _, arr in host_in]
    hu = [pinned_copy(torch, np.zeros(d.numFaceCentered(), np.float32)) for _ in range(3)]
    wg = qesb.WINDSGeneralData(d)
    wg.e, wg.f, wg.g, wg.h, wg.m, wg.n, wg.icellflag, wg.u0, wg.v0, wg.w0 = ins
    wg.u, wg.v, wg.w = (arr for _, arr in hu)
    h2d = sum(a.nbytes for a in ins)
    d2h = 3 * 4 * d.numFaceCentered()

    def e2e_step():
        solver.resetLambda()
        return solver.solve(wg, ITERMAX, set_inputs=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    wall_e2e = (time.perf_counter() - t0) * 1e3 / args.steps
    ms_e2e = max_over_ranks(max(e0.elapsed_time(e1) / args.steps, wall_e2e))
    e2e_ok = bool(np.array_equal(wg.u, du.cpu().numpy()))

    # ---- the fused SOR kernel alone (roofline) ----------------------------------
    solver.resetLambda()
    n_l = 40
    solver.time_sweeps(5)
    ms_sw, k = solver.time_sweeps(n_l)
    per_launch = ms_sw / n_l
    alg_bytes = BYTES_PER_CELL_ITER * updated * k
    achieved = alg_bytes / (per_launch * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    traffic = None
    prof = os.path.join(ROOT, "profiles", "sor_split_city400.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except ValueError:
            traffic = None

    # ---- CPU baseline (rank 0, N = 1) -------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            ms_it, sample, riters = reference_cpu_measure(args.workload, args.cpu_seconds, threads)
            cpu = {"value": ms_it * riters if riters else None, "unit": "ms", "cores": threads,
                   "kind": "reference",
                   "sample": f"Solver_CPU_RB {sample} iterations timed ({ms_it:.2f} ms/iteration) x "
                             f"{riters} iterations to tol {TOL}"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "ms", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {ex}"}

    solver.close()
    if rank == 0:
        value = ms_max / 1.0 / world  # domains solved per step across the job: world
        line = {
            "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.workload} ({Nx}x{Ny}x{Nz}, seed = rank)",
                       "tol": TOL, "itermax": ITERMAX, "iterations": iters,
                       "converged": bool(stats[-1]["converged"]), "path": stats[-1]["path"],
                       "sweeps_per_launch": stats[-1]["sweeps_per_launch"],
                       "variant": variant, "variant_us_per_iteration": [round(x, 2) for x in variant_us],
                       "l2": "working set > L2 (126 MB): lambda, R, mask ~ 1 GB", "parallelism": f"replicas x{world}"},
            "e2e": {"value": ms_e2e / world, "unit": "ms", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "matches_device_result": e2e_ok},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "kernel": ("k_sor_split red+black pair" if variant >= 5 else f"k_sor_tiled (K={k})"),
                         "ms_per_launch": per_launch,
                         "algorithmic_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_sweeps_only(args):
    import qesb

    w = make_city(args.workload, 0)
    with qesb.Solver_B200(w.domain, TOL) as s:
        s.set_inputs(w)
        if args.variant >= 0:
            s.set_option("variant", args.variant)
        else:
            s.autotune()
        ms, k = s.time_sweeps(args.sweeps_only)
    print(json.dumps({"sweeps_only": args.sweeps_only, "k": k, "ms_per_launch": ms / args.sweeps_only}))


def run_profile_solve(args):
    """One solve (R, iterations, correction) for launch-list captures."""
    import qesb

    w = make_city(args.workload, 0)
    with qesb.Solver_B200(w.domain, 0.0) as s:
        if args.variant >= 0:
            s.set_option("variant", args.variant)
        st = s.solve(w, args.profile_solve)
    print(json.dumps({"profile_solve": args.profile_solve, **st}))


def main():
    args = parse()
    if args.profile_solve:
        run_profile_solve(args)
    elif args.sweeps_only:
        run_sweeps_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
