"""Benchmark: ms to the SOR stopping rule per domain, learned warm start vs
plain SOR, on one B200 per rank.

Workload: held-out synthetic cities of 256 x 256 x 64 cells (dx = dy = 2 m,
z stretched 1 m x 1.03^k, 40-80 seed-placed cuboid buildings, power-law
inflow from a random direction), seeds 500000 + i, disjoint from the
warm-start network's training seeds. One step = one batch of B domains
(default 8) taken from their inputs in HBM to corrected winds in HBM:

  prephase (the headline `value`): per domain, the divergence R, an
      over-relaxed red-black SOR pre-phase from lambda = 0 (omega PRE_OMEGA, to
      max|dlambda| <= PRE_TOL in FP64) as the warm start, then the reference
      loop (omega 1.78, max|dlambda| <= 1e-3 in FP64, at most 10 000
      iterations) and the velocity correction; all B domains iterate together
      in qesb_solve_batch (persistent red/black launches in CUDA-graph chunks,
      each domain stopping on its own rule). ms per domain = step time / B.
  arms: the same batch as plain SOR from lambda = 0, the learned network's
      prediction as the start (BF16 tcgen05 convolutions, FP32 accumulation),
      network + pre-phase, and pre-phase alone, each with its iterations and
      its winds' max error against a converged field (first two domains).
  plain_single: the plain arm with the domains solved one after another.

The reference's own tolerance (1e-9) is never reached in FP32, so every arm
stops at 1e-3, the same rule.

  e2e            the warm step through the host API: pinned host inputs copied
                 in (qesb_set_inputs) and u, v, w copied out each step.
  roofline       the SOR sweep kernel of the plain single solves: algorithmic
                 bytes (36 B per updated cell per iteration) over its measured
                 device time per iteration (CUDA events, inside the graphs).
  network        tensor-core rate of one warm-start forward pass.
  reference_gpu  the reference's own GPU solver (Solver_GPU_GlobalMemory, built
                 from its sources into oracle/_ref) on the first domain, from
                 lambda = 0, same tolerance: wall ms, the solve() call.
  cpu_baseline   the reference's Solver_CPU_RB (oracle/_ref) on this host's
                 cores: a bounded sample of iterations, scaled by the iterations
                 the reference needs to reach the rule (tests/golden/ref_iters.json).

--impl reference runs only the reference CPU solver (rank 0), same metric.
Multi-GPU (torchrun): each rank solves its own batch (seeds offset by rank);
no data crosses ranks ("scaling": "weak").
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
WORKLOAD = "city256"
SEED0 = 500000
METRIC = "ms to SOR tolerance per domain: learned warm start vs plain SOR, 1 B200"
BYTES_PER_CELL_ITER = 36  # 6 coefficients + R read (28 B), lambda read + write (8 B)
# Bytes the packed red/black sweep must move per updated cell and iteration:
# its colour's lambda read + write (8), the other colour's lambda read (4),
# R (4) and the wall mask (1).
MOVED_BYTES_PER_CELL_ITER = 17
SIZE_ITERS = 300  # iterations per timed solve of the size sweep
# Over-relaxed pre-phase of the warm start on this grid: omega and its stopping
# tolerance, picked by a sweep of omega in {1.90 .. 1.98} x tol in {1e-3, 3e-3}
# on 256x256x64 cities (every seed tried preferred 1.97 / 3e-3; 1.98 stalled
# on some).
PRE_OMEGA = 1.97
PRE_TOL = 3e-3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--batch", type=int, default=8, help="domains per step")
    ap.add_argument("--weights", default=None, help="warm-start network (default: the committed weights)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 same-SOR error and divergence checks")
    ap.add_argument("--no-sizes", action="store_true", help="skip the 400^2 and 800^2 sweep-speed section")
    ap.add_argument("--no-fire-loop", action="store_true", help="skip the fire-step section")
    ap.add_argument("--variant", type=int, default=-1, help="sweep variant for the profiling drivers (-1: autotune)")
    ap.add_argument("--profile-solve", type=int, default=0,
                    help="profiling driver: one solve of this many iterations (tol 0) with --variant, exit")
    ap.add_argument("--sweeps-only", type=int, default=0,
                    help="profiling driver: set up the workload, run this many sweep launches, exit")
    ap.add_argument("--ensemble", action="store_true",
                    help="batched ensemble: 64 cities of uneven size x 36 wind directions (solves/s, p50/p99)")
    ap.add_argument("--ensemble-domains", type=int, default=64)
    ap.add_argument("--fire-loop", type=int, default=0,
                    help="QES-Fire solve pattern: this many fire steps warm-started from the previous lambda, exit")
    ap.add_argument("--profile-batch", action="store_true",
                    help="profiling driver: the headline batch (pre-phase pipeline) once untimed, once more, exit")
    ap.add_argument("--forward-only", type=int, default=0,
                    help="profiling driver: run this many warm-start forward passes on one domain, exit")
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


def ref_iterations(key, solver="Solver_CPU_RB"):
    path = os.path.join(ROOT, "tests", "golden", "ref_iters.json")
    try:
        return json.load(open(path))[key][solver]["iterations"]
    except (OSError, KeyError):
        return None


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


def reference_cpu_measure(workload, seed, seconds, threads):
    """Reference Solver_CPU_RB (oracle/_ref), `threads` OpenMP threads, timed on a
    bounded sample of iterations, scaled to the reference's iterations to the
    stopping rule. tol < 0 makes the loop run exactly `sample` iterations, so the
    reference's racy max_error reset (Solver_CPU_RB.cpp:166) cannot end it early."""
    from oracle import oracle as O

    O.ref_set_threads(threads)
    w = make_city(workload, seed)
    d = w.domain
    _, _, _, _, t_cal = _quiet(lambda: O.ref_solve(d, w, -1.0, 3, kind=1, want_lambda=False))
    per_it = max(t_cal / 3, 1e-6)
    sample = int(max(5, min(ITERMAX, seconds / per_it)))
    _, _, _, _, t = _quiet(lambda: O.ref_solve(d, w, -1.0, sample, kind=1, want_lambda=False))
    ms_it = 1e3 * t / sample
    iters = ref_iterations(f"{workload}:{seed}") or ref_iterations(workload)
    return ms_it, sample, iters


def run_reference(args):
    """The reference's Solver_CPU_RB on this host, per city of the headline
    batch: ms per iteration sampled on the first city (every city has the same
    grid), times the mean of the iterations the reference needs on each of the
    batch's cities (tests/golden/ref_iters.json, equal to this solver's plain
    iteration counts)."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    seed = SEED0 if args.workload == WORKLOAD else 0
    steps = []
    sample = iters = None
    for _ in range(max(args.steps, 1)):
        ms_it, sample, iters = reference_cpu_measure(args.workload, seed,
                                                     max(2.0, args.cpu_seconds / max(args.steps, 1)), threads)
        steps.append(ms_it)
    ms_it = statistics.median(steps)
    if args.workload == WORKLOAD:
        per_city = [ref_iterations(f"{WORKLOAD}:{SEED0 + i}") for i in range(args.batch)]
        if all(per_city):
            iters = float(np.mean(per_city))
    value = ms_it * iters if iters else None
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload} seeds {seed}..{seed + args.batch - 1}",
                   "solver": "Solver_CPU_RB (reference, OpenMP)",
                   "tol": TOL, "itermax": ITERMAX},
        "cpu_baseline": {"value": value, "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": f"{sample} red-black iterations per step timed on seed {seed}, x {iters} "
                                   f"iterations (mean over the batch's cities) the reference needs to reach "
                                   f"tol {TOL}"},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ms_per_iteration": ms_it,
    }
    print(json.dumps(line), flush=True)


def fp64_checks(w, seed, st, lam, winds):
    """The headline pipeline's FP32 result on one city against an FP64 run of
    the same SOR (same phases, same iteration counts, oracle restatement in
    double), and its FP64 final divergence against the reference solver's
    (Solver_CPU_RB run for the iterations it needs to reach the same rule)."""
    from oracle import oracle as O

    d = w.domain
    t0 = time.time()
    u64, v64, w64, L64, _, _ = O.solve_f64(d, w, -1.0, st["iterations"],
                                           phases=[(PRE_OMEGA, -1.0, st["pre_iterations"])])
    t_f64 = time.time() - t0
    lam_err = float(np.abs(lam.astype(np.float64) - L64).max() / max(np.abs(L64).max(), 1e-30))
    wind_err = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(winds, (u64, v64, w64)))
    out = {"seed": seed, "pre_iterations": st["pre_iterations"], "iterations": st["iterations"],
           "lambda_max_rel_err_vs_fp64": lam_err, "wind_max_err_vs_fp64_m_s": wind_err,
           "max_divergence_fp64": st["max_divergence"], "fp64_run_s": t_f64}
    riters = ref_iterations(f"{WORKLOAD}:{seed}")
    if riters:
        O.ref_set_threads(os.cpu_count() or 1)
        ur, vr, wr, _, _ = _quiet(lambda: O.ref_solve(d, w, -1.0, riters, kind=1, want_lambda=False))
        out["reference_max_divergence"] = O.max_divergence(d, w.icellflag, ur, vr, wr)
        out["reference"] = f"Solver_CPU_RB, {riters} iterations (its count to tol {TOL})"
    return out


def size_rates(peak, workloads=("city400", "city800")):
    """Sweep speed at the large single-city configurations: one autotuned
    solve of SIZE_ITERS iterations (tolerance 0, so every iteration runs)
    after a warm-up solve, per workload; the SOR time comes from the solve's
    own device events around its graphs."""
    import qesb

    out = {}
    for name in workloads:
        w, _ = qesb.random_city(name, 0)
        Nx, Ny, Nz = w.domain.base
        upd = (Nx - 2) * (Ny - 2) * (Nz - 1)
        with qesb.Solver_B200(w.domain, 0.0) as s:
            s.set_inputs(w)
            variant, _ = s.autotune()
            per = []
            for _ in range(3):
                s.resetLambda()
                st = s.solve(w, SIZE_ITERS, set_inputs=False)
                per.append(st["ms_sor"] / st["iterations"])
        ms_it = statistics.median(per[1:])
        alg = BYTES_PER_CELL_ITER * upd / (ms_it * 1e-3) / 1e9
        moved = MOVED_BYTES_PER_CELL_ITER * upd / (ms_it * 1e-3) / 1e9
        out[name] = {"grid": [Nx, Ny, Nz], "updated_cells": upd, "variant": variant, "iterations": SIZE_ITERS,
                     "us_per_iteration": 1e3 * ms_it, "algorithmic_gbs": alg, "algorithmic_frac": alg / peak,
                     "moved_gbs": moved, "moved_frac": moved / peak}
    return out


def fire_inflow(wgd, t, x0=60.0, speed=4.0, updraft=3.0, inflow=1.0, sigma=20.0, zc=30.0):
    """u0, v0, w0 of QES-Fire step t: the sensor field plus a synthetic
    fire-induced wind, for driving the solver as qesFireMain.cpp:232-259 does
    (u0 reset to the sensor field, fire winds added, solve without
    resetLambda). The fire physics (Fire::LevelSetNB, Fire::potential) is not
    on the solve path; this stand-in is a Gaussian updraft over a fire centre
    moving `speed` m per step along x at mid-y, with convergent horizontal
    inflow, fading above zc. Faces of solid cells are zeroed as
    Wall::setVelocityZero does (src/winds/Wall.cpp:805-825)."""
    d = wgd.domain
    nx, ny, nz = d.nx(), d.ny(), d.nz()
    dx, dy = d.dx(), d.dy()
    xf, yf = x0 + speed * t, 0.5 * (ny - 1) * dy
    zc_k = np.minimum(1.0, np.maximum(d.z[:nz - 1], 0.0) / zc)
    zk = np.concatenate([zc_k, zc_k[-1:]])[:, None, None]
    i = np.arange(nx)[None, None, :]
    j = np.arange(ny)[None, :, None]

    def gauss(x, y):
        return np.exp(-((x - xf) ** 2 + (y - yf) ** 2) / sigma ** 2)

    fade = np.exp(-np.maximum(np.concatenate([d.z, d.z[-1:]]) - zc, 0.0) / zc)[:, None, None]
    xu, yu = i * dx, (j + 0.5) * dy
    xv, yv = (i + 0.5) * dx, j * dy
    xw, yw = (i + 0.5) * dx, (j + 0.5) * dy
    du = -inflow * (xu - xf) / sigma * gauss(xu, yu) * fade
    dv = -inflow * (yv - yf) / sigma * gauss(xv, yv) * fade
    dw = updraft * gauss(xw, yw) * zk * fade
    import qesb

    out = qesb.WINDSGeneralData(d)  # shares the flags and coefficients
    out.icellflag, out.e, out.f, out.g, out.h, out.m, out.n = (wgd.icellflag, wgd.e, wgd.f, wgd.g, wgd.h, wgd.m,
                                                                wgd.n)
    shape = (nz, ny, nx)
    out.u0 = (wgd.u0.reshape(shape) + du).astype(np.float32).ravel()
    out.v0 = (wgd.v0.reshape(shape) + dv).astype(np.float32).ravel()
    out.w0 = (wgd.w0.reshape(shape) + dw).astype(np.float32).ravel()
    fl = wgd.icellflag.reshape(d.cell_shape())
    u0, v0, w0 = (a.reshape(shape) for a in (out.u0, out.v0, out.w0))
    solid = (fl == 0) | (fl == 2)
    ks, js, is_ = np.nonzero(solid[:, 1:ny - 1, 1:nx - 1])
    js, is_ = js + 1, is_ + 1
    for a, di, dj, dk in ((u0, 0, 0, 0), (u0, 1, 0, 0), (v0, 0, 0, 0), (v0, 0, 1, 0), (w0, 0, 0, 0), (w0, 0, 0, 1)):
        a[ks + dk, js + dj, is_ + di] = 0.0
    return out


def run_fire_loop(args, steps=None, print_line=True):
    """QES-Fire's solve pattern on one 256x256x64 city: a first solve from
    lambda = 0, then `steps` fire steps, each with new u0 (fire_inflow) and
    Solver::solve without resetLambda, so every solve starts from the previous
    step's lambda, as the reference's fire loop does. Three arms on the same
    inputs: warm (that behaviour), cold (resetLambda before every step), warm
    + over-relaxed pre-phase. Device time per solve (CUDA events) and
    iterations."""
    import torch

    import qesb

    steps = steps or args.fire_loop
    w, _ = qesb.random_city(args.workload, SEED0)
    d = w.domain
    seq = [fire_inflow(w, t) for t in range(1, steps + 1)]
    arms = {}
    with qesb.Solver_B200(d, TOL) as s:
        s.set_inputs(w)
        s.autotune()
        for arm in ("warm", "cold", "warm+prephase"):
            s.set_prephase(PRE_OMEGA if arm == "warm+prephase" else 0.0, PRE_TOL, ITERMAX)
            s.resetLambda()
            s.solve(w, ITERMAX)
            its, pre, ms = [], [], []
            for wt in seq:
                if arm == "cold":
                    s.resetLambda()
                st = s.solve(wt, ITERMAX)
                its.append(st["iterations"])
                pre.append(st["pre_iterations"])
                ms.append(st["ms_total"])
            arms[arm] = {"ms_per_solve": float(np.mean(ms)), "iterations": its, "pre_iterations": pre}
        torch.cuda.synchronize()
    out = {"fire_loop": {"workload": f"{args.workload} seed {SEED0}", "steps": steps,
                         "perturbation": "synthetic fire-induced winds: 3 m/s Gaussian updraft (sigma 20 m) and "
                                         "1 m/s convergent inflow over a fire centre moving 4 m per step",
                         "arms": arms,
                         "speedup_warm_vs_cold": arms["cold"]["ms_per_solve"] / arms["warm"]["ms_per_solve"]}}
    if print_line:
        print(json.dumps(out), flush=True)
    return out["fire_loop"]


def network_flops(net, s):
    """Multiply-add FLOPs of one forward pass (2 per MAC, real channels)."""
    total = 0
    for name, L in net.layers.items():
        lvl = 0 if name == "head" else int(name[1])
        total += 2 * 27 * L.cin * L.cout * s.V(lvl)
    return total


def run_b200(args):
    import torch

    import qesb
    from qesb import warmstart as ws

    rank, local, world = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    B = args.batch
    seeds = [SEED0 + rank * B + i for i in range(B)]  # each rank its own batch: weak scaling
    cities = [make_city(args.workload, sd) for sd in seeds]
    d0 = cities[0].domain
    Nx, Ny, Nz = d0.base
    updated = (Nx - 2) * (Ny - 2) * (Nz - 1)
    nf = d0.numFaceCentered()

    solvers = [qesb.Solver_B200(w.domain, TOL, device=dev) for w in cities]
    for s, w in zip(solvers, cities):
        s.set_stream(stream.cuda_stream)
        s.set_inputs(w)
    # autotuners (untimed set-up, like a library's algorithm search): the sweep
    # shape for single solves of this grid, and the one for this batch's list
    variant, variant_us = solvers[0].autotune()
    batch_variant, _ = qesb.autotune_batch(solvers)
    wpath = args.weights or ws.DEFAULT_WEIGHTS
    net = ws.WarmStartNet.from_file(wpath, device=dev)

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

    outs = [[torch.empty(nf, dtype=torch.float32, device=f"cuda:{dev}") for _ in range(3)] for _ in range(B)]
    uvw = [[o[q].data_ptr() for o in outs] for q in range(3)]
    launches_per_warm = 4 + (4 * net.nlev - 1) + (net.nlev - 1)  # R, input (2), apply + convs + pools

    def set_pre(on):
        for s in solvers:
            s.set_prephase(PRE_OMEGA if on else 0.0, PRE_TOL, ITERMAX)

    def batch_step(use_net, use_pre):
        def step():
            set_pre(use_pre)
            for s in solvers:
                if use_net:
                    net.warm_start(s, stream.cuda_stream)
                else:
                    s.resetLambda()
            st = qesb.solve_batch(solvers, ITERMAX, *uvw)
            return st, (B * launches_per_warm if use_net else 0) + 6 * B + 1 + st[0]["launches"]
        return step

    warm_step = batch_step(False, True)  # the headline pipeline: over-relaxed pre-phase, reference loop

    def plain_single_step():
        set_pre(False)
        sts = []
        for s, o in zip(solvers, outs):
            s.resetLambda()
            sts.append(s.solve_device(ITERMAX, o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr()))
        return sts, sum(x["launches"] for x in sts)

    def timed(fn, steps, warmup, clocks=False):
        # the clock sampler starts before the warm-up so that its first samples
        # (nvidia-smi takes a moment to start) fall inside the timed region
        clk = ClockSampler(dev) if clocks else None
        if clk:
            clk.__enter__()
            time.sleep(0.3)
        for _ in range(warmup):
            fn()
        barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        res, launches = [], 0
        if clk:
            clk.lines.clear()  # keep only the samples taken while the timed steps run
        e0.record(stream)
        for _ in range(steps):
            r, n = fn()
            res.append(r)
            launches += n
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if clk:
            clk.__exit__()
        barrier()
        return e0.elapsed_time(e1) / steps, res, launches, (clk.summary() if clk else None)

    # converged fields of the first two domains (long over-relaxed runs, untimed)
    # to state each arm's wind error
    conv = []
    for s, o in list(zip(solvers, outs))[:2]:
        s.set_prephase(PRE_OMEGA, -1.0, 4000)
        s.resetLambda()
        s.solve_device(1, o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr())
        conv.append([t.clone() for t in o])

    def wind_err():
        return max(float((o[q] - c[q]).abs().max()) for o, c in zip(outs, conv) for q in range(3))

    arms = {}
    for name, (use_net, use_pre) in {"plain": (False, False), "network": (True, False),
                                     "network+prephase": (True, True)}.items():
        ms, res, _, _ = timed(batch_step(use_net, use_pre), max(1, args.steps // 2), 1)
        arms[name] = {"ms_per_domain": max_over_ranks(ms) / B, "iterations": [x["iterations"] for x in res[-1]],
                      "pre_iterations": [x["pre_iterations"] for x in res[-1]], "wind_err_vs_converged": wind_err()}
    ms_warm, res_warm, launches, clocks = timed(warm_step, args.steps, args.warmup, clocks=True)
    ms_warm = max_over_ranks(ms_warm)
    arms["prephase"] = {"ms_per_domain": ms_warm / B, "iterations": [x["iterations"] for x in res_warm[-1]],
                        "pre_iterations": [x["pre_iterations"] for x in res_warm[-1]],
                        "wind_err_vs_converged": wind_err()}
    ms_plain = arms["plain"]["ms_per_domain"] * B
    ms_single, res_single, _, _ = timed(plain_single_step, 1, 1)

    def first_domain_warm():  # the headline pipeline on domain 0 alone (reference GPU comparison)
        s, o = solvers[0], outs[0]
        s.set_prephase(PRE_OMEGA, PRE_TOL, ITERMAX)
        s.resetLambda()
        return s.solve_device(ITERMAX, o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr()), 0

    ms_first, res_first, _, _ = timed(first_domain_warm, 3, 1)
    st_first = res_first[-1]
    lam_first = solvers[0].lambda_
    winds_first = [t.cpu().numpy() for t in outs[0]]

    # ---- end to end through the host API (warm step) -------------------------
    host_keep = [[pinned_copy(torch, a) for a in w.inputs()] for w in cities]  # tensors own the pinned memory
    host_in = [[arr for _, arr in ins] for ins in host_keep]
    host_out = [[torch.empty(nf, dtype=torch.float32, pin_memory=True) for _ in range(3)] for _ in range(B)]
    h2d = sum(a.nbytes for ins in host_in for a in ins)
    d2h = 3 * 4 * nf * B

    def e2e_step():
        for s, ins in zip(solvers, host_in):
            qesb.check(qesb.lib().qesb_set_inputs(s._h, *[a.ctypes.data for a in ins]))
        st, n = warm_step()
        with torch.cuda.stream(stream):
            for o, ho in zip(outs, host_out):
                for q in range(3):
                    ho[q].copy_(o[q], non_blocking=True)
        return st, n

    ms_e2e_serial, _, _, _ = timed(e2e_step, max(1, args.steps // 2), 1)
    torch.cuda.synchronize(dev)
    ms_e2e_serial = max_over_ranks(ms_e2e_serial)

    # Pipelined, as a stream of batches runs: two solver sets on two streams.
    # While one batch solves and its winds are read back, a second host thread
    # loads the next batch's inputs through the same public call
    # (qesb_set_inputs, host -> device, blocking that thread only). Every
    # step's copies still run inside the timed region, the first batch's
    # upload before any overlap; only their order against the other batch's
    # solve changes.
    import threading

    stream2 = torch.cuda.Stream(device=dev)
    solvers2 = [qesb.Solver_B200(w.domain, TOL, device=dev) for w in cities]
    for s2 in solvers2:
        s2.set_stream(stream2.cuda_stream)
        s2.set_prephase(PRE_OMEGA, PRE_TOL, ITERMAX)
    solvers2[0].set_option("batch_variant", batch_variant)
    sets, streams = [solvers, solvers2], [stream, stream2]
    outs2 = [[torch.empty(nf, dtype=torch.float32, device=f"cuda:{dev}") for _ in range(3)] for _ in range(B)]
    set_outs = [outs, outs2]
    set_uvw = [uvw, [[o[q].data_ptr() for o in outs2] for q in range(3)]]
    host_out2 = [[torch.empty(nf, dtype=torch.float32, pin_memory=True) for _ in range(3)] for _ in range(B)]
    set_host_out = [host_out, host_out2]

    def load(k):
        for s_, ins in zip(sets[k], host_in):
            qesb.check(qesb.lib().qesb_set_inputs(s_._h, *[a.ctypes.data for a in ins]))

    def solve_read(k):
        for s_ in sets[k]:
            s_.set_prephase(PRE_OMEGA, PRE_TOL, ITERMAX)
            s_.resetLambda()
        st_ = qesb.solve_batch(sets[k], ITERMAX, *set_uvw[k])
        with torch.cuda.stream(streams[k]):
            for o, ho in zip(set_outs[k], set_host_out[k]):
                for q in range(3):
                    ho[q].copy_(o[q], non_blocking=True)
        return st_

    def pipelined(nsteps):
        load(0)
        for i in range(nsteps):
            cur = i % 2
            failed = []

            def load_next(k=1 - cur):
                try:
                    load(k)
                except Exception as ex:  # noqa: BLE001  (re-raised below, in the timing thread)
                    failed.append(ex)

            th = threading.Thread(target=load_next) if i + 1 < nsteps else None
            if th:
                th.start()
            solve_read(cur)
            if th:
                th.join()
            if failed:
                raise failed[0]
        torch.cuda.synchronize(dev)

    pipelined(2)  # warm-up
    k_e2e = max(2, args.steps // 2)
    barrier()
    torch.cuda.synchronize(dev)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    pipelined(k_e2e)
    p1.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = max_over_ranks(p0.elapsed_time(p1) / k_e2e)
    last = (k_e2e - 1) % 2
    e2e_ok = all(torch.equal(ho[0], o[0].cpu()) for ho, o in zip(set_host_out[last], set_outs[last]))
    e2e_ok = e2e_ok and all(torch.equal(a[0], b[0]) for a, b in zip(set_outs[last], outs if last else outs2))
    for s2 in solvers2:
        s2.close()

    # ---- roofline of the dominant kernel: the list sweep of the headline step ---------
    # The headline step is ~97 % red/black list sweeps. Its domain-iterations
    # (pre-phase and reference loop, every domain) times the algorithmic bytes
    # per updated cell, over the whole timed step (R, layout changes and the
    # correction included), is a lower bound on the sweep kernel's rate. One
    # launch is a half-sweep over the active list; per launch of the full list
    # that is 1/2 x batch x updated cells x 36 B.
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
        tpeak = float(peaks.get("bf16_tflops", 1590.0))
    except (OSError, KeyError, ValueError):
        peak, peak_src, tpeak = 6650.0, "fallback", 1590.0
    dom_iters = sum(x["iterations"] + x["pre_iterations"] for x in res_warm[-1])
    achieved = BYTES_PER_CELL_ITER * updated * dom_iters / (ms_warm * 1e-3) / 1e9
    moved = MOVED_BYTES_PER_CELL_ITER * updated * dom_iters / (ms_warm * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "sor_zm_batch_city256.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except ValueError:
            traffic = None
    headline_sweep = {"domain_iterations": dom_iters, "us_per_domain_iteration": 1e3 * ms_warm / dom_iters,
                      "moved_gbs_lower_bound": moved, "moved_frac": moved / peak, "batch_variant": batch_variant}

    # the same kernel family on one domain at a time (the plain single solves)
    sor_ms = [x["ms_sor"] / max(x["iterations"], 1) for x in res_single[-1]]
    ms_it = statistics.median(sor_ms)
    alg_bytes = BYTES_PER_CELL_ITER * updated
    single_domain = {"kernel": "red+black sweep pair (variant %d), per iteration inside the solve graphs" % variant,
                     "ms_per_iteration": ms_it, "algorithmic_bytes_per_iteration": alg_bytes,
                     "achieved": alg_bytes / (ms_it * 1e-3) / 1e9,
                     "frac": alg_bytes / (ms_it * 1e-3) / 1e9 / peak,
                     "note": "one 256^2 domain's sweep data (~70 MB) stays in L2 between launches"}

    # ---- the sweep at the 400^2 x 100 and 800^2 x 128 configurations ------------------
    sizes = None
    if not args.no_sizes:
        try:
            sizes = size_rates(peak)
        except Exception as ex:  # noqa: BLE001
            sizes = {"unavailable": str(ex)[:200]}

    # ---- the network alone ---------------------------------------------------------
    s0 = net.net_shapes(solvers[0])
    fwd = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(2):
        net.forward(s0, stream.cuda_stream)
    fwd[0].record(stream)
    nf_rep = 5
    for _ in range(nf_rep):
        net.forward(s0, stream.cuda_stream)
    fwd[1].record(stream)
    torch.cuda.synchronize(dev)
    ms_fwd = fwd[0].elapsed_time(fwd[1]) / nf_rep
    flops = network_flops(net, s0)

    # ---- QES-Fire's solve pattern: fire steps warm-started from the previous lambda ----
    fire = None
    if not args.no_fire_loop and rank == 0:
        try:
            fire = run_fire_loop(args, steps=8, print_line=False)
        except Exception as ex:  # noqa: BLE001
            fire = {"unavailable": str(ex)[:200]}

    # ---- log-law wall treatment (Wall::wallLogBC) on domain 0's solved winds --------
    wall_log = None
    try:
        tmp = [o.clone() for o in outs[0]]
        dzn = float(np.min(d0.dz_array))
        solvers[0].wall_log_law(0.1, dzn, *[x.data_ptr() for x in tmp])
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        for _ in range(5):
            solvers[0].wall_log_law(0.1, dzn, *[x.data_ptr() for x in tmp])
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
        wall_log = {"us_per_call": 1e3 * ev[0].elapsed_time(ev[1]) / 5, "launches_per_call": 7, "z0": 0.1,
                    "workload": "domain 0 of the headline batch, after its solve"}
    except Exception as ex:  # noqa: BLE001
        wall_log = {"unavailable": str(ex)[:200]}

    # ---- reference GPU solver, CPU baseline, FP64 checks (rank 0, N = 1) --------------
    ref_gpu = None
    cpu = None
    precision = None
    if rank == 0 and world == 1:
        for s in solvers:
            s.close()
        solvers = []
        torch.cuda.synchronize(dev)
        if not args.no_reference_gpu:
            try:
                from oracle import oracle as O

                if O.ref_gpu_available():
                    w = cities[0]
                    u, v, ww, secs, iters = O.ref_solve_gpu(w.domain, w, TOL, ITERMAX)
                    ref_gpu = {"ms": 1e3 * secs, "iterations": iters, "seed": seeds[0],
                               "solver": "Solver_GPU_GlobalMemory::solve (reference, wall clock incl. its "
                                         "allocations and copies)"}
                else:
                    ref_gpu = {"unavailable": "oracle/_ref/libqesref_gpu.so not built"}
            except Exception as ex:  # noqa: BLE001
                ref_gpu = {"unavailable": str(ex)[:200]}
        if not args.no_fp64:
            try:
                precision = fp64_checks(cities[0], seeds[0], st_first, lam_first, winds_first)
            except Exception as ex:  # noqa: BLE001
                precision = {"unavailable": str(ex)[:200]}
        if not args.no_cpu_baseline:
            try:
                threads = os.cpu_count() or 1
                ms_c, sample, riters = reference_cpu_measure(args.workload, seeds[0], args.cpu_seconds, threads)
                per_city = [ref_iterations(f"{args.workload}:{sd}") for sd in seeds]
                if all(per_city):
                    riters = float(np.mean(per_city))
                cpu = {"value": ms_c * riters if riters else None, "unit": "ms", "cores": threads,
                       "kind": "reference",
                       "sample": f"Solver_CPU_RB on seed {seeds[0]}: {sample} iterations timed "
                                 f"({ms_c:.2f} ms/iteration) x {riters} iterations to tol {TOL} (mean over "
                                 f"the batch's cities)"}
            except Exception as ex:  # noqa: BLE001
                cpu = {"value": None, "unit": "ms", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {ex}"}
    for s in solvers:
        s.close()

    if rank == 0:
        value = ms_warm / B
        line = {
            "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_warm, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.workload} ({Nx}x{Ny}x{Nz}), held-out seeds {seeds[0]}..{seeds[-1]} "
                                   f"(+{B} per rank)",
                       "batch": B, "tol": TOL, "itermax": ITERMAX, "network": os.path.basename(wpath),
                       "network_levels": net.nlev, "channels": list(net.CH),
                       "sweep_variant": variant, "batch_variant": batch_variant,
                       "parallelism": f"replicas x{world}",
                       "warm_start": f"red-black SOR at omega {PRE_OMEGA} from lambda = 0 to max|dlambda| <= "
                                     f"{PRE_TOL}, then the reference loop (omega 1.78, tol {TOL}); the learned "
                                     f"network's start is measured in arms (network, network+prephase) and is "
                                     f"not in this pipeline because it does not shorten it",
                       "l2": "8 domains x ~40 MB packed sweep data + network buffers > L2 (126 MB) per step"},
            "arms": arms,
            "network_ms_per_domain": ms_fwd,
            "plain_single": {"ms_per_domain": ms_single / B,
                             "iterations": [x["iterations"] for x in res_single[-1]]},
            "speedup_vs_plain": (ms_plain / ms_warm),
            "reference_gpu": ref_gpu,
            "first_domain_ms": ms_first,
            "speedup_vs_reference_gpu": (ref_gpu["ms"] / ms_first) if ref_gpu and "ms" in ref_gpu else None,
            "e2e": {"value": ms_e2e / B, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "matches_device_result": bool(e2e_ok),
                    "how": "public API (qesb_set_inputs from pinned host arrays, qesb_solve_batch, winds read "
                           "back to pinned host memory) on two solver sets: the next batch's inputs load on a "
                           "second host thread while the current batch solves; device-timed over the steps",
                    "serial_value": ms_e2e_serial / B},
            "headline_sweep": headline_sweep,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "kernel": "red/black list sweep (variant %d) over the batch's domains, timed as the "
                                   "whole headline step (lower bound)" % batch_variant,
                         "algorithmic_bytes_per_launch": BYTES_PER_CELL_ITER * updated * B // 2,
                         "moved_frac": moved / peak, "single_domain": single_domain},
            "sizes": sizes,
            "wall_log_law": wall_log,
            "fire_loop": fire,
            "network": {"bound": "tensor", "ms_per_forward": ms_fwd, "flops_per_forward": flops,
                        "achieved_tflops": flops / (ms_fwd * 1e-3) / 1e12, "peak_tflops": tpeak,
                        "frac": flops / (ms_fwd * 1e-3) / 1e12 / tpeak},
            "precision": precision,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        barrier()  # rank 0 ran the fire-step section alone: the ranks leave together
        dist.destroy_process_group()


def run_ensemble(args):
    """Batched ensemble: cities with Nx, Ny ~ U[64, 256] and Nz ~ U[32, 96]
    (dx = dy = 2 m, z stretched 1.03, building count scaled from the 400 x 400
    config's 60), each at 36 wind directions 10 degrees apart. The 36 solves of
    a city run as one qesb_solve_batch (inputs built on the device beforehand
    and reported as setup_ms_per_solve; only the batch is timed, CUDA events): over-relaxed pre-phase warm start, reference
    loop, correction; the list sweep's launch shape tuned once (qesb_autotune_batch
    on the first city's 36 solves) and used for every city. solves/s = all solves /
    the sum of batch times; latency of a solve = device time from its batch's
    first sweep to the poll that ended it."""
    import torch

    import qesb

    from qesb import shard

    rank, local, world = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    rng = np.random.default_rng(20260907)
    nd, ndir = args.ensemble_domains, 36
    dims = [(int(a), int(b), int(c)) for a, b, c in zip(rng.integers(64, 257, nd), rng.integers(64, 257, nd),
                                                       rng.integers(32, 97, nd))]
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    lat, batch_ms, iters, pre_iters, cells_total = [], [], [], [], 0
    shapes, setup_ms = [], []
    batch_shape = None  # the list sweep shape, tuned once on the first city's batch
    for d in shard.rank_share(nd, world, rank):  # cities of this rank; none crosses ranks
        Nx, Ny, Nz = dims[d]
        dom = qesb.Domain(Nx, Ny, Nz, 2.0, 2.0, 1.0, qesb.city_dz(Nz, 1.0, 1.03))
        nb = max(3, int(round(60 * Nx * Ny / 160000)))
        c = qesb.city_random(dom, 700000 + d, nb)
        solvers = [qesb.Solver_B200(dom, TOL, device=dev) for _ in range(ndir)]
        try:
            om = qesb.prephase_omega(Nx, Ny)
            # inputs built on the device (qesb_city_build_device), one set per
            # direction, handed to the handles as device arrays
            nc_, nf_ = dom.numCellCentered(), dom.numFaceCentered()
            names = ("icellflag", "e", "f", "g", "h", "m", "n", "u0", "v0", "w0")
            torch.cuda.synchronize(dev)
            t_set = time.perf_counter()
            arrays = []
            for k in range(ndir):
                a = {q: torch.empty(nc_ if q not in ("u0", "v0", "w0") else nf_,
                                    dtype=torch.int32 if q == "icellflag" else torch.float32,
                                    device=f"cuda:{dev}") for q in names}
                torch.cuda.current_stream(dev).synchronize()
                qesb.city_build_device(dom, c.buildings,
                                       qesb.Inflow(c.inflow.u_ref, c.inflow.z_ref, c.inflow.p, 10.0 * k),
                                       {q: v.data_ptr() for q, v in a.items()}, stream.cuda_stream)
                arrays.append(a)
            for s, a in zip(solvers, arrays):
                s.set_stream(stream.cuda_stream)
                s.set_inputs_device(*[a[q].data_ptr() for q in ("e", "f", "g", "h", "m", "n", "icellflag", "u0",
                                                                 "v0", "w0")])
                s.set_prephase(om, PRE_TOL, ITERMAX)
            torch.cuda.synchronize(dev)
            setup_ms.append(1e3 * (time.perf_counter() - t_set))
            if batch_shape is None:
                batch_shape, _ = qesb.autotune_batch(solvers)
            solvers[0].set_option("batch_variant", batch_shape)
            nf = dom.numFaceCentered()
            outs = [[torch.empty(nf, dtype=torch.float32, device=f"cuda:{dev}") for _ in range(3)]
                    for _ in range(ndir)]
            ptrs = [[o[q].data_ptr() for o in outs] for q in range(3)]
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = qesb.solve_batch(solvers, ITERMAX, *ptrs)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            batch_ms.append(e0.elapsed_time(e1))
            lat += [x["ms_sor"] for x in st]
            iters += [x["iterations"] for x in st]
            pre_iters += [x["pre_iterations"] for x in st]
            assert all(x["converged"] for x in st)
        finally:
            for s in solvers:
                s.close()
        cells_total += ndir * Nx * Ny * (Nz + 1)
        shapes.append((Nx, Ny, Nz))
    total_ms = shard.max_over_ranks(float(np.sum(batch_ms)), device=f"cuda:{dev}" if world > 1 else None)
    setup_total = shard.max_over_ranks(float(np.sum(setup_ms)), device=f"cuda:{dev}" if world > 1 else None)
    lat = shard.gather_lists(lat)
    iters, pre_iters = shard.gather_lists(iters), shard.gather_lists(pre_iters)
    cells_total = int(sum(shard.gather_lists([cells_total])))
    shapes = shard.gather_lists(shapes)
    n = nd * ndir
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "ensemble solves/s (cities of uneven size x 36 wind directions, batched)",
        "value": n / (total_ms * 1e-3), "unit": "solves/s", "n_gpus": world, "higher_is_better": True,
        "scaling": "strong",
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{nd} cities, Nx,Ny ~ U[64,256], Nz ~ U[32,96], x {ndir} directions",
                   "solves": n, "batch": ndir, "tol": TOL, "itermax": ITERMAX,
                   "warm_start": "over-relaxed pre-phase, omega = 2 - 7.5/max(Nx, Ny) within [1.85, 1.97], "
                                 f"to {PRE_TOL}", "cells_total": cells_total, "batch_variant": batch_shape},
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "setup_ms_per_solve": setup_total / n,
        "setup": "inputs (flags, wall coefficients, winds) built on the device by qesb_city_build_device "
                 "and handed over with qesb_set_inputs_device; wall clock, not in value",
        "ms_total": total_ms, "iterations_mean": float(np.mean(iters)),
        "pre_iterations_mean": float(np.mean(pre_iters)),
        "mcell_iterations_per_s": float(sum(ndir * (a - 2) * (b - 2) * (z - 1) * 1.0 for a, b, z in shapes) *
                                        (np.mean(iters) + np.mean(pre_iters)) / (total_ms * 1e-3) / 1e6),
    }
    print(json.dumps(line), flush=True)


def run_sweeps_only(args):
    import qesb

    w = make_city(args.workload, SEED0 if args.workload == WORKLOAD else 0)
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

    w = make_city(args.workload, SEED0 if args.workload == WORKLOAD else 0)
    with qesb.Solver_B200(w.domain, 0.0) as s:
        if args.variant >= 0:
            s.set_option("variant", args.variant)
        st = s.solve(w, args.profile_solve)
    print(json.dumps({"profile_solve": args.profile_solve, **st}))


def run_profile_batch(args):
    """The headline step (a batch of B cities, over-relaxed pre-phase, reference
    loop, correction) twice, for launch-list captures."""
    import torch

    import qesb

    cities = [make_city(args.workload, SEED0 + i) for i in range(args.batch)]
    solvers = [qesb.Solver_B200(w.domain, TOL) for w in cities]
    try:
        for s, w in zip(solvers, cities):
            s.set_inputs(w)
            s.set_prephase(PRE_OMEGA, PRE_TOL, ITERMAX)
        if args.variant >= 0:
            solvers[0].set_option("variant", args.variant)
        nf = cities[0].domain.numFaceCentered()
        outs = [[torch.empty(nf, dtype=torch.float32, device="cuda:0") for _ in range(3)] for _ in cities]
        ptrs = [[o[q].data_ptr() for o in outs] for q in range(3)]
        for _ in range(2):
            for s in solvers:
                s.resetLambda()
            st = qesb.solve_batch(solvers, ITERMAX, *ptrs)
        torch.cuda.synchronize()
    finally:
        for s in solvers:
            s.close()
    print(json.dumps({"profile_batch": args.batch, "iterations": [x["iterations"] for x in st],
                      "pre_iterations": [x["pre_iterations"] for x in st]}))


def run_forward_only(args):
    """Warm-start forward passes on one domain, for network captures."""
    import torch

    import qesb
    from qesb import warmstart as ws

    w = make_city(args.workload, SEED0 if args.workload == WORKLOAD else 0)
    net = ws.WarmStartNet.from_file(args.weights or ws.DEFAULT_WEIGHTS, device=0)
    with qesb.Solver_B200(w.domain, TOL) as s:
        s.set_inputs(w)
        for _ in range(args.forward_only):
            net.warm_start(s)
        torch.cuda.synchronize()
        net.check_err()
    print(json.dumps({"forward_only": args.forward_only}))


def main():
    args = parse()
    if args.profile_solve:
        run_profile_solve(args)
    elif args.sweeps_only:
        run_sweeps_only(args)
    elif args.forward_only:
        run_forward_only(args)
    elif args.profile_batch:
        run_profile_batch(args)
    elif args.ensemble:
        run_ensemble(args)
    elif args.fire_loop:
        run_fire_loop(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
