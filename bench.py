"""Benchmark: ms to the SOR stopping rule per domain, learned warm start vs
plain SOR, on one B200 per rank.

Workload: held-out synthetic cities of 256 x 256 x 64 cells (dx = dy = 2 m,
z stretched 1 m x 1.03^k, 40-80 seed-placed cuboid buildings, power-law
inflow from a random direction), seeds 500000 + i, disjoint from the
warm-start network's training seeds. One step = one batch of B domains
(default 8) taken from their inputs in HBM to corrected winds in HBM.

Stopping rule, the same for every arm and for the reference: the reference
loop `while (iter < itermax && max_error > tol)` with the reference's own
tol = 1e-9 (never met in FP32) and itermax = 10000, plus the window rule:
after every WINDOW-th iteration n the loop also ends when
max|lambda_n - lambda_(n - WINDOW)| <= WINDOW_TOL (FP64, all cells). With
it, plain SOR's winds land within 1e-3 m/s of the converged field; the
per-iteration change alone never falls below the FP32 rounding flutter.

Arms (all batched, qesb_solve_batch, each domain stopping on its own):
  plain             red-black SOR from lambda = 0 (the method's fallback and judge)
  prephase          an over-relaxed red-black pre-phase from lambda = 0 (omega
                    PRE_OMEGA to max|dlambda| <= PRE_TOL) as the warm start
  network           the learned network's prediction as the start
  network+prephase  the network's start, then the pre-phase
each then running the reference loop to the rule and the velocity
correction. `value` is the HEADLINE arm's ms per domain = step time / B.

  e2e            the headline step through the host API: pinned host inputs
                 copied in (qesb_set_inputs), u, v, w copied out, each step.
  roofline       the red/black list sweep, the kernel that dominates the step:
                 the bytes the layout moves per updated cell and iteration
                 (17 B) over the device time of every sweep launch of the timed
                 steps (CUDA events around the sweep loops, qesb_stats.ms_sweeps).
  cpu_baseline   the reference's Solver_CPU_RB (oracle/_ref) run in full, to
                 the rule's iteration count, on this host's cores.

--impl reference runs only the reference CPU solver (rank 0), same metric.
--gpus N without torchrun re-launches itself as N ranks; each rank solves
its own batch (seeds offset by rank); no data crosses ranks ("scaling": "weak").
"""
import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "qes-public_b200"))
sys.path.insert(0, ROOT)

TOL = 1e-9          # the reference's own tolerance (Solver.h), never met in FP32
ITERMAX = 10000
WINDOW, WINDOW_TOL = 32, 4e-3
WORKLOAD = "city256"
SEED0 = 500000
METRIC = "ms to SOR tolerance per domain: learned warm start vs plain SOR, 1 B200"
# Bytes the packed red/black sweep must move per updated cell and iteration:
# its colour's lambda read + write (8), the other colour's lambda read (4),
# R (4) and the wall mask (1).
MOVED_BYTES_PER_CELL_ITER = 17
ALG_BYTES_PER_CELL_ITER = 36  # 6 coefficients + R read (28 B), lambda read + write (8 B)
SIZE_ITERS = 300  # iterations per timed solve of the size sweep
PRE_OMEGA = 1.97
PRE_TOL = 2e-3
HEADLINE = "network+prephase"  # the metric's method: the learned start, then the pre-phase
ARMS = {"plain": (False, False), "prephase": (False, True), "network": (True, False),
        "network+prephase": (True, True)}
# After the network's start the pre-phase begins with a few sweeps at a smaller
# omega (qesb_set_prephase_start), which damp the start's rough, wall-adjacent
# error before the over-relaxation amplifies it; from lambda = 0 there is
# nothing rough to damp and the pre-phase starts at once.
START_STAGE = (1.8, 8)


def start_stage(use_net, use_pre):
    return START_STAGE if use_net and use_pre else (0.0, 0)


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--batch", type=int, default=8, help="domains per step")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend for N > 1 (gloo: the CPU rehearsal of --plan)")
    ap.add_argument("--plan", action="store_true",
                    help="print each rank's share of the work and exit (no GPU work; runs on CPU with gloo)")
    ap.add_argument("--weights", default=None, help="warm-start network (default: the committed weights)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 same-SOR error and divergence checks")
    ap.add_argument("--no-sizes", action="store_true", help="skip the 400^2 and 800^2 sweep-speed section")
    ap.add_argument("--no-fire-loop", action="store_true", help="skip the fire-step section")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble section")
    ap.add_argument("--variant", type=int, default=-1, help="sweep variant for the profiling drivers (-1: autotune)")
    ap.add_argument("--profile-solve", type=int, default=0,
                    help="profiling driver: one solve of this many iterations (tol 0) with --variant, exit")
    ap.add_argument("--sweeps-only", type=int, default=0,
                    help="profiling driver: set up the workload, run this many sweep launches, exit")
    ap.add_argument("--ensemble", action="store_true",
                    help="batched ensemble alone: cities of uneven size x 36 wind directions (solves/s, p50/p99)")
    ap.add_argument("--ensemble-domains", type=int, default=64)
    ap.add_argument("--ensemble-list-cells", type=int, default=250_000_000,
                    help="cells per ensemble launch list (whole cities; 0: one city per list)")
    ap.add_argument("--fire-loop", type=int, default=0,
                    help="QES-Fire solve pattern: this many fire steps warm-started from the previous lambda, exit")
    ap.add_argument("--profile-batch", action="store_true",
                    help="profiling driver: the headline batch once untimed, once more, exit")
    ap.add_argument("--conv-path", type=int, default=0,
                    help="network convolution kernels for --forward-only (qesb_net_set_conv_path)")
    ap.add_argument("--forward-only", type=int, default=0,
                    help="profiling driver: run this many warm-start forward passes on one domain, exit")
    return ap.parse_args(argv)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def maybe_relaunch(args):
    """--gpus N > 1 outside torchrun: run this script as N ranks (one process
    per GPU) and exit with their status. Inside torchrun the world size must
    be N."""
    from qesb import shard

    world = int(os.environ.get("WORLD_SIZE", 0))
    if world == 0 and args.gpus > 1:
        cmd = shard.launch_command(sys.executable, os.path.abspath(__file__), args.gpus, _free_port(), sys.argv[1:])
        sys.exit(subprocess.call(cmd))
    if world and world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE {world}")


def init_group(args, world, local):
    """Process group of the ranks (no-op for one rank): NCCL over the GPUs, or
    gloo for the CPU rehearsal; a short timeout so that a missing rank ends in
    an error."""
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    if args.backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=300))
    return dist


def run_plan(args):
    """Each rank's share of the headline workload, gathered and printed by
    rank 0 (the launch and sharding logic without GPU work)."""
    from qesb import shard

    rank, local, world = dist_env()
    dist = init_group(args, world, local)
    mine = {"rank": rank, "seeds": shard.rank_seeds(SEED0, args.batch, rank)}
    everything = shard.gather_lists([mine])
    comm = dist.get_world_size() if dist else 1
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"plan": {"world": world, "communicator_size": comm, "backend": args.backend,
                                   "shares": sorted(everything, key=lambda x: x["rank"])}}), flush=True)


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


def ref_counts():
    """The reference's own iteration counts to the rule (tests/golden/ref_iters.json,
    made by tests/golden/make_ref_iters.py from the reference build)."""
    path = os.path.join(ROOT, "tests", "golden", "ref_iters.json")
    doc = json.load(open(path))
    r = doc["rule"]
    assert (r["tol"], r["itermax"], r["window"], r["window_tol"]) == (TOL, ITERMAX, WINDOW, WINDOW_TOL), r
    return doc


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


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


# ---------------------------------------------------------------------------
# the reference on the host
# ---------------------------------------------------------------------------
def reference_solves(seeds, threads, counts, keep_winds=False):
    """Full solves of the reference's Solver_CPU_RB (oracle/_ref) on the
    seeds' cities, built without the product library (oracle/city.py), each
    for the iterations the reference needs to reach the rule (tol < 0 and
    itermax = that count: the same iterates as the rule's run, without the
    OpenMP race on its max_error reset, Solver_CPU_RB.cpp:166). Returns
    [(seed, seconds of solve(), iterations, winds or None)]."""
    from oracle import city as OC
    from oracle import oracle as O

    O.ref_set_threads(threads)
    out = []
    for seed in seeds:
        w = OC.random_city(WORKLOAD, seed)
        n = counts[f"{WORKLOAD}:{seed}"]["Solver_CPU_RB"]["iterations"]
        u, v, ww, _, t = _quiet(lambda: O.ref_solve(w.domain, w, -1.0, n, kind=1, want_lambda=False))
        out.append((seed, t, n, (w, u, v, ww) if keep_winds else None))
    return out


def serial_solver_cpu_sample(seed, counts, iters=60):
    """Serial Solver_CPU (the reference's default build) timed on a bounded
    sample of its iterations on one core, and its own iteration count to the
    rule: the extrapolated time of one full serial solve."""
    from oracle import city as OC
    from oracle import oracle as O

    w = OC.random_city(WORKLOAD, seed)
    _, _, _, _, t = _quiet(lambda: O.ref_solve(w.domain, w, -1.0, iters, kind=0, want_lambda=False))
    n = counts[f"{WORKLOAD}:{seed}"]["Solver_CPU"]["iterations"]
    return {"seed": seed, "iterations_timed": iters, "ms_per_iteration": 1e3 * t / iters,
            "iterations_to_rule": n, "ms_per_solve_extrapolated": 1e3 * t / iters * n, "cores": 1,
            "note": "extrapolated: a bounded sample of iterations x the reference's own count to the rule"}


def run_reference(args):
    """The reference's Solver_CPU_RB on this host's cores, one full solve of one
    headline city per step (cycling through the batch's seeds), to the rule's
    iteration count. ms per domain = the mean of the timed solves."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    counts = ref_counts()
    threads = os.cpu_count() or 1
    seeds = [SEED0 + i for i in range(args.batch)]
    from oracle import city as OC

    t_build = time.time()
    for sd in seeds:  # untimed: the inputs of every step
        OC.random_city(WORKLOAD, sd)
    build_s = time.time() - t_build
    for k in range(args.warmup):
        reference_solves([seeds[k % len(seeds)]], threads, counts)
    t0 = time.time()
    timed = []
    for k in range(args.steps):
        timed += reference_solves([seeds[k % len(seeds)]], threads, counts)
    wall = time.time() - t0
    ms = [1e3 * t for _, t, _, _ in timed]
    value = float(np.mean(ms))
    serial = serial_solver_cpu_sample(seeds[0], counts)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{WORKLOAD} (256x256x64), held-out seeds {seeds[0]}..{seeds[-1]}",
                   "batch": args.batch, "tol": TOL, "itermax": ITERMAX, "window": WINDOW,
                   "window_tol": WINDOW_TOL, "solver": "Solver_CPU_RB (reference, OpenMP), one city per step"},
        "cpu_baseline": {"value": value, "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} full Solver_CPU_RB solves to the rule ("
                                   f"{', '.join(str(n) for _, _, n, _ in timed[:len(seeds)])} iterations), "
                                   f"one per step, {threads} threads, {cpu_model()}"},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_wall_s": wall, "input_build_s": build_s,
        "ms_per_solve": ms, "iterations": [n for _, _, n, _ in timed],
        "solver_cpu_serial": serial,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def fp64_checks(w, seed, st, lam, winds, ref_div=None):
    """The headline pipeline's FP32 result on one city against an FP64 run of
    the same SOR (same phases, same iteration counts, oracle restatement in
    double), and its FP64 final divergence beside the reference solver's."""
    from oracle import oracle as O

    d = w.domain
    t0 = time.time()
    phases = [(PRE_OMEGA, -1.0, st["pre_iterations"])] if st["pre_iterations"] else None
    u64, v64, w64, L64, _, _ = O.solve_f64(d, w, -1.0, st["iterations"], phases=phases)
    t_f64 = time.time() - t0
    lam_err = float(np.abs(lam.astype(np.float64) - L64).max() / max(np.abs(L64).max(), 1e-30))
    wind_err = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(winds, (u64, v64, w64)))
    out = {"seed": seed, "pre_iterations": st["pre_iterations"], "iterations": st["iterations"],
           "lambda_max_rel_err_vs_fp64": lam_err, "wind_max_err_vs_fp64_m_s": wind_err,
           "max_divergence_fp64": st["max_divergence"], "fp64_run_s": t_f64}
    if ref_div is not None:
        out["reference_max_divergence"] = ref_div
        out["reference"] = "Solver_CPU_RB to the rule on the same city (its own iteration count)"
    return out


def precision_device(s, outs, use_net, use_pre, net=None, omega=PRE_OMEGA):
    """One solve of the handle's domain with the arm's start, to the rule, then
    the same SOR in FP64 on the device from the same start with its iteration
    counts (qesb_fp64_same_sor): the FP32 result's lambda and wind errors."""
    import torch

    s.set_prephase(omega if use_pre else 0.0, PRE_TOL, ITERMAX)
    s.set_prephase_start(*start_stage(use_net, use_pre))
    if use_net:
        net.warm_start(s)
        lam0 = s.lambda_
    else:
        s.resetLambda()
        lam0 = None
    ptrs = [o.data_ptr() for o in outs]
    st = s.solve_device(ITERMAX, *ptrs)
    torch.cuda.synchronize()
    rep = s.fp64_same_sor(omega if use_pre else 0.0, st["pre_iterations"], st["iterations"], *ptrs, lambda0=lam0)
    return st, {"pre_iterations": st["pre_iterations"], "iterations": st["iterations"],
                "stop": st["converged"], "lambda_max_rel_err_vs_fp64": rep["lambda_max_rel_err"],
                "wind_max_err_vs_fp64_m_s": rep["wind_max_err"], "max_divergence_fp64": st["max_divergence"],
                "fp64_run_ms": rep["ms"], "how": "qesb_fp64_same_sor: the same red-black SOR in FP64 on the "
                                                 "device, same start and iteration counts"}


def precision_city800():
    """The FP32 pipeline on one 800 x 800 x 128 city (150 buildings, seed 0)
    against an FP64 run of the same SOR (configuration 2's precision report)."""
    import torch

    import qesb

    w = make_city("city800", 0)
    nf = w.domain.numFaceCentered()
    outs = [torch.empty(nf, dtype=torch.float32, device="cuda") for _ in range(3)]
    with qesb.Solver_B200(w.domain, TOL) as s:
        s.set_inputs(w)
        s.set_window_rule(WINDOW, WINDOW_TOL)
        st, out = precision_device(s, outs, False, True, omega=qesb.prephase_omega(800, 800))
    out.update({"seed": 0, "grid": [800, 800, 128], "ms_solve": st["ms_total"],
                "pre_omega": qesb.prephase_omega(800, 800)})
    return out


def size_rates(peak, workloads=("city400", "city800")):
    """Sweep speed at the large single-city configurations: one autotuned
    solve of SIZE_ITERS iterations (tolerance -1, so every iteration runs)
    after a warm-up solve, per workload; the time is the solve's own sweep
    loop (CUDA events around it)."""
    import qesb

    out = {}
    for name in workloads:
        w, _ = qesb.random_city(name, 0)
        Nx, Ny, Nz = w.domain.base
        upd = (Nx - 2) * (Ny - 2) * (Nz - 1)
        with qesb.Solver_B200(w.domain, -1.0) as s:
            s.set_inputs(w)
            variant, _ = s.autotune()
            per = []
            for _ in range(3):
                s.resetLambda()
                st = s.solve(w, SIZE_ITERS, set_inputs=False)
                per.append((st["ms_sweeps"] if st["ms_sweeps"] > 0 else st["ms_sor"]) / st["iterations"])
        ms_it = statistics.median(per[1:])
        moved = MOVED_BYTES_PER_CELL_ITER * upd / (ms_it * 1e-3) / 1e9
        alg = ALG_BYTES_PER_CELL_ITER * upd / (ms_it * 1e-3) / 1e9
        out[name] = {"grid": [Nx, Ny, Nz], "updated_cells": upd, "variant": variant, "iterations": SIZE_ITERS,
                     "us_per_iteration": 1e3 * ms_it, "moved_gbs": moved, "moved_frac": moved / peak,
                     "algorithmic_36B_gbs": alg}
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
    inputs, every solve to the rule: warm (that behaviour), cold (resetLambda
    before every step), warm + over-relaxed pre-phase. Device time per solve
    (CUDA events) and iterations."""
    import torch

    import qesb

    steps = steps or args.fire_loop
    w, _ = qesb.random_city(args.workload, SEED0)
    d = w.domain
    seq = [fire_inflow(w, t) for t in range(1, steps + 1)]
    arms = {}
    with qesb.Solver_B200(d, TOL) as s:
        s.set_inputs(w)
        s.set_window_rule(WINDOW, WINDOW_TOL)
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


def peaks():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(p["hbm_gbs"]), "measured", float(p.get("bf16_tflops", 1590.0))
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback", 1590.0


def run_b200(args):
    import torch

    import qesb
    from qesb import shard
    from qesb import warmstart as ws

    rank, local, world = dist_env()
    dist = init_group(args, world, local)
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    B = args.batch
    seeds = shard.rank_seeds(SEED0, B, rank)  # each rank its own batch: weak scaling
    cities = [make_city(args.workload, sd) for sd in seeds]
    d0 = cities[0].domain
    Nx, Ny, Nz = d0.base
    updated = (Nx - 2) * (Ny - 2) * (Nz - 1)
    nf = d0.numFaceCentered()

    def new_solvers(strm):
        out = [qesb.Solver_B200(w.domain, TOL, device=dev) for w in cities]
        for s in out:
            s.set_stream(strm.cuda_stream)
            s.set_window_rule(WINDOW, WINDOW_TOL)
        return out

    solvers = new_solvers(stream)
    for s, w in zip(solvers, cities):
        s.set_inputs(w)
    # autotuners (untimed set-up, like a library's algorithm search): the sweep
    # shape for single solves of this grid, and the one for this batch's list
    variant, _ = solvers[0].autotune()
    batch_variant, _ = qesb.autotune_batch(solvers)
    wpath = args.weights or ws.DEFAULT_WEIGHTS
    net = ws.WarmStartNet.from_file(wpath, device=dev)  # the network alone (forward timing, FLOPs)
    cnet = ws.WarmNet(wpath, device=dev)  # the arms' starts: the C ABI, the batch's forward in one pass

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return shard.max_over_ranks(x, device=f"cuda:{dev}") if dist else x

    outs = [[torch.empty(nf, dtype=torch.float32, device=f"cuda:{dev}") for _ in range(3)] for _ in range(B)]
    uvw = [[o[q].data_ptr() for o in outs] for q in range(3)]
    # per batched start: R, input (2), apply per domain; convolutions and poolings once
    launches_per_net = 4 * B + (4 * net.nlev - 1) + (net.nlev - 1)

    def set_arm(sset, use_net, use_pre):
        for s in sset:
            s.set_prephase(PRE_OMEGA if use_pre else 0.0, PRE_TOL, ITERMAX)
            s.set_prephase_start(*start_stage(use_net, use_pre))

    def start_batch(sset, use_net, use_pre):
        # the arm's settings and start (the learned start, or lambda = 0) of a batch
        set_arm(sset, use_net, use_pre)
        if use_net:
            cnet.warm_start_batch(sset)
        else:
            for s in sset:
                s.resetLambda()

    def batch_step(use_net, use_pre, sset=None, ptrs=None, strm=None, started=False):
        # started: the batch's start is already in place (a pipeline prepared it)
        sset, ptrs, strm = sset or solvers, ptrs or uvw, strm or stream

        def step():
            if not started:
                start_batch(sset, use_net, use_pre)
            st = qesb.solve_batch(sset, ITERMAX, *ptrs)
            return st, (launches_per_net if use_net else 0) + 6 * B + st[0]["launches"]
        return step

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

    # converged fields of the first two domains (long over-relaxed runs, then the
    # reference omega, no stopping rule; untimed) to state each arm's wind error
    conv = []
    for s, o in list(zip(solvers, outs))[:2]:
        s.set_window_rule(0, 0.0)
        s.set_tolerance(-1.0)
        s.set_prephase(1.97, -1.0, 8000)
        s.resetLambda()
        s.solve_device(3000, o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr())
        conv.append([t.clone() for t in o])
        s.set_tolerance(TOL)
        s.set_window_rule(WINDOW, WINDOW_TOL)

    def wind_err():
        return max(float((o[q] - c[q]).abs().max()) for o, c in zip(outs, conv) for q in range(3))

    arms, arm_res = {}, {}
    for name, (use_net, use_pre) in ARMS.items():
        if name == HEADLINE:
            continue
        ms, res, _, _ = timed(batch_step(use_net, use_pre), max(1, args.steps // 2), 1)
        arm_res[name] = res
        arms[name] = {"ms_per_domain": max_over_ranks(ms) / B, "iterations": [x["iterations"] for x in res[-1]],
                      "pre_iterations": [x["pre_iterations"] for x in res[-1]], "wind_err_vs_converged": wind_err()}
    use_net, use_pre = ARMS[HEADLINE]
    head_step = batch_step(use_net, use_pre)
    ms_head, res_head, launches, clocks = timed(head_step, args.steps, args.warmup, clocks=True)
    ms_head = max_over_ranks(ms_head)
    arms[HEADLINE] = {"ms_per_domain": ms_head / B, "iterations": [x["iterations"] for x in res_head[-1]],
                      "pre_iterations": [x["pre_iterations"] for x in res_head[-1]],
                      "wind_err_vs_converged": wind_err()}
    ms_plain = arms["plain"]["ms_per_domain"] * B
    # precision of domain 0 under the headline arm: FP64 replay on the device,
    # and (rank 0, below) the oracle's FP64 restatement on the host as a cross-check
    st_first, prec_first = precision_device(solvers[0], outs[0], use_net, use_pre, cnet)
    lam_first = solvers[0].lambda_
    winds_first = [t.cpu().numpy() for t in outs[0]]

    # ---- end to end through the host API (the headline step) -----------------
    host_keep = [[pinned_copy(torch, a) for a in w.inputs()] for w in cities]  # tensors own the pinned memory
    host_in = [[arr for _, arr in ins] for ins in host_keep]
    host_out = [[torch.empty(nf, dtype=torch.float32, pin_memory=True) for _ in range(3)] for _ in range(B)]
    # icellflag, u0, v0, w0 (WINDSGeneralData.inputs() order): what qesb_set_inputs_flags takes
    FLAGS_ONLY = slice(6, 10)
    h2d_full = sum(a.nbytes for ins in host_in for a in ins)
    h2d = sum(a.nbytes for ins in host_in for a in ins[FLAGS_ONLY])
    d2h = 3 * 4 * nf * B

    def e2e_step():
        for s, ins in zip(solvers, host_in):
            qesb.check(qesb.lib().qesb_set_inputs(s._h, *[a.ctypes.data for a in ins]))
        st, n = head_step()
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
    stream2 = torch.cuda.Stream(device=dev)
    solvers2 = new_solvers(stream2)
    solvers2[0].set_option("batch_variant", batch_variant)
    sets, streams = [solvers, solvers2], [stream, stream2]
    outs2 = [[torch.empty(nf, dtype=torch.float32, device=f"cuda:{dev}") for _ in range(3)] for _ in range(B)]
    set_outs = [outs, outs2]
    set_uvw = [uvw, [[o[q].data_ptr() for o in outs2] for q in range(3)]]
    host_out2 = [[torch.empty(nf, dtype=torch.float32, pin_memory=True) for _ in range(3)] for _ in range(B)]
    set_host_out = [host_out, host_out2]
    steps_of_set = [batch_step(use_net, use_pre, sets[k], set_uvw[k], streams[k], started=True) for k in range(2)]

    def load(k, flags_only):
        # a batch's inputs, then its start: on the loading thread, while the other batch solves
        for s_, ins in zip(sets[k], host_in):
            if flags_only:  # the stair-step coefficients computed from the flags on the device
                qesb.check(qesb.lib().qesb_set_inputs_flags(s_._h, *[a.ctypes.data for a in ins[FLAGS_ONLY]]))
            else:
                qesb.check(qesb.lib().qesb_set_inputs(s_._h, *[a.ctypes.data for a in ins]))
        start_batch(sets[k], use_net, use_pre)

    def solve_read(k):
        st_, _ = steps_of_set[k]()
        with torch.cuda.stream(streams[k]):
            for o, ho in zip(set_outs[k], set_host_out[k]):
                for q in range(3):
                    ho[q].copy_(o[q], non_blocking=True)
        return st_

    def pipelined(nsteps, flags_only=True):
        load(0, flags_only)
        for i in range(nsteps):
            cur = i % 2
            failed = []

            def load_next(k=1 - cur):
                try:
                    load(k, flags_only)
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

    k_e2e = max(4, args.steps)  # a stream of batches: the first upload and the last read-back are not overlapped
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_pipeline(flags_only):
        pipelined(2, flags_only)  # warm-up
        barrier()
        torch.cuda.synchronize(dev)
        p0.record(stream)
        pipelined(k_e2e, flags_only)
        p1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(p0.elapsed_time(p1) / k_e2e)

    ms_e2e_full = timed_pipeline(False)  # the reference's full input arrays
    ms_e2e = timed_pipeline(True)
    last = (k_e2e - 1) % 2
    # the host copies are the device results, and both solver sets give the same winds
    e2e_ok = all(torch.equal(ho[q], o[q].cpu()) for ho, o in zip(set_host_out[last], set_outs[last]) for q in range(3))
    e2e_ok = e2e_ok and all(torch.equal(a[q], b[q]) for a, b in zip(set_outs[last], outs if last else outs2)
                            for q in range(3))
    for s2 in solvers2:
        s2.close()

    # ---- roofline of the dominant kernel: the red/black list sweep --------------
    # Every sweep launch of the timed headline steps (pre-phase and reference
    # loop, the window checks between them included), timed by CUDA events on
    # the launching stream around the loops (qesb_stats.ms_sweeps); the bytes
    # are those the split layout must move per updated cell and iteration.
    peak, peak_src, tpeak = peaks()
    sweep_ms = sum(r[0]["ms_sweeps"] for r in res_head)
    dom_iters = sum(x["iterations"] + x["pre_iterations"] for r in res_head for x in r)
    list_launches = sum(r[0]["launches"] for r in res_head)
    moved = MOVED_BYTES_PER_CELL_ITER * updated * dom_iters / (sweep_ms * 1e-3) / 1e9
    alg = ALG_BYTES_PER_CELL_ITER * updated * dom_iters / (sweep_ms * 1e-3) / 1e9
    traffic, prof_note = None, None
    prof = os.path.join(ROOT, "profiles", "sor_zm_batch_city256.json")
    if os.path.exists(prof):
        try:
            pj = json.load(open(prof))
            traffic = pj.get("dram_bytes_per_launch")
            prof_note = pj.get("launch")
        except ValueError:
            traffic = None
    roofline = {"bound": "hbm", "achieved": moved, "peak": peak, "unit": "GB/s", "frac": moved / peak,
                "traffic": traffic, "peak_source": peak_src,
                "kernel": "red/black list sweep (variant %d): every launch of the timed steps' sweep loops, CUDA "
                          "events on the launching stream around them" % batch_variant,
                "bytes_per_cell_iteration": MOVED_BYTES_PER_CELL_ITER,
                "moved_bytes_per_full_list_launch": MOVED_BYTES_PER_CELL_ITER * updated * B // 2,
                "traffic_launch": prof_note, "domain_iterations": dom_iters, "sweep_ms": sweep_ms,
                "launches": list_launches, "us_per_domain_iteration": 1e3 * sweep_ms / dom_iters,
                "algorithmic_36B_gbs": alg, "algorithmic_36B_frac": alg / peak,
                "sweep_share_of_step": sweep_ms / (ms_head * args.steps)}

    # ---- the sweep at the 400^2 x 100 and 800^2 x 128 configurations ------------
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
    # the batch's start as the headline runs it: R, inputs, one stacked forward, applies
    for _ in range(2):
        cnet.warm_start_batch(solvers)
    fwd[0].record(stream)
    for _ in range(nf_rep):
        cnet.warm_start_batch(solvers)
    fwd[1].record(stream)
    torch.cuda.synchronize(dev)
    ms_start_batch = fwd[0].elapsed_time(fwd[1]) / nf_rep / B

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

    for s in solvers:
        s.close()
    solvers = []

    # ---- the batched ensemble (64 uneven cities x 36 directions) -----------------
    ensemble = None
    if not args.no_ensemble:
        try:
            ensemble = ensemble_run(args, print_line=False, dist=dist, dev=dev)
        except Exception as ex:  # noqa: BLE001
            ensemble = {"unavailable": str(ex)[:200]}

    # ---- reference GPU solver, CPU baseline, FP64 checks (rank 0, N = 1) --------------
    ref_gpu = cpu = precision = None
    if rank == 0 and world == 1:
        torch.cuda.synchronize(dev)
        counts = None
        try:
            counts = ref_counts()
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "ms", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {ex}"}
        ref_div = None
        if counts and not args.no_cpu_baseline:
            try:
                threads = os.cpu_count() or 1
                runs = reference_solves(seeds[:2], threads, counts, keep_winds=True)
                from oracle import oracle as O

                rw, ru, rv, rww = runs[0][3]
                ref_div = O.max_divergence(rw.domain, rw.icellflag, ru, rv, rww)
                ms_c = [1e3 * t for _, t, _, _ in runs]
                cpu = {"value": float(np.mean(ms_c)), "unit": "ms", "cores": threads, "kind": "reference",
                       "sample": f"full Solver_CPU_RB solves of seeds {seeds[0]}, {seeds[1]} to the rule "
                                 f"({runs[0][2]}, {runs[1][2]} iterations), {threads} threads, {cpu_model()}; "
                                 f"ms per solve {', '.join('%.0f' % m for m in ms_c)}",
                       "solver_cpu_serial": serial_solver_cpu_sample(seeds[0], counts)}
            except Exception as ex:  # noqa: BLE001
                cpu = {"value": None, "unit": "ms", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {ex}"}
        if not args.no_reference_gpu and counts:
            try:
                from oracle import oracle as O

                if O.ref_gpu_available():
                    w = cities[0]
                    n_rb = counts[f"{WORKLOAD}:{seeds[0]}"]["Solver_CPU_RB"]["iterations"]
                    _, _, _, secs, iters = O.ref_solve_gpu(w.domain, w, -1.0, n_rb)
                    ref_gpu = {"ms": 1e3 * secs, "iterations": n_rb, "seed": seeds[0],
                               "solver": "Solver_GPU_GlobalMemory::solve (reference, wall clock incl. its "
                                         "allocations and copies), the rule's red-black iteration count"}
                else:
                    ref_gpu = {"unavailable": "oracle/_ref/libqesref_gpu.so not built"}
            except Exception as ex:  # noqa: BLE001
                ref_gpu = {"unavailable": str(ex)[:200]}
        if not args.no_fp64:
            precision = {"city256": dict(prec_first, seed=seeds[0])}
            try:
                if not use_net:
                    precision["city256"]["host_oracle_cross_check"] = fp64_checks(
                        cities[0], seeds[0], st_first, lam_first, winds_first, ref_div)
            except Exception as ex:  # noqa: BLE001
                precision["city256"]["host_oracle_cross_check"] = {"unavailable": str(ex)[:200]}
            try:
                precision["city800"] = precision_city800()
            except Exception as ex:  # noqa: BLE001
                precision["city800"] = {"unavailable": str(ex)[:200]}

    if rank == 0:
        value = ms_head / B
        ms_pre_arm = arms["prephase"]["ms_per_domain"]
        learned_note = (f"the learned start pays: {ms_pre_arm / value:.3f}x the pre-phase alone (arms.prephase)"
                        if value < ms_pre_arm else
                        f"the pre-phase alone (arms.prephase) is faster ({value / ms_pre_arm:.3f}x): the network's "
                        "start saves fewer pre-phase iterations than its forward pass costs")
        line = {
            "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_head, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.workload} ({Nx}x{Ny}x{Nz}), held-out seeds {seeds[0]}..{seeds[-1]} "
                                   f"(+{B} per rank)",
                       "batch": B, "tol": TOL, "itermax": ITERMAX, "window": WINDOW, "window_tol": WINDOW_TOL,
                       "headline_arm": HEADLINE, "network": os.path.basename(wpath),
                       "network_levels": net.nlev, "channels": list(net.CH),
                       "sweep_variant": variant, "batch_variant": batch_variant,
                       "parallelism": f"replicas x{world}",
                       "warm_start": f"the learned network's prediction (BF16 tcgen05 convolutions, half "
                                     f"resolution, the batch's inputs stacked in one forward pass), then the "
                                     f"pre-phase: {START_STAGE[1]} red-black sweeps at omega {START_STAGE[0]}, "
                                     f"then omega {PRE_OMEGA} to max|dlambda| <= {PRE_TOL}; then the reference "
                                     f"loop (omega 1.78) to the rule; arms holds plain SOR, the pre-phase alone "
                                     f"and the network alone",
                       "learned_start_note": learned_note,
                       "l2": "8 domains x ~40 MB packed sweep data + network buffers > L2 (126 MB) per step"},
            "arms": arms,
            "speedup_vs_plain": ms_plain / ms_head,
            "network_ms_per_domain": ms_fwd,
            "e2e": {"value": ms_e2e / B, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "matches_device_result": bool(e2e_ok),
                    "how": "public API from pinned host arrays: qesb_set_inputs_flags (icellflag, u0, v0, w0; the "
                           "stair-step wall coefficients, the reference's default mesh, computed from the flags on "
                           "the device), the batched learned start, qesb_solve_batch, winds read back to pinned "
                           "host memory; two solver sets: while one batch solves, a second host thread loads the "
                           "next batch's inputs and runs its learned start; device-timed over the steps",
                    "full_arrays_value": ms_e2e_full / B, "full_arrays_h2d_bytes_per_step": h2d_full,
                    "full_arrays_how": "the same with qesb_set_inputs and the reference's full input arrays "
                                       "(e, f, g, h, m, n, icellflag, u0, v0, w0)",
                    "serial_value": ms_e2e_serial / B,
                    "serial_how": "full arrays, load and solve one after the other"},
            "roofline": roofline,
            "sizes": sizes,
            "network": {"bound": "tensor", "ms_per_forward": ms_fwd, "flops_per_forward": flops,
                        "achieved_tflops": flops / (ms_fwd * 1e-3) / 1e12, "peak_tflops": tpeak,
                        "frac": flops / (ms_fwd * 1e-3) / 1e12 / tpeak,
                        "batched_start_ms_per_domain": ms_start_batch,
                        "batched_frac": flops / (ms_start_batch * 1e-3) / 1e12 / tpeak,
                        "batched_how": f"qesb_warm_start_batch over the {B} domains (R, inputs, one forward over "
                                       "the inputs stacked along z, applies), CUDA events, per domain"},
            "ensemble": ensemble,
            "wall_log_law": wall_log,
            "fire_loop": fire,
            "reference_gpu": ref_gpu,
            "precision": precision,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist:
        barrier()  # rank 0 ran the CPU sections alone: the ranks leave together
        dist.destroy_process_group()


def ensemble_run(args, print_line=True, dist=None, dev=0):
    """Batched ensemble: cities with Nx, Ny ~ U[64, 256] and Nz ~ U[32, 96]
    (dx = dy = 2 m, z stretched 1.03, building count scaled from the 400 x 400
    config's 60), each at 36 wind directions 10 degrees apart, 2304 solves for
    64 cities. Inputs are built on the device (qesb_city_build_device,
    reported as setup, not timed). Cities are packed into launch lists of
    uneven sizes (whole cities, up to --ensemble-list-cells cells a list), each
    list one qesb_solve_batch: over-relaxed pre-phase warm start, reference
    loop to the rule, correction; the list sweep's launch shape tuned once on
    the first list. solves/s = all solves / the sum of list times (CUDA
    events); the latency of a solve = device time from the start of its list's
    iterations (pre-phase included) to the poll that ended it."""
    import torch

    import qesb
    from qesb import shard

    rank, local, world = dist_env()
    rng = np.random.default_rng(20260907)
    nd, ndir = args.ensemble_domains, 36
    dims = [(int(a), int(b), int(c)) for a, b, c in zip(rng.integers(64, 257, nd), rng.integers(64, 257, nd),
                                                       rng.integers(32, 97, nd))]
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    mine = shard.rank_share(nd, world, rank)  # cities of this rank; none crosses ranks
    lists, cur, cur_cells = [], [], 0
    for d in mine:
        Nx, Ny, Nz = dims[d]
        cells = ndir * Nx * Ny * (Nz + 1)
        if cur and cur_cells + cells > args.ensemble_list_cells:
            lists.append(cur)
            cur, cur_cells = [], 0
        cur.append(d)
        cur_cells += cells
    if cur:
        lists.append(cur)
    lat, list_ms, iters, pre_iters, cells_total, shapes, setup_ms, list_sizes = [], [], [], [], 0, [], [], []
    batch_shape = None
    names = ("icellflag", "e", "f", "g", "h", "m", "n", "u0", "v0", "w0")
    for lst in lists:
        solvers, arrays, outs = [], [], []
        try:
            torch.cuda.synchronize(dev)
            t_set = time.perf_counter()
            for d in lst:
                Nx, Ny, Nz = dims[d]
                dom = qesb.Domain(Nx, Ny, Nz, 2.0, 2.0, 1.0, qesb.city_dz(Nz, 1.0, 1.03))
                nb = max(3, int(round(60 * Nx * Ny / 160000)))
                c = qesb.city_random(dom, 700000 + d, nb)
                om = qesb.prephase_omega(Nx, Ny)
                nc_, nf_ = dom.numCellCentered(), dom.numFaceCentered()
                for k in range(ndir):
                    a = {q: torch.empty(nc_ if q not in ("u0", "v0", "w0") else nf_,
                                        dtype=torch.int32 if q == "icellflag" else torch.float32,
                                        device=f"cuda:{dev}") for q in names}
                    torch.cuda.current_stream(dev).synchronize()
                    qesb.city_build_device(dom, c.buildings,
                                           qesb.Inflow(c.inflow.u_ref, c.inflow.z_ref, c.inflow.p, 10.0 * k),
                                           {q: v.data_ptr() for q, v in a.items()}, stream.cuda_stream)
                    s = qesb.Solver_B200(dom, TOL, device=dev)
                    s.set_stream(stream.cuda_stream)
                    s.set_window_rule(WINDOW, WINDOW_TOL)
                    s.set_inputs_device(*[a[q].data_ptr() for q in ("e", "f", "g", "h", "m", "n", "icellflag",
                                                                     "u0", "v0", "w0")])
                    s.set_prephase(om, PRE_TOL, ITERMAX)
                    solvers.append(s)
                    arrays.append(a)
                    outs.append([torch.empty(nf_, dtype=torch.float32, device=f"cuda:{dev}") for _ in range(3)])
                shapes.append((Nx, Ny, Nz))
                cells_total += ndir * Nx * Ny * (Nz + 1)
            torch.cuda.synchronize(dev)
            setup_ms.append(1e3 * (time.perf_counter() - t_set))
            if batch_shape is None:
                batch_shape, _ = qesb.autotune_batch(solvers)
            solvers[0].set_option("batch_variant", batch_shape)
            ptrs = [[o[q].data_ptr() for o in outs] for q in range(3)]
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = qesb.solve_batch(solvers, ITERMAX, *ptrs)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            list_ms.append(e0.elapsed_time(e1))
            list_sizes.append(len(solvers))
            lat += [x["ms_sor"] for x in st]
            iters += [x["iterations"] for x in st]
            pre_iters += [x["pre_iterations"] for x in st]
            assert all(x["converged"] for x in st)
        finally:
            for s in solvers:
                s.close()
            del arrays, outs
    dv = f"cuda:{dev}" if dist else None
    total_ms = shard.max_over_ranks(float(np.sum(list_ms)), device=dv)
    setup_total = shard.max_over_ranks(float(np.sum(setup_ms)), device=dv)
    lat = shard.gather_lists(lat)
    iters, pre_iters = shard.gather_lists(iters), shard.gather_lists(pre_iters)
    cells_total = int(sum(shard.gather_lists([cells_total])))
    list_sizes = shard.gather_lists(list_sizes)
    n = nd * ndir
    out = {
        "metric": "ensemble solves/s (cities of uneven size x 36 wind directions, batched)",
        "value": n / (total_ms * 1e-3), "unit": "solves/s", "n_gpus": world, "higher_is_better": True,
        "scaling": "strong", "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{nd} cities, Nx,Ny ~ U[64,256], Nz ~ U[32,96], x {ndir} directions",
                   "solves": n, "launch_lists": len(list_sizes), "solves_per_list": list_sizes,
                   "cells_per_list_cap": args.ensemble_list_cells, "tol": TOL,
                   "itermax": ITERMAX, "window": WINDOW, "window_tol": WINDOW_TOL,
                   "warm_start": "over-relaxed pre-phase, omega = 2 - 7.5/max(Nx, Ny) within [1.85, 1.97], "
                                 f"to {PRE_TOL}", "cells_total": cells_total, "batch_variant": batch_shape},
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "setup_ms_per_solve": setup_total / n,
        "setup": "inputs (flags, wall coefficients, winds) built on the device by qesb_city_build_device "
                 "and handed over with qesb_set_inputs_device; wall clock, not in value",
        "ms_total": total_ms, "iterations_mean": float(np.mean(iters)),
        "pre_iterations_mean": float(np.mean(pre_iters)),
    }
    if print_line and rank == 0:
        print(json.dumps(out), flush=True)
    return out


def run_ensemble(args):
    rank, local, world = dist_env()
    dist = init_group(args, world, local)
    ensemble_run(args, print_line=True, dist=dist, dev=local if world > 1 else 0)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


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
    with qesb.Solver_B200(w.domain, -1.0) as s:
        if args.variant >= 0:
            s.set_option("variant", args.variant)
        st = s.solve(w, args.profile_solve)
    print(json.dumps({"profile_solve": args.profile_solve, **st}))


def run_profile_batch(args):
    """The headline step (a batch of B cities, its arm, the rule) twice, for
    launch-list captures."""
    import torch

    import qesb
    from qesb import warmstart as ws

    use_net, use_pre = ARMS[HEADLINE]
    cities = [make_city(args.workload, SEED0 + i) for i in range(args.batch)]
    solvers = [qesb.Solver_B200(w.domain, TOL) for w in cities]
    net = ws.WarmNet(args.weights or ws.DEFAULT_WEIGHTS) if use_net else None
    try:
        for s, w in zip(solvers, cities):
            s.set_inputs(w)
            s.set_window_rule(WINDOW, WINDOW_TOL)
            s.set_prephase(PRE_OMEGA if use_pre else 0.0, PRE_TOL, ITERMAX)
            s.set_prephase_start(*start_stage(use_net, use_pre))
        if args.variant >= 0:
            solvers[0].set_option("variant", args.variant)
        nf = cities[0].domain.numFaceCentered()
        outs = [[torch.empty(nf, dtype=torch.float32, device="cuda:0") for _ in range(3)] for _ in cities]
        ptrs = [[o[q].data_ptr() for o in outs] for q in range(3)]
        for _ in range(2):
            if net:
                net.warm_start_batch(solvers)
            else:
                for s in solvers:
                    s.resetLambda()
            st = qesb.solve_batch(solvers, ITERMAX, *ptrs)
        torch.cuda.synchronize()
    finally:
        for s in solvers:
            s.close()
        if net:
            net.close()
    print(json.dumps({"profile_batch": args.batch, "iterations": [x["iterations"] for x in st],
                      "pre_iterations": [x["pre_iterations"] for x in st]}))


def run_forward_only(args):
    """Batched learned starts (qesb_warm_start_batch over the B cities of the
    headline batch, one forward pass each), for network captures."""
    import torch

    import qesb
    from qesb import warmstart as ws

    cities = [make_city(args.workload, SEED0 + i) for i in range(args.batch)]
    solvers = [qesb.Solver_B200(w.domain, TOL) for w in cities]
    qesb.check(qesb.lib().qesb_net_set_conv_path(args.conv_path))
    net = ws.WarmNet(args.weights or ws.DEFAULT_WEIGHTS, device=0)
    try:
        for s, w in zip(solvers, cities):
            s.set_inputs(w)
        for _ in range(args.forward_only):
            net.warm_start_batch(solvers)
        torch.cuda.synchronize()
    finally:
        net.close()
        for s in solvers:
            s.close()
    print(json.dumps({"forward_only": args.forward_only, "batch": args.batch}))


def main():
    args = parse()
    maybe_relaunch(args)
    if args.plan:
        run_plan(args)
    elif args.profile_solve:
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
