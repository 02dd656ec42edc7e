"""The reference's own iteration counts to the benchmark's stopping rule, and
its serial Solver_CPU winds there; written to tests/golden/ref_iters.json and
tests/golden/solver_cpu_city256_<seed>.npz.

Stopping rule (the same for every solver and every arm of the benchmark): the
reference loop `while (iter < itermax && max_error > tol)` with the
reference's own tol = 1e-9 (never met in FP32) and itermax = 10000, plus the
window rule: after every WINDOW-th iteration n the loop also ends when
max|lambda_n - lambda_(n - WINDOW)| <= WINDOW_TOL over all cells, in double.

The reference solvers have no window rule, so each is run WINDOW iterations
per Solver::solve call, lambda carried from call to call (bit-identical to
one long run: every call recomputes the same R and copies lambda to
lambda_old at the top of each iteration), and the drift is taken here between
calls. Cities come from oracle/city.py (no product code). Run where the
reference build oracle/_ref exists:

    python tests/golden/make_ref_iters.py [seed ...]   (default 500000..500007)

Each (seed, solver) runs in its own single-threaded process: Solver_CPU is
serial, and Solver_CPU_RB at one thread has no max_error reset race
(Solver_CPU_RB.cpp:166); the calls use tol < 0, so the loop runs exactly
WINDOW iterations either way. The fixture keeps the serial Solver_CPU winds
on every 4th face column in x and y (all layers) and the max divergence of
the full field; ref_iters.json holds every run's max divergence (FP64, fluid
cells, k <= nz-4, the solver's final check).
"""
import json
import os
import sys
import time
from multiprocessing import get_context

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

WORKLOAD = "city256"
TOL, ITERMAX = 1e-9, 10000
WINDOW, WINDOW_TOL = 32, 4e-3
FIXTURE_SEEDS = (500000, 500001)
STRIDE = 4


def run(args):
    seed, kind = args
    os.environ["OMP_NUM_THREADS"] = "1"
    from oracle import city as OC
    from oracle import oracle as O

    O.ref_set_threads(1)
    w = OC.random_city(WORKLOAD, seed)
    d = w.domain
    lam = np.zeros(d.numCellCentered(), np.float32)
    n, secs, drift = 0, 0.0, -1.0
    t0 = time.time()
    while n < ITERMAX:
        step = min(WINDOW, ITERMAX - n)
        (u, v, ww, nxt, t), _ = O.capture_stdout(lambda: O.ref_solve(d, w, -1.0, step, kind=kind, lam=lam))
        secs += t
        n += step
        if step == WINDOW:
            drift = float(np.abs(nxt.astype(np.float64) - lam.astype(np.float64)).max())
        lam = nxt
        if step == WINDOW and drift <= WINDOW_TOL:
            break
    out = {"iterations": n, "window_drift": drift, "solve_seconds_1thread": secs,
           "ms_per_iteration_1thread": 1e3 * secs / n, "wall_s": time.time() - t0,
           "max_div": O.max_divergence(d, w.icellflag, u, v, ww)}
    if kind == 0 and seed in FIXTURE_SEEDS:
        shape = (d.nz(), d.ny(), d.nx())
        sub = (slice(None), slice(None, None, STRIDE), slice(None, None, STRIDE))
        np.savez_compressed(os.path.join(HERE, f"solver_cpu_{WORKLOAD}_{seed}.npz"),
                            u=u.reshape(shape)[sub], v=v.reshape(shape)[sub], w=ww.reshape(shape)[sub],
                            stride=STRIDE, iterations=n, window=WINDOW, window_tol=WINDOW_TOL,
                            window_drift=drift, max_div=O.max_divergence(d, w.icellflag, u, v, ww))
    return seed, kind, out


def main():
    seeds = [int(s) for s in sys.argv[1:]] or list(range(500000, 500008))
    path = os.path.join(HERE, "ref_iters.json")
    res = {}
    jobs = [(s, k) for s in seeds for k in (0, 1)]
    with get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        for seed, kind, out in pool.imap_unordered(run, jobs):
            name = "Solver_CPU" if kind == 0 else "Solver_CPU_RB"
            res.setdefault(f"{WORKLOAD}:{seed}", {})[name] = out
            print(seed, name, out, flush=True)
    doc = {"rule": {"tol": TOL, "itermax": ITERMAX, "window": WINDOW, "window_tol": WINDOW_TOL},
           "cpu": os.popen("grep -m1 'model name' /proc/cpuinfo").read().split(":")[-1].strip(), **res}
    json.dump(doc, open(path, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
