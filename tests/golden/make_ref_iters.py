"""Iterations the reference's own solvers need to reach the benchmark's
stopping rule on the benchmark workloads; written to tests/golden/ref_iters.json.

Stopping rule: the reference loop `while (iter < itermax && max_error > tol)`
with tol = 1e-3 (reachable in FP32; the reference's 1e-9 is not) and
itermax = 10000. Run where the reference build oracle/_ref exists:

    OMP_NUM_THREADS=1 python tests/golden/make_ref_iters.py [workload[:seed] ...]

Solver_CPU_RB runs single-threaded here: its max_error reset races between
OpenMP threads (Solver_CPU_RB.cpp:166) and can end the loop early.
The iteration count is recovered from the reference's own
"[Solver] Residual after N itertations" line (Solver_CPU.cpp:152).
"""
import json
import os
import re
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "qes-public_b200"))
sys.path.insert(0, ROOT)

import qesb  # noqa: E402
from oracle import oracle as O  # noqa: E402

TOL, ITERMAX = 1e-3, 10000


def run(workload, kind):
    name, _, seed = workload.partition(":")
    seed = int(seed or 0)
    w, c = qesb.random_city(name, seed) if name != "cuboid100" else (qesb.cuboid100(), None)
    d = w.domain
    fd = sys.stdout.fileno()
    saved = os.dup(fd)
    with tempfile.TemporaryFile(mode="w+") as tmp:
        sys.stdout.flush()
        os.dup2(tmp.fileno(), fd)
        try:
            _, _, _, _, secs = O.ref_solve(d, w, TOL, ITERMAX, kind=kind, want_lambda=False)
        finally:
            sys.stdout.flush()
            os.dup2(saved, fd)
            os.close(saved)
        tmp.seek(0)
        text = tmp.read()
    m = re.findall(r"Residual after (\d+) itertations: ([0-9.eE+-]+)", text)
    iters, resid = int(m[-1][0]), float(m[-1][1])
    return {"iterations": iters, "residual": resid, "seconds": secs,
            "ms_per_iteration_1thread": 1e3 * secs / iters}


def main():
    os.environ["OMP_NUM_THREADS"] = "1"
    path = os.path.join(HERE, "ref_iters.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for wl in sys.argv[1:] or ["cuboid100", "city400"]:
        for kind, name in ((1, "Solver_CPU_RB"), (0, "Solver_CPU")):
            r = run(wl, kind)
            out.setdefault(wl, {"tol": TOL, "itermax": ITERMAX})[name] = r
            print(wl, name, r, flush=True)
            json.dump(out, open(path, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
