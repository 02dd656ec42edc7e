"""Train and evaluate the learned warm start.

    python qes-public_b200/train_warmstart.py --out DIR [--train 2000] [--eval 200] [--epochs 3]

Training data: seeded 128 x 128 x 64 synthetic cities (20-40 buildings,
stretched z, power-law inflow); the target of each is the converged lambda
(--target converged: an over-relaxed run of --target-iters red-black
iterations, then 1000 at the reference's omega) or the lambda after
--target-iters iterations from lambda = 0 (--target iters). Evaluation:
held-out 256 x 256 x 64 cities (seeds 500000 + i, disjoint from training),
each solved to the benchmark's stopping rule (the reference's tol 1e-9 and
itermax 10000, plus the window rule: 32 iterations, 4e-3) in four arms: plain
SOR from lambda = 0, the network's start, the over-relaxed pre-phase, the
network's start then the pre-phase (beginning with START_STAGE's sweeps at
a smaller omega); reports each arm's iterations and device
ms (network included), and its largest wind difference from the converged
field. --eval-only WEIGHTS evaluates a trained network without training.
Writes DIR/warmstart_city.qwn (weights, the library format qesb_warmnet_load reads) and
DIR/warmstart_report.json.
"""
import argparse
import json
import math
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import qesb  # noqa: E402
from qesb import warmstart as ws  # noqa: E402

TRAIN_SEED0, EVAL_SEED0 = 1000, 500000
TOL, ITERMAX, WINDOW, WINDOW_TOL = 1e-9, 10000, 32, 4e-3
PRE_OMEGA, PRE_TOL = 1.97, 2e-3
START_STAGE = (1.8, 8)  # the pre-phase's first sweeps after the network's start (the benchmark's setting)


def converge(solver, w, omega, pre_iters, ref_iters=1000):
    """lambda converged to the FP32 noise floor: pre_iters over-relaxed
    red-black iterations, then ref_iters at the reference's omega, no stopping
    rule (the handle's rule settings are restored)."""
    solver.set_tolerance(-1.0)
    solver.set_window_rule(0, 0.0)
    solver.set_prephase(omega, -1.0, pre_iters)
    solver.resetLambda()
    solver.solve(w, ref_iters, set_inputs=False)
    solver.set_prephase(0.0, 0.0, 0)
    solver.set_tolerance(TOL)


def generate(net, n, workload, target_iters, threads=8, target="converged"):
    """Compact inputs [n][V][5] (BF16) and targets [n][V] (FP32) on the device."""
    torch = net.torch
    pool = ThreadPoolExecutor(max_workers=threads)
    make = lambda k: qesb.random_city(workload, TRAIN_SEED0 + k)[0]  # noqa: E731
    ahead = [pool.submit(make, k) for k in range(min(n, 2 * threads))]

    def cities():  # at most 2*threads cities in host memory at once
        for k in range(n):
            w = ahead[k].result()
            ahead[k] = None
            if k + 2 * threads < n:
                ahead.append(pool.submit(make, k + 2 * threads))
            yield w

    X = T = weight = None
    solver = None
    s = None
    scale = torch.zeros(1, dtype=torch.int32, device=net.dev)
    torch.cuda.synchronize()  # its zero fill is torch's work; the kernels that use it run on the solver's
    t0 = time.time()
    for k, w in enumerate(cities()):
        if solver is None:
            solver = qesb.Solver_B200(w.domain, 0.0)
            s = net.net_shapes(solver)
            f = ws.shapes_of(solver)
            V = s.V(0)
            X = torch.empty((n, V, 5), dtype=torch.bfloat16, device=net.dev)
            T = torch.empty((n, V), dtype=torch.float32, device=net.dev)
            weight = torch.empty(V, dtype=torch.float32, device=net.dev)
            if net.res == 2:  # full-resolution target and weight, averaged 2x2x2
                Tf = torch.empty(f.V(0), dtype=torch.float32, device=net.dev)
                Wf = torch.empty(f.V(0), dtype=torch.float32, device=net.dev)
            torch.cuda.synchronize()
        solver.set_inputs(w)
        if target == "converged":
            converge(solver, w, qesb.prephase_omega(f.W, f.H), target_iters)
        else:
            solver.resetLambda()
            solver.solve(w, target_iters, set_inputs=False)
        net.input_from(solver, s, scale)
        if net.res == 1:
            qesb.check(qesb.lib().qesb_warm_target(solver._h, T[k].data_ptr(), weight.data_ptr(), scale.data_ptr()))
        else:
            hs = solver.stream_ptr()
            qesb.check(qesb.lib().qesb_warm_target(solver._h, Tf.data_ptr(), Wf.data_ptr(), scale.data_ptr()))
            qesb.check(qesb.lib().qesb_net_pool2_f32(Tf.data_ptr(), T[k].data_ptr(), f.D, f.H, f.W, hs))
            qesb.check(qesb.lib().qesb_net_pool2_f32(Wf.data_ptr(), weight.data_ptr(), f.D, f.H, f.W, hs))
        torch.cuda.synchronize()  # the input and target kernels ran on the solver's stream
        xb = net._bufs(s)["x"].view(s.V(0), ws.IN_CH)
        X[k].copy_(xb[:, :5])
        if k % 200 == 0:
            torch.cuda.synchronize()
            print(f"  generated {k + 1}/{n} ({time.time() - t0:.1f} s)", flush=True)
    torch.cuda.synchronize()
    solver.close()
    pool.shutdown()
    return X, T, weight, s


def train(net, X, T, weight, s, epochs, lr0, log_every=200, coarse=((8, 0.0),)):
    torch = net.torch
    n = X.shape[0]
    V = s.V(0)
    inv = 1.0 / float(weight.sum())
    xb = net._bufs(s)["x"].view(V, ws.IN_CH)
    xb.zero_()
    total = epochs * n
    losses = []
    g = torch.Generator().manual_seed(0)
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        order = torch.randperm(n, generator=g).tolist()
        for i in order:
            lr = 1e-5 + 0.5 * (lr0 - 1e-5) * (1 + math.cos(math.pi * step / total))
            xb[:, :5].copy_(X[i])
            net.forward(s)
            net.backward(s, T[i], weight, inv, coarse=coarse)
            net.adam(lr)
            step += 1
            if step % log_every == 0 or step == total:
                loss = float(net.loss.item())
                losses.append((step, loss))
                print(f"  step {step}/{total} loss {loss:.5f} lr {lr:.2e} ({time.time() - t0:.1f} s)", flush=True)
    torch.cuda.synchronize()
    net.check_err()
    return losses, time.time() - t0


def evaluate(net, n, workload):
    """Four arms per held-out city under the benchmark's rule (see the module
    docstring); ms are device time (CUDA events) of the start and the solve."""
    torch = net.torch
    rows = []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    solver = None
    for k in range(n):
        w, _ = qesb.random_city(workload, EVAL_SEED0 + k)
        if solver is None:
            solver = qesb.Solver_B200(w.domain, TOL)
            solver.set_inputs(w)
            solver.autotune()
        solver.set_inputs(w)
        converge(solver, w, 1.97, 8000, 3000)
        uc = (w.u.copy(), w.v.copy(), w.w.copy())
        solver.set_window_rule(WINDOW, WINDOW_TOL)
        row = {"seed": EVAL_SEED0 + k}
        for arm, (use_net, use_pre) in {"plain": (0, 0), "network": (1, 0), "prephase": (0, 1),
                                        "network+prephase": (1, 1)}.items():
            solver.set_prephase(PRE_OMEGA if use_pre else 0.0, PRE_TOL, ITERMAX)
            solver.set_prephase_start(*(START_STAGE if use_net and use_pre else (0.0, 0)))
            solver.resetLambda()
            torch.cuda.synchronize()
            ev[0].record(torch.cuda.ExternalStream(solver.stream_ptr()))
            if use_net:
                net.warm_start(solver)
            st = solver.solve(w, ITERMAX, set_inputs=False)
            ev[1].record(torch.cuda.ExternalStream(solver.stream_ptr()))
            torch.cuda.synchronize()
            row[arm] = {"iterations": st["iterations"], "pre_iterations": st["pre_iterations"],
                        "ms": ev[0].elapsed_time(ev[1]), "stop": st["converged"],
                        "wind_err_vs_converged": max(float(np.abs(a - b).max()) for a, b in zip((w.u, w.v, w.w), uc))}
        rows.append(row)
        if k % 20 == 0:
            print(f"  evaluated {k + 1}/{n}: {row}", flush=True)
    solver.close()
    return rows


def summary(rows):
    out = {}
    for arm in ("plain", "network", "prephase", "network+prephase"):
        its = np.array([r[arm]["iterations"] + r[arm]["pre_iterations"] for r in rows], float)
        ms = np.array([r[arm]["ms"] for r in rows], float)
        out[arm] = {"iterations_mean": float(its.mean()), "ms_mean": float(ms.mean()),
                    "wind_err_max": max(r[arm]["wind_err_vs_converged"] for r in rows),
                    "all_stopped_by_rule": all(r[arm]["stop"] == 2 for r in rows)}
    p, pp = out["plain"]["ms_mean"], out["prephase"]["ms_mean"]
    for arm in out:
        out[arm]["speedup_vs_plain"] = p / out[arm]["ms_mean"]
        out[arm]["speedup_vs_prephase"] = pp / out[arm]["ms_mean"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--eval", type=int, default=200)
    ap.add_argument("--eval-only", default=None, help="evaluate this weights file, no training")
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--target", default="converged", choices=["converged", "iters"])
    ap.add_argument("--target-iters", type=int, default=4000)
    ap.add_argument("--train-workload", default="city128")
    ap.add_argument("--eval-workload", default="city256")
    ap.add_argument("--levels", type=int, default=4, help="encoder-decoder levels (channels 16, 32, 64, 128, 128, ...)")
    ap.add_argument("--seed", type=int, default=0, help="weight initialisation seed")
    ap.add_argument("--res", type=int, default=1, help="1: network at full resolution, 2: at half resolution")
    ap.add_argument("--coarse-beta", type=float, default=0.0,
                    help="weight of the 8x8x8-block error term of the loss (0: plain MSE)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    report = {}
    if args.eval_only:
        net = ws.WarmStartNet.from_file(args.eval_only, device=0)
        report["weights"] = os.path.basename(args.eval_only)
    else:
        channels = tuple(min(128, 16 << l) for l in range(args.levels))
        net = ws.WarmStartNet(device=0, seed=args.seed, channels=channels, res=args.res)
        t0 = time.time()
        X, T, weight, s = generate(net, args.train, args.train_workload, args.target_iters, target=args.target)
        t_gen = time.time() - t0
        losses, t_train = train(net, X, T, weight, s, args.epochs, args.lr, coarse=((8, args.coarse_beta),))
        del X, T
        net.save(os.path.join(args.out, "warmstart_city.qwn"))
        report["train"] = {"n": args.train, "workload": args.train_workload, "epochs": args.epochs,
                           "target": args.target, "target_iters": args.target_iters, "res": args.res,
                           "coarse_beta": args.coarse_beta, "generate_s": t_gen, "train_s": t_train,
                           "losses": losses}
    rows = evaluate(net, args.eval, args.eval_workload)
    report["eval"] = {"n": args.eval, "workload": args.eval_workload, "seeds": [EVAL_SEED0, EVAL_SEED0 + args.eval - 1],
                      "rule": {"tol": TOL, "itermax": ITERMAX, "window": WINDOW, "window_tol": WINDOW_TOL},
                      "prephase": {"omega": PRE_OMEGA, "tol": PRE_TOL,
                                   "start_stage_after_network": list(START_STAGE)},
                      "summary": summary(rows), "rows": rows}
    json.dump(report, open(os.path.join(args.out, "warmstart_report.json"), "w"), indent=1)
    print(json.dumps(report["eval"]["summary"]))


if __name__ == "__main__":
    main()
