"""Train and evaluate the learned warm start.

    python qes-public_b200/train_warmstart.py --out DIR [--train 2000] [--eval 200] [--epochs 3]

Training data: seeded 128 x 128 x 64 synthetic cities (20-40 buildings,
stretched z, power-law inflow); the target of each is the lambda this solver
reaches after --target-iters red-black iterations from lambda = 0. Evaluation:
held-out 256 x 256 x 64 cities (seeds disjoint from training), each solved to
the benchmark's stopping rule (max|dlambda| <= 1e-3, FP64) from lambda = 0 and
from the network's prediction; reports iterations, device ms (network
included) and the largest wind difference between the two results.
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
TOL = 1e-3


def generate(net, n, workload, target_iters, threads=8):
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


def evaluate(net, n, workload, itermax=10000):
    torch = net.torch
    rows = []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    solver = None
    for k in range(n):
        w, _ = qesb.random_city(workload, EVAL_SEED0 + k)
        if solver is None:
            solver = qesb.Solver_B200(w.domain, TOL)
        solver.set_inputs(w)
        solver.resetLambda()
        torch.cuda.synchronize()
        ev[0].record()
        plain = solver.solve(w, itermax, set_inputs=False)
        ev[1].record()
        up = (w.u.copy(), w.v.copy(), w.w.copy())
        solver.resetLambda()
        torch.cuda.synchronize()
        ev[2].record()
        net.warm_start(solver)
        warm = solver.solve(w, itermax, set_inputs=False)
        ev[3].record()
        torch.cuda.synchronize()
        dw = max(float(np.abs(a - b).max()) for a, b in zip((w.u, w.v, w.w), up))
        rows.append({"seed": EVAL_SEED0 + k, "plain_iters": plain["iterations"], "warm_iters": warm["iterations"],
                     "plain_ms": ev[0].elapsed_time(ev[1]), "warm_ms": ev[2].elapsed_time(ev[3]),
                     "max_dwind": dw})
    solver.close()
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--eval", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--lr", type=float, default=1e-3)
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
    channels = tuple(min(128, 16 << l) for l in range(args.levels))
    net = ws.WarmStartNet(device=0, seed=args.seed, channels=channels, res=args.res)
    t0 = time.time()
    X, T, weight, s = generate(net, args.train, args.train_workload, args.target_iters)
    t_gen = time.time() - t0
    losses, t_train = train(net, X, T, weight, s, args.epochs, args.lr, coarse=((8, args.coarse_beta),))
    del X, T
    wpath = os.path.join(args.out, "warmstart_city.qwn")
    net.save(wpath)
    rows = evaluate(net, args.eval, args.eval_workload)
    it_p = np.array([r["plain_iters"] for r in rows], float)
    it_w = np.array([r["warm_iters"] for r in rows], float)
    ms_p = np.array([r["plain_ms"] for r in rows], float)
    ms_w = np.array([r["warm_ms"] for r in rows], float)
    report = {
        "train": {"n": args.train, "workload": args.train_workload, "epochs": args.epochs, "target_iters":
                  args.target_iters, "coarse_beta": args.coarse_beta, "generate_s": t_gen, "train_s": t_train,
                  "losses": losses},
        "eval": {"n": args.eval, "workload": args.eval_workload, "tol": TOL,
                 "plain_iters_mean": it_p.mean(), "warm_iters_mean": it_w.mean(),
                 "iters_ratio_mean": float((it_p / it_w).mean()),
                 "plain_ms_mean": ms_p.mean(), "warm_ms_mean": ms_w.mean(),
                 "ms_ratio_mean": float((ms_p / ms_w).mean()),
                 "max_dwind": max(r["max_dwind"] for r in rows), "rows": rows},
    }
    json.dump(report, open(os.path.join(args.out, "warmstart_report.json"), "w"), indent=1)
    e = report["eval"]
    print(json.dumps({k: v for k, v in e.items() if k != "rows"}))


if __name__ == "__main__":
    main()
