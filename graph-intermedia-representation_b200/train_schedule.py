"""Trains the schedule network on traces this library generates itself.

For a suite of synthetic graphs (power-law R-MAT of several sizes and weight ranges, and
high-diameter lattices), the method sweeps its own choices and keeps the fastest:

  SSSP  the Delta-stepping bucket width, over the six candidate values, per graph, weight kind
        and lane count; the sample is the group's feature row (sssp features) with the class of
        the fastest Delta;
  BFS   the direction-switch thresholds (alpha, beta) over a grid; the samples are the
        per-level feature rows of the fastest setting's run with the direction it took;
  SCC   the forward-backward pivot rule (max out x in degree, max out + in, max in-degree, no
        forward-backward pass), per graph; the sample is the build's feature row with the class
        of the fastest rule.

The network (8 features -> 32 tanh -> 12 logits) is then trained on the GPU by this library's
own forward/backward/SGD kernels (gir_dev_sched_train), and its weights are written to
schedule_weights.npy beside this file, where DeviceGraph.use_learned_schedule() loads them.
Results never depend on the schedule: every choice gives bit-identical levels and distances.

  python graph-intermedia-representation_b200/train_schedule.py [--out FILE] [--quick]
"""
import argparse
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def timed(fn, reps=2):
    best = float("inf")
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t)
    return best


def suite(pkg, quick):
    G = pkg.graphs
    out = []
    r18 = G.rmat(18, seed=31, permute=True, weights=(1, 255), name="rmat_s18")
    out.append((r18, "hash"))
    out.append((r18, "stored"))
    r20 = G.rmat(20, seed=32, permute=True, weights=(1, 1023), name="rmat_s20_w1023")
    out.append((r20, "stored"))
    out.append((G.lattice(side=300, seed=41), "stored"))
    if not quick:
        lj = G.rmat_lj()
        out.append((lj, "hash"))
        out.append((lj, "stored"))
        out.append((G.lattice(side=800, seed=42), "stored"))
        out.append((G.lattice(side=1500, seed=43), "stored"))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "schedule_weights.npy"))
    ap.add_argument("--summary", default=None)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--lr", type=float, default=0.5)
    args = ap.parse_args()
    import torch
    pkg = importlib.import_module("graph-intermedia-representation_b200")
    native = pkg.native
    deltas = pkg.DeviceGraph.delta_choices()
    xs, ys, log = [], [], []
    for g, wk in suite(pkg, args.quick):
        d = pkg.DeviceGraph.from_graph(g)
        wm = native.WEIGHT_HASH if wk == "hash" else native.WEIGHT_STORED
        for lanes in (8, 64):
            src = torch.from_numpy(pkg.graphs.sources_with_edges(g, lanes, 5 + lanes)).to("cuda:0")
            out = torch.empty((lanes, g.V), dtype=torch.int64, device="cuda:0")
            times = []
            feat = None
            for k, D in enumerate(deltas):
                t = timed(lambda: d.sssp(src, delta=int(D), weights=wm, out=out), reps=1 if g.V > 2_000_000 else 2)
                times.append(t)
                if feat is None:
                    fx, _ = d.sched_trace()
                    feat = fx[0]
            best = int(np.argmin(times))
            log.append({"graph": g.name, "weights": wk, "lanes": lanes, "sssp_ms": [round(1e3 * t, 2) for t in times],
                        "best_delta": int(deltas[best])})
            rng = np.random.default_rng(len(log))
            for _ in range(40):  # one row per sweep, replicated with small noise to balance the BFS rows
                xs.append(feat * (1 + 0.01 * rng.standard_normal(feat.shape)).astype(np.float32))
                ys.append(2 + best)
            print(json.dumps(log[-1]), flush=True)
        if wk == "hash" or g.name.startswith("lattice"):
            # SCC build: the four pivot rules (same SCCs; only the time differs)
            times, feat = [], None
            for rule in range(4):
                d.set_param(native.PARAM_PIVOT, rule)
                d.build(native.LAYER_SCC)
                times.append(timed(lambda: d.build(native.LAYER_SCC)))
                if feat is None:
                    feat = d.sched_trace()[0][0]
            d.set_param(native.PARAM_PIVOT, -1)
            best = int(np.argmin(times))
            log.append({"graph": g.name, "scc_ms_by_pivot_rule": [round(1e3 * t, 2) for t in times], "best_rule": best})
            rng = np.random.default_rng(100 + len(log))
            for _ in range(40):
                xs.append(feat * (1 + 0.01 * rng.standard_normal(feat.shape)).astype(np.float32))
                ys.append(8 + best)
            print(json.dumps(log[-1]), flush=True)
            for lanes in (1, 8, 64):
                src = torch.from_numpy(pkg.graphs.sources_with_edges(g, lanes, 9 + lanes)).to("cuda:0")
                out = torch.empty((lanes, g.V), dtype=torch.int32, device="cuda:0")
                res = []
                for alpha in (2.0, 6.0, 15.0, 40.0, 150.0, 600.0):
                    for beta in (2.0, 6.0, 18.0, 80.0, 300.0):
                        d.set_param(native.PARAM_ALPHA, alpha)
                        d.set_param(native.PARAM_BETA, beta)
                        res.append((timed(lambda: d.bfs(src, out=out)), alpha, beta))
                t, alpha, beta = min(res)
                d.set_param(native.PARAM_ALPHA, alpha)
                d.set_param(native.PARAM_BETA, beta)
                d.bfs(src, out=out)
                fx, fy = d.sched_trace()
                xs.extend(fx)
                ys.extend(fy.tolist())
                fixed = [r[0] for r in res if r[1] == 15.0 and r[2] == 18.0][0]
                log.append({"graph": g.name, "lanes": lanes, "bfs_best": [alpha, beta], "bfs_ms": round(1e3 * t, 3),
                            "bfs_fixed_ms": round(1e3 * fixed, 3), "levels": len(fy)})
                print(json.dumps(log[-1]), flush=True)
                d.set_param(native.PARAM_ALPHA, 15.0)
                d.set_param(native.PARAM_BETA, 18.0)
        d.close()
    x = np.asarray(xs, np.float32)
    y = np.asarray(ys, np.int32)
    # train on the GPU with the library's own kernels
    g0 = pkg.graphs.rmat(8, seed=1, weights=None)
    d = pkg.DeviceGraph.from_graph(g0, weights=False)
    loss0 = d.sched_grad(x, y)[1]
    loss = d.sched_train(x, y, steps=args.steps, lr=args.lr)
    logits = d.sched_forward(x)
    pred = np.where(y < 2, np.argmax(logits[:, :2], 1),
                    np.where(y < 8, 2 + np.argmax(logits[:, 2:8], 1), 8 + np.argmax(logits[:, 8:], 1)))
    acc = float((pred == y).mean())
    w = d.sched_get_weights()
    d.close()
    np.save(args.out, w)
    summary = {"samples": int(len(y)), "loss_before": float(loss0), "loss_after": float(loss), "train_accuracy": acc,
               "sweeps": log, "out": args.out}
    print(json.dumps({k: v for k, v in summary.items() if k != "sweeps"}), flush=True)
    if args.summary:
        with open(args.summary, "w") as f:
            json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
