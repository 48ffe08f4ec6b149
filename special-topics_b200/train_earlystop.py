"""Trains and evaluates the learned early stop on the inverted-F variant family.

  python special-topics_b200/train_earlystop.py --out DIR [--train 4096] [--test 512] [--epochs 200]

1. Transients: the batched FP32 solver runs every training variant
   (seeds 1000..) for all LABEL_END = 7000 steps; the port V/I traces are
   kept.  (FP32 problems hold the x = max wall at zero, so the runs do not
   develop the reference's late-time growth.)
2. Labels: the run's two slowest-decaying resonances in 1-4 GHz, from a
   matrix pencil of order 12 over [n_in, 7000) of its own traces
   (earlystop.mode_label); inputs: the first n_in steps, 4x decimated and
   scaled (earlystop.inputs_from_traces, the same values the device input
   builder produces).
3. Training: the CUDA network (fdtd_es_train, Adam, BF16 weights) on those
   pairs, in stages of decreasing learning rate.
4. Evaluation on held-out seeds (10000..): plain FP64 batched runs of the full
   step count give the reference S11 (301 points, 1-4 GHz) and the plain
   time-to-S11.  FP32 runs stopped by StopPolicy.refined(): "learned" starts
   the refined candidate from the network's modes, "no_network" starts it
   from the run's own pencil (the same rule without the network), and
   "pencil_rule" is the pencils' agreement alone (the safe rule without the
   network); plain FP32 full-length runs are reported for context.  Reported: the share of runs
   within 0.1 dB (max over the 301 points), time-to-S11 of each method, steps
   run.

Writes DIR/es_weights.npz (EsNet.save: parameters, architecture, target
scaling) and DIR/es_metrics.json.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np


def _package():
    name = "special_topics_b200"
    if name in sys.modules:
        return sys.modules[name]
    d = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location(name, os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


def _label(args):
    V, I, n0, n1, dt = args
    _package()
    from special_topics_b200 import earlystop as ES
    return ES.mode_label(V, I, n0, n1, dt)


# labels come from the whole run: the FP32 runs hold the x = max wall at zero
# (fdtd_ctx_set_x_wall), so they do not develop the reference's late growth
LABEL_END = 7000
_T0 = time.perf_counter()


def log(msg: str) -> None:
    print(f"[{time.perf_counter() - _T0:8.1f} s] {msg}", flush=True)


def build_set(ES, pool, seeds, steps, policy, tiling):
    probs = ES.variant_problems(seeds, steps, pool)
    log(f"{len(probs)} training problems built")
    V, I, dev_s = ES.run_variants(probs, LABEL_END, "f32-table", tiling=tiling, progress=log)
    log(f"training transients done ({dev_s:.1f} device s)")
    dts = [p.grid.dt for p in probs]
    labels = pool.map(_label, [(V[q], I[q], policy.n_in, LABEL_END, dts[q]) for q in range(len(seeds))])
    log(f"{sum(t is not None for t in labels)} labels")
    x, y, keep = [], [], []
    for q, t in enumerate(labels):
        if t is None:
            continue
        xi, _ = ES.inputs_from_traces(V[q], I[q], ES.ARCH["in_length"], policy.decim)
        x.append(xi)
        y.append(t)
        keep.append(q)
    return np.array(x, np.float32), np.array(y, np.float32), keep, dev_s


def plain_reference(ES, pool, seeds, policy, tiling, group=128):
    """S11 of plain FP64 batched runs of the full step count, and their wall
    time (problem construction excluded).  The FP64 engines build their
    per-cell coefficients on the device from the material grids."""
    from special_topics_b200.backend import Batch, Engine
    freqs = ES.S11_FREQS
    seeds = list(seeds)
    ref, t_plain = [], 0.0
    for g0 in range(0, len(seeds), group):
        probs = ES.variant_problems(seeds[g0:g0 + group], policy.n_total, pool)
        engs = [Engine(p, "f64") for p in probs]
        try:
            t0 = time.perf_counter()
            with Batch(engs) as b:
                if tiling:   # shared-memory stages (prefetch 3, 4) are a material-table form
                    b.set_shape(dict(tiling, prefetch=min(tiling.get("prefetch", 1), 2)))
                b.run(policy.n_total)
            for e in engs:
                ref.append(ES.s11_db(e.voltages()[0], e.currents()[0], e.problem.grid.dt, freqs))
            t_plain += time.perf_counter() - t0
        finally:
            for e in engs:
                e.close()
        del probs, engs
        log(f"plain FP64 reference: {min(g0 + group, len(seeds))} of {len(seeds)} runs")
    return np.array(ref), t_plain


def evaluate_plain(ES, probs, ref, tiling, traces_out, group=128):
    """Plain FP32 runs of the full step count; their traces, dt and the FP64
    reference S11 go to traces_out for replaying stop rules offline."""
    from special_topics_b200.backend import Batch, Engine
    V32, I32, dts = [], [], []
    for g0 in range(0, len(probs), group):
        engs = [Engine(p, "f32-table") for p in probs[g0:g0 + group]]
        try:
            with Batch(engs) as b:
                if tiling:
                    b.set_shape(tiling)
                b.run(engs[0].problem.grid.numberOfTimeSteps)
            for e in engs:
                V32.append(e.voltages()[0].astype(np.float32))
                I32.append(e.currents()[0].astype(np.float32))
                dts.append(e.problem.grid.dt)
        finally:
            for e in engs:
                e.close()
    np.savez_compressed(traces_out, V=np.array(V32), I=np.array(I32), dt=np.array(dts), ref=ref)


def evaluate(ES, probs, ref, t_plain, net, policy, tiling, group=128, traces_out=None,
             methods=("learned", "no_network", "pencil_rule"), plain_f32=True, subsets=None):
    """Plain FP64 reference vs the early-stopped FP32 runs (with and without
    the network) and, with plain_f32, plain FP32 runs of the full step count.
    subsets: {name: run indices} reported separately for every method."""
    from special_topics_b200.backend import Batch, Engine
    freqs = ES.S11_FREQS
    out = {"plain_f64": {"time_s": t_plain, "steps": policy.n_total * len(probs)}}
    rules = {"learned": (True, policy), "no_network": (False, policy),
             "pencil_rule": (False, ES.StopPolicy.refined(vp=False))}
    for name in methods:
        use_net, pol = rules[name]
        errs, stops, winners, t = [], [], [], 0.0
        for g0 in range(0, len(probs), group):
            engs = [Engine(p, "f32-table") for p in probs[g0:g0 + group]]
            try:
                t0 = time.perf_counter()
                res = ES.run_with_early_stop(engs, net, pol, tiling, use_network=use_net)
                s11 = [ES.s11_db(r["V"], r["I"], e.problem.grid.dt, freqs) for r, e in zip(res, engs)]
                t += time.perf_counter() - t0
                log(f"{name}: {g0 + len(engs)} of {len(probs)} runs")
            finally:
                for e in engs:
                    e.close()
            for q, r in enumerate(res):
                errs.append(float(np.abs(s11[q] - ref[g0 + q]).max()))
                stops.append(r["stopped_at"])
                winners.append(r["winner"])
        errs = np.array(errs)
        out[name] = {"time_s": t, "steps": int(np.sum(stops)), "mean_stop_step": float(np.mean(stops)),
                     "within_0p1_dB": float(np.mean(errs <= 0.1)), "max_err_dB_median": float(np.median(errs)),
                     "max_err_dB_p90": float(np.percentile(errs, 90)), "max_err_dB_worst": float(errs.max()),
                     "stops": {str(c): int(np.sum(np.array(stops) == c)) for c in sorted(set(stops))},
                     "winners": {w: winners.count(w) for w in set(winners)}}
        for sub, idx in (subsets or {}).items():
            e, st = errs[idx], np.array(stops)[idx]
            out[name][sub] = {"runs": len(idx), "within_0p1_dB": float(np.mean(e <= 0.1)),
                              "max_err_dB_worst": float(e.max()), "mean_stop_step": float(st.mean())}
    if not plain_f32:
        out["runs"] = len(probs)
        if "learned" in out:
            out["time_to_s11_ratio_plain_over_learned"] = out["plain_f64"]["time_s"] / out["learned"]["time_s"]
        return out
    # plain FP32 runs of the full step count, for context (no early stop); their
    # traces (saved to traces_out) let other stop rules be replayed offline
    errs, t = [], 0.0
    V32, I32, dts = [], [], []
    for g0 in range(0, len(probs), group):
        engs = [Engine(p, "f32-table") for p in probs[g0:g0 + group]]
        try:
            t0 = time.perf_counter()
            with Batch(engs) as b:
                if tiling:
                    b.set_shape(tiling)
                b.run(policy.n_total)
            s11 = [ES.s11_db(e.voltages()[0], e.currents()[0], e.problem.grid.dt, freqs) for e in engs]
            t += time.perf_counter() - t0
            for e in engs:
                V32.append(e.voltages()[0])
                I32.append(e.currents()[0])
                dts.append(e.problem.grid.dt)
        finally:
            for e in engs:
                e.close()
        errs += [float(np.abs(s11[q] - ref[g0 + q]).max()) for q in range(len(s11))]
    if traces_out:
        np.savez(traces_out, V=np.array(V32), I=np.array(I32), dt=np.array(dts), ref=ref)
    errs = np.array(errs)
    out["plain_f32"] = {"time_s": t, "within_0p1_dB": float(np.mean(errs <= 0.1)),
                        "max_err_dB_median": float(np.median(errs)), "max_err_dB_worst": float(errs.max())}
    for name in methods:
        out[f"time_to_s11_ratio_plain_over_{name}"] = out["plain_f64"]["time_s"] / out[name]["time_s"]
    out["runs"] = len(probs)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--test", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--max-resid", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cache", default=None, help="npz of a previous run's training set and test reference")
    ap.add_argument("--save-test-traces", action="store_true",
                    help="also write the held-out runs' FP32 traces (es_test_traces.npz, about 110 KB per run) "
                         "for replaying stop rules offline")
    ap.add_argument("--no-eval", action="store_true", help="train and save only")
    ap.add_argument("--eval-only", default=None, metavar="WEIGHTS",
                    help="no training: evaluate these weights on the held-out seeds (learned rule and the "
                         "pencil rule against plain FP64), the tuned and untouched halves reported apart")
    ap.add_argument("--shape", default="16,4,1,0,0",
                    help="batch launch shape chunk,rows,prefetch,group,streams[,width] (backend.Batch.set_tiling); "
                         "64,16,1,0,0,16 is the batch tuner's shape for the variants")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    # one BLAS thread per pool worker (inherited by the spawned processes)
    for v in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    # workers register the package under its import name before any task arrives
    pool = mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1), initializer=_package)
    _package()
    from special_topics_b200 import earlystop as ES
    policy = ES.StopPolicy.refined(max_resid=args.max_resid)
    tiling = dict(zip(("chunk", "rows", "prefetch", "group", "streams", "width"),
                      (int(v) for v in args.shape.split(","))))
    metrics = {"policy": policy.__dict__, "arch": ES.ARCH}
    t0 = time.perf_counter()
    test_seeds = range(10000, 10000 + args.test)
    test_probs = ES.variant_problems(test_seeds, policy.n_total, pool)
    log(f"{len(test_probs)} test problems built")
    if args.eval_only:
        ref, t_plain = plain_reference(ES, pool, test_seeds, policy, tiling)
        log("plain FP64 reference done")
        pool.close()
        net = ES.EsNet.load(args.eval_only, max_batch=128)
        ES.start_fit_pool()
        # the stop rule's thresholds were chosen on seeds 10000..10255
        seeds = np.array(list(test_seeds))
        subsets = {"seeds_10000_10255": np.flatnonzero(seeds < 10256).tolist(),
                   "seeds_10256_up": np.flatnonzero(seeds >= 10256).tolist()}
        metrics["weights"] = os.path.basename(args.eval_only)
        metrics["evaluation"] = evaluate(ES, test_probs, ref, t_plain, net, policy, tiling,
                                         methods=("learned", "pencil_rule"), plain_f32=False, subsets=subsets)
        ES.stop_fit_pool()
        net.close()
        with open(os.path.join(args.out, "es_eval_metrics.json"), "w") as f:
            json.dump(metrics, f, indent=1)
        print(json.dumps(metrics["evaluation"]), flush=True)
        return
    if args.cache and os.path.exists(args.cache):
        z = np.load(args.cache)
        x, y, ref, t_plain = z["x"], z["y"], z["ref"], float(z["t_plain"])
        metrics["train_set"] = {"runs": args.train, "labelled": len(x), "from_cache": True}
    else:
        x, y, keep, dev_s = build_set(ES, pool, range(1000, 1000 + args.train), policy.n_total, policy, tiling)
        metrics["train_set"] = {"runs": args.train, "labelled": len(keep), "solver_device_s": dev_s,
                                "wall_s": time.perf_counter() - t0}
        np.savez(os.path.join(args.out, "es_train_set.npz"), x=x, y=y)
        ref, t_plain = plain_reference(ES, pool, test_seeds, policy, tiling)
        np.savez(os.path.join(args.out, "es_data.npz"), x=x, y=y, ref=ref, t_plain=t_plain)
    # target scaling: each output standardised over the training set
    mu, sd = y.mean(axis=0), y.std(axis=0) + 1e-6
    yn = (y - mu) / sd
    n_val = max(1, len(x) // 16)
    xv, yv = x[:n_val], yn[:n_val]
    net = ES.EsNet(out_dim=y.shape[1], max_batch=512)
    net.init(args.seed)
    losses = []
    t0 = time.perf_counter()
    w = np.ones(y.shape[1], np.float32)
    for stage, lr in enumerate((1e-3, 3e-4, 1e-4)):
        ep = args.epochs // 3
        losses += net.train(x[n_val:], yn[n_val:], epochs=ep, batch=args.batch, w=w, lr=lr, weight_decay=1e-4,
                            seed=args.seed + stage).tolist()
    metrics["training"] = {"wall_s": time.perf_counter() - t0, "epochs": len(losses), "first_loss": losses[0],
                           "last_loss": losses[-1], "val_loss": net.loss_grad(xv, yv, w, grad=False)[0]}
    pv = net.forward(xv) * sd + mu
    fr = np.abs(pv[:, 0::2] - y[:n_val, 0::2]) * ES.F_SCALE / (y[:n_val, 0::2] * ES.F_SCALE + ES.F_CENTER)
    metrics["val_pole_err"] = {"f_rel_median_per_slot": np.median(fr, axis=0).tolist(),
                               "alpha_rel_median_per_slot": np.median(np.abs(np.exp(pv[:, 1::2] - y[:n_val, 1::2]) - 1),
                                                                      axis=0).tolist()}
    net.out_mu, net.out_sd = mu.astype(np.float32), sd.astype(np.float32)
    net.save(os.path.join(args.out, "es_weights.npz"))
    log(f"trained: {metrics['training']}")
    with open(os.path.join(args.out, "es_metrics.json"), "w") as f:
        json.dump(metrics, f, indent=1)
    if args.no_eval:
        if args.save_test_traces:
            evaluate_plain(ES, test_probs, ref, tiling, os.path.join(args.out, "es_test_traces.npz"))
        pool.close()
        net.close()
        return
    metrics["evaluation"] = evaluate(ES, test_probs, ref, t_plain, net, policy, tiling,
                                     traces_out=os.path.join(args.out, "es_test_traces.npz")
                                     if args.save_test_traces else None)
    with open(os.path.join(args.out, "es_metrics.json"), "w") as f:
        json.dump(metrics, f, indent=1)
    print(json.dumps(metrics["evaluation"]), flush=True)
    pool.close()
    net.close()


if __name__ == "__main__":
    main()
