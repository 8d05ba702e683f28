"""Train the learned Steiner placement network on the GPU.

    python -m gpu_cdt_refine_b200.train_placement [--labels descendants|one-step]
        [--inputs N] [--points 200000] [--theta 20] [--epochs E]
        [--out gpu_cdt_refine_b200/data/placement_mlp.npy] [--eval 2]

Inputs are seeded instances of the clustered distribution (64 isotropic
Gaussians plus 10% uniform background, segments 5% of the points), seeds 1000,
1001, ...; every network is trained by the library's own forward/backward
kernels with Adam (gqm_mlp_train).  The placement network's target t = 0 (keep
the off-center) is encoded as -0.25, so that "keep" is learned as an output
below 0, where the placement rule falls back to the off-center.

Labels:

* ``descendants`` (default): exploration runs (gqm_learn_explore) insert every
  candidate's point at a level t drawn from {0, 1/32, ..., 1} (--levels) and record the
  parent tree of the inserted vertices; a row's label is its descendant count
  (inserted rows and midpoints below it, down to --depth generations).
  Regression networks (--ensemble of them, averaged) learn the expected count
  from the features with the inserted t in the free feature slot T_SLOT; each
  candidate's placement target is the level with the smallest predicted count,
  the off-center unless another level is predicted lower by more than
  --margin.  With --iterations > 1, later explorations follow the last network
  except for a fraction --eps of random levels.
* ``one-step``: plain refinements (gqm_learn_collect) label each candidate
  with the level, of nine, whose new triangles include the fewest below theta.

--eval N refines N held-out inputs (seeds 9100, ...) with the plain rule and
with the trained network and reports both vertex counts and certificates.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import inputs, refine

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "placement_mlp.npy")
T_SLOT = 25  # features_of leaves slots 25..30 zero; the regression network reads t here
LEVELS = 33  # default number of levels t = 0, 1/(L-1), ..., 1


def collect(n_inputs, points, theta, rows_per_input, seed0=1000, device=0):
    """One-step rows of n_inputs seeded inputs (at most rows_per_input of each,
    a seeded sample); inputs are built on host threads while the GPU refines."""
    from concurrent.futures import ThreadPoolExecutor
    feats, tgts = [], []
    rng = np.random.default_rng(seed0)
    with ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1))) as ex:
        futs = [ex.submit(inputs.clustered, seed0 + s, points, points // 20) for s in range(n_inputs)]
        for fut in futs:
            f, t = refine.learn_collect(fut.result(), theta, device=device, cap=8 * points)
            if f.shape[0] > rows_per_input:
                keep = np.sort(rng.choice(f.shape[0], rows_per_input, replace=False))
                f, t = f[keep], t[keep]
            feats.append(f)
            tgts.append(t)
    return np.concatenate(feats), np.concatenate(tgts)


def explore(n_inputs, points, theta, depth, seed0=1000, device=0, mlp=None, eps=1.0, levels=LEVELS):
    """Exploration rows of n_inputs seeded inputs: (features, t_used, descendant
    count) of every inserted candidate where the learned rule applies, plus
    run totals.  With a network, candidates take its t except for a fraction
    eps that draw a level."""
    from concurrent.futures import ThreadPoolExecutor
    X, T, D = [], [], []
    info = {"rows": 0, "inserted": 0, "candidates": 0, "midpoints": 0}
    with ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1))) as ex:
        futs = [ex.submit(inputs.clustered, seed0 + s, points, points // 20) for s in range(n_inputs)]
        for s, fut in enumerate(futs):
            r = refine.learn_explore(fut.result(), theta, levels=levels, seed=seed0 + s, device=device, mlp=mlp,
                                     eps=eps)
            d = refine.descendants(r["parent"], r["inserted"], r["midpoints"], depth)
            keep = (r["level"] != -1) & (r["inserted"] == 1)
            X.append(r["features"][keep])
            T.append(r["t_used"][keep])
            D.append(d[keep].astype(np.float32))
            info["rows"] += int(r["level"].shape[0])
            info["inserted"] += int(r["inserted"].sum())
            info["candidates"] += int(keep.sum())
            info["midpoints"] += int(r["midpoints"].sum())
    return np.concatenate(X), np.concatenate(T), np.concatenate(D), info


def with_t(X, t):
    Z = np.array(X, np.float32, copy=True)
    Z[:, T_SLOT] = t
    return Z


def descendant_targets(X, T, D, epochs, batch, lr, margin, clip, device=0, seed=0, ensemble=4, nlevels=LEVELS):
    """Regression networks of the descendant count (`ensemble` of them, from
    different initialisations and shuffles, their predictions averaged), and
    the placement target of every row: the level predicted lowest (the
    off-center unless another level is lower by more than `margin`)."""
    y = np.minimum(D, clip).astype(np.float32)
    levels = np.arange(nlevels, dtype=np.float32) / (nlevels - 1)
    pred, losses = 0.0, []
    for k in range(ensemble):
        reg, loss = refine.mlp_train(refine.mlp_init(1 + seed + k, float(y.mean())), with_t(X, T), y, epochs=epochs,
                                     batch=batch, lr=lr, seed=seed + k, device=device)
        losses.append(loss)
        pred = pred + np.stack([refine.mlp_infer(reg, with_t(X, t), device=device) for t in levels], axis=1)
    pred = pred / ensemble
    loss = float(np.mean(losses))
    best = pred.argmin(axis=1)
    gain = pred[:, 0] - pred[np.arange(pred.shape[0]), best]
    best = np.where(gain > margin, best, 0)
    tgt = levels[best]
    # observed mean count per inserted level (the exploration's own evidence)
    observed = {f"{t:.2f}": float(y[np.isclose(T, t)].mean()) if np.any(np.isclose(T, t)) else None for t in levels}
    stats = {"regression_loss": loss, "label_variance": float(y.var()), "observed_mean_by_t": observed,
             "predicted_mean_by_t": {f"{t:.2f}": float(pred[:, j].mean()) for j, t in enumerate(levels)},
             "rows_moved": float((best > 0).mean()),
             "predicted_gain_per_moved_row": float(gain[best > 0].mean()) if np.any(best > 0) else 0.0}
    return tgt.astype(np.float32), stats


def evaluate(params, n, points, theta, device=0):
    from .certify import certify
    out = []
    for s in range(n):
        cdt = inputs.clustered(seed=9100 + s, n=points, nseg=points // 20)
        a, sa = refine.refine(cdt, theta, device=device)
        b, sb = refine.refine(cdt, theta, device=device, mlp=params)
        ca, cb = certify(a, cdt, theta), certify(b, cdt, theta)
        out.append({"seed": 9100 + s, "plain_vertices": a.numberofpoints, "learned_vertices": b.numberofpoints,
                    "vertex_reduction": (a.numberofpoints - b.numberofpoints) / a.numberofpoints,
                    "plain_ms": sa["device_ms"], "learned_ms": sb["device_ms"],
                    "learned_used": sb["learned_used"], "learned_candidates": sb["learned_candidates"],
                    "certified": bool(ca["ok"] and cb["ok"]), "min_angle_deg": cb["min_angle_deg"]})
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--labels", choices=["descendants", "one-step"], default="descendants")
    ap.add_argument("--inputs", type=int, default=None)
    ap.add_argument("--points", type=int, default=200_000)
    ap.add_argument("--theta", type=float, default=20.0)
    ap.add_argument("--rows-per-input", type=int, default=20_000, help="one-step labels: rows kept per input")
    ap.add_argument("--depth", type=int, default=5, help="descendant labels: generations counted (0: all)")
    ap.add_argument("--margin", type=float, default=0.0, help="descendant labels: predicted gain to leave t = 0")
    ap.add_argument("--clip", type=float, default=64.0, help="descendant labels: counts clipped for the regression")
    ap.add_argument("--iterations", type=int, default=1,
                    help="descendant labels: rounds of exploration; from the second on, candidates take the last "
                         "network's t except for a fraction --eps that draw a level")
    ap.add_argument("--eps", type=float, default=0.3)
    ap.add_argument("--train-seed", type=int, default=0,
                    help="descendant labels: regression k starts from seed train_seed + k, the placement network "
                         "from train_seed + 10")
    ap.add_argument("--ensemble", type=int, default=4, help="descendant labels: regression networks averaged")
    ap.add_argument("--levels", type=int, default=LEVELS, help="descendant labels: levels of t explored and chosen")
    ap.add_argument("--epochs", type=int, default=None)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--eval", type=int, default=0)
    ap.add_argument("--eval-points", type=int, default=100_000)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    t0 = time.time()
    report = {"labels": a.labels, "points": a.points, "theta": a.theta}
    if a.labels == "one-step":
        n_in = a.inputs or 500
        epochs = a.epochs or 30
        X, T = collect(n_in, a.points, a.theta, a.rows_per_input, device=a.device)
        t1 = time.time()
    else:
        n_in = a.inputs or 128
        epochs = a.epochs or 20
        net = None
        report["iterations"] = []
        for it in range(a.iterations):
            # a fresh set of inputs per iteration (seeds 1000 + 10000 * it, ...)
            X, Tu, D, info = explore(n_in, a.points, a.theta, a.depth, seed0=1000 + 10000 * it, device=a.device,
                                     mlp=net, eps=a.eps if net is not None else 1.0, levels=a.levels)
            T, st = descendant_targets(X, Tu, D, epochs, a.batch, a.lr, a.margin, a.clip, device=a.device,
                                       seed=a.train_seed, ensemble=a.ensemble, nlevels=a.levels)
            Tenc = np.where(T == 0, -0.25, T).astype(np.float32)
            ps = a.train_seed + 10
            net, loss = refine.mlp_train(refine.mlp_init(ps, float(Tenc.mean())), with_t(X, 0.0), Tenc,
                                         epochs=epochs, batch=a.batch, lr=a.lr, seed=ps, device=a.device)
            st.update(info)
            st["placement_loss"] = loss
            if a.eval:
                st["eval"] = evaluate(net, a.eval, a.eval_points, a.theta, device=a.device)
            report["iterations"].append(st)
        t1 = time.time()
        report["depth"] = a.depth
        report["margin"] = a.margin
        report["eps"] = a.eps
        p = net
    if a.labels == "one-step":
        Tenc = np.where(T == 0, -0.25, T).astype(np.float32)
        p, loss = refine.mlp_train(refine.mlp_init(0, float(Tenc.mean())), with_t(X, 0.0), Tenc, epochs=epochs,
                                   batch=a.batch, lr=a.lr, device=a.device)
    t2 = time.time()
    if a.out:
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        np.save(a.out, p)
    report.update({"rows_trained": int(X.shape[0]), "inputs": n_in, "epochs": epochs, "collect_s": t1 - t0,
                   "train_s": t2 - t1, "final_loss": loss, "target_variance": float(Tenc.var()), "out": a.out})
    if a.eval and a.labels == "one-step":
        report["eval"] = evaluate(p, a.eval, a.eval_points, a.theta, device=a.device)
    print(json.dumps(report))
    return report


if __name__ == "__main__":
    main()
