"""Train the learned Steiner placement network on the GPU.

    python -m gpu_cdt_refine_b200.train_placement [--inputs 500] [--points 200000]
        [--theta 20] [--rows-per-input 20000] [--epochs 30]
        [--out gpu_cdt_refine_b200/data/placement_mlp.npy]

Training rows come from plain refinements (gqm_learn_collect) of seeded inputs
of the clustered distribution (64 isotropic Gaussians plus 10% uniform
background, segments 5% of the points), seeds 1000, 1001, ...; the network is
trained by the library's own forward/backward kernels with Adam
(gqm_mlp_train).  A target of 0 (keep the off-center) is encoded as -0.25 so
that the trained network answers "keep" with an output below 0, where the
placement rule falls back to the off-center.
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


def collect(n_inputs, points, theta, rows_per_input, seed0=1000, device=0):
    """Rows of n_inputs seeded inputs (at most rows_per_input of each, a seeded
    sample); inputs are built on host threads while the GPU refines."""
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--inputs", type=int, default=500)
    ap.add_argument("--points", type=int, default=200_000)
    ap.add_argument("--theta", type=float, default=20.0)
    ap.add_argument("--rows-per-input", type=int, default=20_000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    t0 = time.time()
    X, T = collect(a.inputs, a.points, a.theta, a.rows_per_input)
    t1 = time.time()
    Tenc = np.where(T == 0, -0.25, T).astype(np.float32)
    p, loss = refine.mlp_train(refine.mlp_init(0, float(Tenc.mean())), X, Tenc, epochs=a.epochs, batch=a.batch,
                               lr=a.lr)
    t2 = time.time()
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.save(a.out, p)
    print(json.dumps({"rows": int(X.shape[0]), "inputs": a.inputs, "points": a.points, "theta": a.theta,
                      "collect_s": t1 - t0, "train_s": t2 - t1, "final_loss": loss,
                      "target_variance": float(Tenc.var()), "out": a.out}))


if __name__ == "__main__":
    main()
