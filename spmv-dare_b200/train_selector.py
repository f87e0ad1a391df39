"""Trains the learned selector on an autotuning database and evaluates it on held-out matrices.

    python spmv-dare_b200/train_selector.py [--train data/tune_selector_train.npz]
        [--test data/tune_selector_test.npz] [--out data/selector_model.npz]

Training rows: every class within `near` (default 1%) of a matrix's best time is a label of
that matrix's features (the classes the autotuner cannot tell apart), so the network learns
the near-optimal set rather than one arbitrary winner.  Evaluation on held-out matrices:
the throughput of the chosen class relative to the exhaustive autotuner's best (1.0 = the
best), for the MLP and for the library default without it (tuning.DEFAULT_CLASS); and the
tuning cost: exhaustive (conversion + timing of every class, from the database) against the
MLP's (GPU features of a matrix already on the device + one forward pass), measured here.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_db(path):
    """A database as arrays; classes appended to tuning.CLASSES after it was built read as
    not timed (NaN)."""
    from spmv_dare_b200 import tuning

    with np.load(path) as z:
        db = {k: z[k] for k in z.files}
    t = db["times_ms"]
    if t.shape[1] < len(tuning.CLASSES):
        db["times_ms"] = np.concatenate([t, np.full((t.shape[0], len(tuning.CLASSES) - t.shape[1]), np.nan)], axis=1)
    return db


def ratios(times, chosen):
    """Per-matrix throughput of the chosen class over the best class."""
    t = np.where(np.isfinite(times), times, np.inf)
    best = np.min(t, axis=1)
    pick = t[np.arange(t.shape[0]), chosen]
    return np.where(np.isfinite(pick), best / pick, 0.0)


def near_best_rows(F, times, near=0.01):
    """(features, labels): one row per (matrix, class within `near` of its best time)."""
    t = np.where(np.isfinite(times), times, np.inf)
    best = np.min(t, axis=1, keepdims=True)
    ii, cc = np.nonzero(t <= best * (1.0 + near))
    return F[ii], cc


def train(sb, db, epochs=400, near=0.01, seed=0, log=None):
    from spmv_dare_b200 import selector

    Fx, y = near_best_rows(db["features"], db["times_ms"], near)
    return selector.Selector.train(Fx, y, epochs=epochs, batch=128, lr=3e-3, weight_decay=1e-4, seed=seed, log=log)


def evaluate(sel, db):
    from spmv_dare_b200 import tuning

    pred = sel.predict(db["features"])
    r_mlp = ratios(db["times_ms"], pred)
    r_def = ratios(db["times_ms"], np.full(pred.size, tuning.DEFAULT_CLASS))
    return {"matrices": int(pred.size), "mlp_ratio_mean": float(r_mlp.mean()), "mlp_ratio_min": float(r_mlp.min()),
            "mlp_within_5pct": float(np.mean(r_mlp >= 0.95)), "default_ratio_mean": float(r_def.mean()),
            "default_ratio_min": float(r_def.min()), "exhaustive_ratio_mean": 1.0,
            "exhaustive_tune_s_mean": float(np.mean(db["tune_s"])), "pred": pred}


def mlp_cost(sb, sel, db, count=8):
    """Seconds per matrix of the MLP's tuning: device features + one forward pass (host
    wall time, median of 3 queries per matrix, median over `count` held-out matrices
    regenerated on the GPU from their stored parameters; the CSR arrays are already on the
    GPU)."""
    import torch

    from spmv_dare_b200 import selector, workloads

    costs = []
    names = [str(k) for k in db["param_names"]]
    for i in range(min(count, db["seeds"].size)):
        q = dict(zip(names, db["params"][i].tolist()))
        p = dict(rows=int(q["rows"]), cols=int(q["rows"]), avg=q["avg"], std=q["std"], skew=q["skew"], bw=q["bw"],
                 neigh=q["neigh"], cross=q["cross"], distribution="gamma" if db["gamma"][i] else "normal",
                 placement="random", seed=int(db["seeds"][i]))
        drp, dci, _ = workloads.generate_device(sb, p)
        m, n, nnz = p["rows"], p["cols"], int(dci.numel())
        sel.predict(selector.features_device(drp, dci, m, n, nnz))          # warm-up
        torch.cuda.synchronize()
        per = []
        for _ in range(3):
            t0 = time.perf_counter()
            sel.predict(selector.features_device(drp, dci, m, n, nnz))
            per.append(time.perf_counter() - t0)
        costs.append(float(np.median(per)))
    return float(np.median(costs))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", default=os.path.join(HERE, "data", "tune_selector_train.npz"))
    ap.add_argument("--test", default=os.path.join(HERE, "data", "tune_selector_test.npz"))
    ap.add_argument("--out", default=None)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--near", type=float, default=0.01)
    a = ap.parse_args(argv)
    sys.path.insert(0, HERE)
    import tune_db

    sb = tune_db.load_package()
    tr, te = load_db(a.train), load_db(a.test)
    sel = train(sb, tr, epochs=a.epochs, near=a.near, log=lambda s: print(s, file=sys.stderr))
    ev = evaluate(sel, te)
    ev.pop("pred")
    ev["mlp_tune_s"] = mlp_cost(sb, sel, te)
    ev["tuning_cost_ratio"] = ev["exhaustive_tune_s_mean"] / ev["mlp_tune_s"]
    ev["train_matrices"] = int(tr["features"].shape[0])
    if a.out:
        sel.save(a.out)
    print(json.dumps(ev))


if __name__ == "__main__":
    sys.exit(main())
