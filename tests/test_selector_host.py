"""Host logic of the learned selector and its committed data, without a GPU: the training
database's arrays, the near-best labels and throughput ratios of train_selector.py, and the
committed model (spmv-dare_b200/data/selector_model.npz) judged on the held-out database
through the FP64 restatement of its forward pass (oracle.mlp_loss_grad)."""
import importlib
import os

import numpy as np
import pytest

from conftest import ROOT

DATA = os.path.join(ROOT, "spmv-dare_b200", "data")


def _mods(sb):
    return (importlib.import_module("spmv_dare_b200.train_selector"), importlib.import_module("spmv_dare_b200.tuning"),
            importlib.import_module("spmv_dare_b200.selector"))


def test_databases_are_well_formed(sb):
    ts, tuning, _ = _mods(sb)
    tr = ts.load_db(os.path.join(DATA, "tune_selector_train.npz"))
    te = ts.load_db(os.path.join(DATA, "tune_selector_test.npz"))
    for db, lo in ((tr, 0), (te, 50000)):
        t = db["times_ms"]
        assert t.shape == (db["seeds"].size, len(tuning.CLASSES)) and db["features"].shape == (t.shape[0], 10)
        assert db["seeds"][0] == lo and np.all(np.diff(db["seeds"]) == 1)       # consecutive seeds
        assert np.all(np.isfinite(t[:, tuning.DEFAULT_CLASS])) and np.all(t[np.isfinite(t)] > 0)
        assert np.all((db["m"] >= 1e4) & (db["m"] <= 2e6))
        assert np.array_equal(db["best"], np.argmin(np.where(np.isfinite(t), t, np.inf), axis=1))
    assert tr["seeds"].size >= 6000 and te["seeds"].size == 2000


def test_labels_and_ratios(sb):
    ts, _, _ = _mods(sb)
    t = np.array([[1.0, 1.005, 2.0, np.inf], [3.0, 1.5, 1.5, np.nan]])
    F = np.arange(20.0).reshape(2, 10)
    Fx, y = ts.near_best_rows(F, t, near=0.01)
    assert list(y) == [0, 1, 1, 2] and np.array_equal(Fx[2], F[1])
    r = ts.ratios(t, np.array([2, 3]))
    assert r[0] == 0.5 and r[1] == 0.0                  # an untimed class scores 0


def test_committed_model_regret_on_held_out_matrices(sb, orc):
    """The committed network (FP32 parameters, logits recomputed in FP64) within 5% of the
    exhaustive autotuner on the 2,000 held-out matrices and above the library default."""
    ts, tuning, sel = _mods(sb)
    te = ts.load_db(os.path.join(DATA, "tune_selector_test.npz"))
    with np.load(os.path.join(DATA, "selector_model.npz")) as z:
        params, dims, mean, std = z["params"], tuple(int(d) for d in z["dims"]), z["mean"], z["std"]
    assert dims == (10, 64, 64, len(tuning.CLASSES))
    Z = ((sel.model_inputs(te["features"]) - mean) / std).astype(np.float32).astype(np.float64)
    _, _, logits = orc.mlp_loss_grad(params.astype(np.float64), dims, Z, np.zeros(Z.shape[0], np.int64))
    r = ts.ratios(te["times_ms"], np.argmax(logits, axis=1))
    d = ts.ratios(te["times_ms"], np.full(r.size, tuning.DEFAULT_CLASS))
    assert r.mean() >= 0.95, r.mean()
    assert r.mean() >= d.mean() + 0.005, (r.mean(), d.mean())
