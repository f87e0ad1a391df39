"""Learned selector on the GPU: structural-feature kernel and the MLP's hand-written
forward / backward / softmax cross-entropy / Adam kernels, each against its CPU oracle.

Tolerances: features (FP64 sums, atomics in any order) relative 1e-10 of the oracle; MLP
loss and gradients (FP32 kernels vs the FP64 oracle) within 1e-4 of the gradient's scale;
Adam within 1e-5 relative.
"""
import importlib

import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


def _sel(sb):
    return importlib.import_module("spmv_dare_b200.selector")


@pytest.mark.parametrize("name", golden_names())
def test_features_match_oracle_on_golden(sb, orc, name):
    g = load_golden(name)
    rp, ci = g["row_ptr"], g["col_ind"]
    m, n = rp.size - 1, int(g["n"])
    got = _sel(sb).features(rp, ci, m, n)
    ref = orc.features(rp, ci, m, n)
    assert np.allclose(got, ref, rtol=1e-10, atol=1e-12), (got, ref)


@pytest.mark.parametrize("args", [(20000, 20000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7),
                                  (15000, 18000, 8, 3, "normal", "random", 0.4, 10, 1.0, 0.8, 21)])
def test_features_match_oracle_generated(sb, orc, args):
    gen = sb.generate_artificial(*args)
    m, n = gen.m, args[1]
    got = _sel(sb).features(gen.row_ptr, gen.col_ind, m, n)
    assert np.allclose(got, orc.features(gen.row_ptr, gen.col_ind, m, n), rtol=1e-10, atol=1e-12)


def test_features_device_path_equals_host_path(sb):
    import torch

    g = load_golden("gen_gamma_skew_2000")
    rp, ci = g["row_ptr"], g["col_ind"]
    m, n = rp.size - 1, int(g["n"])
    S = _sel(sb)
    h = S.features(rp, ci, m, n)
    d = S.features_device(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), m, n, int(rp[-1]))
    assert np.allclose(h, d, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("B,dims", [(96, (10, 64, 64, 24)), (7, (10, 5, 3, 2)), (300, (10, 64, 64, 24))])
def test_mlp_loss_and_gradients_match_oracle(sb, orc, B, dims):
    import torch

    S = _sel(sb)
    rng = np.random.default_rng(B)
    p = S.MLP.init_params(dims, 3)
    p[p.size - dims[3]:] = rng.normal(scale=0.1, size=dims[3])      # non-zero output bias
    X = rng.normal(size=(B, dims[0])).astype(np.float32)
    y = rng.integers(0, dims[3], B).astype(np.int32)
    mlp = S.MLP(dims, params=p)
    loss = mlp.loss_grad(torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda())
    g = mlp.grads()
    loss_o, g_o, z_o = orc.mlp_loss_grad(p.astype(np.float64), dims, X.astype(np.float64), y)
    assert abs(loss - loss_o) <= 1e-5 * max(1.0, abs(loss_o))
    scale = np.max(np.abs(g_o))
    assert np.max(np.abs(g - g_o)) <= 1e-4 * scale, np.max(np.abs(g - g_o)) / scale
    logits = mlp.logits(torch.from_numpy(X).cuda()).cpu().numpy()
    assert np.max(np.abs(logits - z_o)) <= 1e-4 * max(1.0, np.max(np.abs(z_o)))


def test_adam_step_matches_restatement(sb):
    import torch

    S = _sel(sb)
    dims = (10, 64, 64, 24)
    rng = np.random.default_rng(1)
    p0 = S.MLP.init_params(dims, 9)
    X = torch.from_numpy(rng.normal(size=(64, 10)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.integers(0, 24, 64).astype(np.int32)).cuda()
    mlp = S.MLP(dims, params=p0)
    p, m1, m2 = p0.astype(np.float64), np.zeros(p0.size), np.zeros(p0.size)
    lr, b1, b2, eps, wd = 1e-2, 0.9, 0.999, 1e-8, 1e-3
    for t in range(1, 4):
        mlp.loss_grad(X, y)
        g = mlp.grads().astype(np.float64)
        mlp.adam_step(lr, b1, b2, eps, wd)
        m1 = b1 * m1 + (1 - b1) * g
        m2 = b2 * m2 + (1 - b2) * g * g
        p = p - lr * ((m1 / (1 - b1 ** t)) / (np.sqrt(m2 / (1 - b2 ** t)) + eps) + wd * p)
        got = mlp.params().astype(np.float64)
        assert np.max(np.abs(got - p)) <= 1e-5 * max(1.0, np.max(np.abs(p)))
        mlp.set_params(p.astype(np.float32))


def test_training_learns_a_separable_rule(sb):
    """A rule the features determine (which of 4 feature regions) is learned to >= 95%."""
    S = _sel(sb)
    rng = np.random.default_rng(0)
    F = np.abs(rng.normal(size=(3500, 10))) + 0.1
    labels = (F[:, 2] > 0.8).astype(int) * 2 + (F[:, 7] > 0.8).astype(int)
    sel = S.Selector.train(F[:3000], labels[:3000], epochs=100, batch=100, lr=3e-3, seed=2)
    assert sel.losses[-1] < 0.5 * sel.losses[0]
    acc = np.mean(sel.predict(F[3000:]) == labels[3000:])     # 0.964 with the FP64 oracle
    assert acc >= 0.95, acc


def test_trained_selector_regret_and_gain(sb):
    """Trained by the library's kernels on the committed autotuning database (6,074 matrices,
    seeds 0-6073, rows log-uniform in [1e4, 2e6], 29 classes) and judged on 2,000 held-out
    matrices (seeds 50000-51999) against the exhaustive autotuner:
    * within 5% of exhaustive-autotune throughput on average;
    * better than the method without it (the library default class) on average;
    * at >= 100x lower tuning cost (device features + one forward pass against the
      conversions and timing runs of all classes)."""
    ts = importlib.import_module("spmv_dare_b200.train_selector")
    import os

    data = os.path.join(os.path.dirname(sb.__file__), "data")
    tr = ts.load_db(os.path.join(data, "tune_selector_train.npz"))
    te = ts.load_db(os.path.join(data, "tune_selector_test.npz"))
    sel = ts.train(sb, tr, epochs=300)
    ev = ts.evaluate(sel, te)
    assert ev["mlp_ratio_mean"] >= 0.95, ev
    assert ev["mlp_ratio_mean"] >= ev["default_ratio_mean"] + 0.005, ev
    cost = ts.mlp_cost(sb, sel, te, count=4)
    assert ev["exhaustive_tune_s_mean"] / cost >= 100.0, (ev["exhaustive_tune_s_mean"], cost)


def test_selector_save_load_roundtrip(sb, tmp_path):
    S = _sel(sb)
    rng = np.random.default_rng(4)
    F = np.abs(rng.normal(size=(200, 10))) + 0.1
    y = (F[:, 0] > 1.0).astype(int)
    sel = S.Selector.train(F, y, epochs=20, batch=50, seed=1)
    p = tmp_path / "sel.npz"
    sel.save(p)
    sel2 = S.Selector.load(p)
    assert np.array_equal(sel.predict(F), sel2.predict(F))
    assert np.allclose(sel.proba(F), sel2.proba(F), rtol=0, atol=0)
