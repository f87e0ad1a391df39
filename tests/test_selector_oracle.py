"""CPU pins of the selector's oracle restatements (no GPU).

* features(): against the reference generator's own statistics
  (artificial_matrix_generation.c:529-570) and its csr_cross_row_similarity
  (matrix_util.h:269-328), on matrices the reference generator makes;
* mlp_loss_grad(): against central finite differences of its own loss, in FP64.
"""
import numpy as np
import pytest

CONFIGS = [
    (3000, 3000, 10, 2, "normal", "random", 0.3, 0, 1.0, 0.5, 14),
    (5000, 5000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7),
    (4000, 4000, 30, 10, "normal", "random", 0.2, 50, 1.5, 0.6, 3),
    (2000, 2500, 5, 5, "gamma", "random", 0.4, 150, 1.0, 0.9, 11),
]


@pytest.mark.parametrize("cfg", CONFIGS)
def test_features_restatement_matches_reference_statistics(orc, cfg):
    if not orc.ref_available("gen"):
        pytest.skip("reference generator not built here")
    rp, ci, v, st = orc.ref_generate(*cfg)
    m, n = rp.size - 1, cfg[1]
    f = orc.features(rp, ci, m, n)
    avg = st["avg_nnz_per_row"]
    assert f[0] == pytest.approx(np.log2(m + 1.0), rel=1e-15)
    assert f[1] == pytest.approx(np.log2(int(rp[-1]) + 1.0), rel=1e-15)
    assert f[2] == pytest.approx(avg, rel=1e-13)
    assert f[3] == pytest.approx(st["std_nnz_per_row"] / avg, rel=1e-12)
    assert f[4] == pytest.approx(st["skew"], rel=1e-12)
    assert f[5] == pytest.approx(st["avg_bw"] / n, rel=1e-12)
    assert f[6] == pytest.approx(st["avg_sc"], rel=1e-12)
    assert f[7] == pytest.approx(st["avg_num_neighbours"], rel=1e-12)
    assert f[8] == pytest.approx(orc.ref_cross_row_similarity(rp, ci, n), rel=1e-12)
    assert f[9] == pytest.approx(st["avg_clustering"], rel=1e-12)


def test_features_restatement_edge_cases(orc):
    # all rows empty; one row; a diagonal
    assert np.all(orc.features(np.zeros(6, np.int32), np.zeros(0, np.int32), 5, 5)[2:] == 0)
    f = orc.features(np.array([0, 3], np.int32), np.array([1, 2, 5], np.int32), 1, 8)
    assert f[5] == pytest.approx(5 / 8) and f[7] == pytest.approx(2 / 3) and f[9] == pytest.approx(2 / 3)
    d = orc.features(np.arange(11, dtype=np.int32), np.arange(10, dtype=np.int32), 10, 10)
    assert d[8] == pytest.approx(0.9) and d[4] == 0.0     # the last row has no next row but counts


def test_mlp_oracle_gradient_matches_finite_differences(orc):
    rng = np.random.default_rng(5)
    dims = (10, 16, 12, 7)
    _, total = orc.mlp_offsets(dims)
    p = rng.normal(scale=0.4, size=total)
    X = rng.normal(size=(9, 10))
    y = rng.integers(0, 7, 9)
    loss, g, _ = orc.mlp_loss_grad(p, dims, X, y)
    h = 1e-6
    idx = rng.choice(total, 60, replace=False)
    for i in idx:
        e = np.zeros(total)
        e[i] = h
        fd = (orc.mlp_loss_grad(p + e, dims, X, y)[0] - orc.mlp_loss_grad(p - e, dims, X, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), i
