"""Batched SpMV: many uneven matrices, mixed formats, one persistent launch (work queue)
and its CUDA graph; every matrix's y is bit-identical to its own single-matrix handle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _matrices(sb, count, seed):
    rng = np.random.default_rng(seed)
    mats = []
    for k in range(count):
        rows = int(np.exp(rng.uniform(np.log(300), np.log(20000))))
        avg = float(rng.uniform(5, 60))
        g = sb.generate_artificial(rows, rows, avg, avg * float(rng.uniform(0.1, 1.0)),
                                   "normal" if rng.random() < 0.5 else "gamma", "random",
                                   float(rng.uniform(0.01, 0.5)), float(rng.uniform(0, 200)),
                                   float(rng.uniform(0.5, 2.0)), float(rng.uniform(0.0, 0.8)), 1000 + k)
        mats.append((g.row_ptr, g.col_ind, 2.0 * g.values - 1.0, g.m, g.m))
    return mats


FORMAT_CYCLE = ["csr_naive", {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 256}, "sell",
                {"format": "sell_sorted", "vec_len": 8}, {"format": "sell_c_s", "sellcs_c": 64, "sellcs_sigma": 512}]


@pytest.mark.parametrize("graph", [False, True])
def test_batch_equals_single_matrix_handles(sb, graph):
    import torch

    mats = _matrices(sb, 24, 7)
    formats = [FORMAT_CYCLE[i % len(FORMAT_CYCLE)] for i in range(len(mats))]
    b = sb.Batch(mats, formats)
    assert b.count == 24 and b.total_nnz == sum(int(m[0][-1]) for m in mats)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, b.total_x)
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((b.total_y,), 5.0, dtype=torch.float64, device="cuda")
    for _ in range(3):                      # repeated launches reuse the queue / the graph
        b.spmv(xd, yd, graph=graph)
    b.sync()
    y = yd.cpu().numpy()
    for i, ((rp, ci, v, m, n), f) in enumerate(zip(mats, formats)):
        params = dict(f) if isinstance(f, dict) else {"format": f}
        fmt = params.pop("format")
        mf = sb.csr_to_format(rp, ci, v, m, n, int(rp[-1]), format=fmt, **params)
        xo, yo = b.x_offsets[i], b.y_offsets[i]
        y1 = mf.spmv(x[xo:xo + n])
        assert np.array_equal(y[yo:yo + m].view(np.uint64), y1.view(np.uint64)), (i, fmt)


def test_batch_rejects_unbatchable_format(sb):
    mats = _matrices(sb, 2, 9)
    with pytest.raises(sb.SpmvError):
        sb.Batch(mats, ["csr_naive", "div_rf"])
