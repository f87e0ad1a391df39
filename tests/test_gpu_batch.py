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


@pytest.mark.parametrize("graph", [False, True])
def test_all_csr_batch_runs_as_one_block_diagonal_spmv(sb, graph):
    """An all-csr_naive batch is one SpMV of the block-diagonal matrix (merged on the
    device, warp-specialised kernel): y bit-identical to each matrix's own handle, with
    empty and one-row matrices among them."""
    import torch

    mats = _matrices(sb, 20, 11)
    mats.insert(5, (np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), 0, 3))       # no rows
    mats.insert(9, (np.array([0, 2], np.int32), np.array([0, 4], np.int32), np.array([1.5, -2.0]), 1, 6))
    b = sb.Batch(mats, ["csr_naive"] * len(mats))
    assert b.total_nnz == sum(int(m[0][-1]) for m in mats) and b.num_blocks > 0
    x = np.random.default_rng(5).uniform(-1, 1, b.total_x)
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((b.total_y,), 5.0, dtype=torch.float64, device="cuda")
    for _ in range(3):
        b.spmv(xd, yd, graph=graph)
    b.sync()
    y = yd.cpu().numpy()
    for i, (rp, ci, v, m, n) in enumerate(mats):
        if m == 0:
            continue
        mf = sb.csr_to_format(rp, ci, v, m, n, int(rp[-1]), format="csr_naive")
        xo, yo = b.x_offsets[i], b.y_offsets[i]
        assert np.array_equal(y[yo:yo + m].view(np.uint64), mf.spmv(x[xo:xo + n]).view(np.uint64)), i


def test_all_csr_batch_rejects_column_outside_its_matrix(sb):
    mats = _matrices(sb, 3, 13)
    rp, ci, v, m, n = mats[1]
    ci = ci.copy()
    ci[0] = n                  # valid in the merged matrix's width, invalid for matrix 1
    mats[1] = (rp, ci, v, m, n)
    with pytest.raises(sb.SpmvError):
        sb.Batch(mats, ["csr_naive"] * 3)
