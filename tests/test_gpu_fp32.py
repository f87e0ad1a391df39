"""FP32 storage variant (FP32 values, exact int32 indices, Dot2-compensated FP32 rows).

Bars: y bit-identical to the oracle's sequential Dot2 rows (every row with the default
warp-specialised kernel; with kernel 0, rows that fit one staged block, longer rows being
reduced by a compensated tree and checked by tolerance), and max relative error against
the FP64 result <= 1e-6 per row, relative to max(|y_i|, sum_j |a_ij x_j|).
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_row_error

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-6


def _run(sb, rp, ci, v, x, **kw):
    mf = sb.csr_to_format(rp, ci, v, rp.size - 1, x.size, int(rp[-1]), format="csr_naive", value_type="f32", **kw)
    y32 = mf.spmv(x.astype(np.float32), np.full(mf.m, 1.0, np.float32))
    y64 = mf.spmv(x, np.full(mf.m, 1.0))          # FP64 buffers: x rounded once, y widened
    return mf, y32, y64


@pytest.mark.parametrize("kernel", [-1, 4, 0, 7])
@pytest.mark.parametrize("name", golden_names())
def test_fp32_variant_matches_dot2_oracle(sb, orc, name, kernel):
    """Kernel 4 (warp-specialised, the default): every row, long ones included, is one
    sequential Dot2 chain, bit-identical to the oracle.  Kernel 0 reduces rows longer than
    one staged block with a compensated tree: only the other rows are bit-identical.
    Kernel 7 (segmented: Dot2 per lane, compensated merges across lanes and chunks) fixes
    another order: it is held to the error bound and to within 2e-7 of the oracle's rows."""
    g = load_golden(name)
    rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
    mf, y32, y64 = _run(sb, rp, ci, v, x, kernel=kernel)
    assert mf.export("values").dtype == np.float32
    assert np.array_equal(mf.export("values"), v.astype(np.float32))
    ref = orc.csr_f32_dot2(rp, ci, v.astype(np.float32), x.astype(np.float32))
    lens = np.diff(rp)
    gold, absy = orc.csr_gold(rp, ci, v, x)
    if kernel == 7:
        scale = np.maximum(np.abs(ref.astype(np.float64)), absy)
        assert np.all(np.abs(y32.astype(np.float64) - ref) <= 2e-7 * np.maximum(scale, 1e-30))
    else:
        short = lens <= 2048 if kernel == 0 else np.ones(lens.size, bool)
        assert np.array_equal(y32[short].view(np.uint32), ref[short].view(np.uint32))
    assert np.array_equal(y64.astype(np.float32).view(np.uint32), y32.view(np.uint32))
    assert rel_row_error(y32.astype(np.float64), gold, absy) <= TOL_F32


@pytest.mark.parametrize("kw", [dict(row_assign=1), dict(row_assign=1, block_nnz=256), dict(row_assign=1, threads=512,
                                                                                          block_rows=256)])
def test_fp32_longest_first_rows_match_dot2_oracle(sb, orc, kw):
    """row_assign 1 (the row threads of a block take its rows longest first): the same bits."""
    for name in golden_names():
        g = load_golden(name)
        rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
        mf, y32, y64 = _run(sb, rp, ci, v, x, **kw)
        ref = orc.csr_f32_dot2(rp, ci, v.astype(np.float32), x.astype(np.float32))
        assert np.array_equal(y32.view(np.uint32), ref.view(np.uint32)), (name, kw)
        assert np.array_equal(y64.astype(np.float32).view(np.uint32), y32.view(np.uint32))


@pytest.mark.parametrize("sigma", [512, 32, 4096])
def test_fp32_slices_match_dot2_oracle(sb, orc, sigma):
    """The FP32 variant on SELL-C-sigma slices of 32 rows (FP32 values column-major, column
    offsets packed per 8 x 32 tile with a base and a fixed bit width, padding skipped): y is
    the CSR rows' sequential Dot2 bit for bit, through FP32 and FP64 buffers, on every golden
    case, on rows up to 3,000 entries (heavy slices) and on tiles needing 0 to 22 bits."""
    cases = [load_golden(n) for n in golden_names()]
    rng = np.random.default_rng(23)
    m, n = 30000, 4000000
    lens = rng.integers(0, 40, m)
    lens[rng.choice(m, 60, replace=False)] = rng.integers(200, 3000, 60)
    lens[rng.choice(m, 700, replace=False)] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    spans = 2 ** rng.integers(0, 23, m)
    ci = np.concatenate([np.sort(rng.choice(max(k, min(n, s)), size=k, replace=False)) + rng.integers(0, n - max(k, min(n, s)) + 1)
                         if k else np.zeros(0, np.int64) for k, s in zip(lens, spans)]).astype(np.int32)
    cases.append(dict(row_ptr=rp, col_ind=ci, values=rng.uniform(-1, 1, ci.size), x=rng.uniform(-1, 1, n)))
    for g in cases:
        rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
        mf = sb.csr_to_format(rp, ci, v, rp.size - 1, x.size, int(rp[-1]), format="sell_c_s", sellcs_c=32,
                              sellcs_sigma=sigma, value_type="f32")
        assert mf.format_name == "SELL_C_s_F32_Dot2_B200"
        ref = orc.csr_f32_dot2(rp, ci, v.astype(np.float32), x.astype(np.float32))
        for _ in range(2):                                # the work queue is reset by each launch
            y32 = mf.spmv(x.astype(np.float32), np.full(mf.m, 1.0, np.float32))
            assert np.array_equal(y32.view(np.uint32), ref.view(np.uint32)), (rp.size - 1, sigma)
        y64 = mf.spmv(x, np.full(mf.m, 1.0))
        assert np.array_equal(y64.astype(np.float32).view(np.uint32), ref.view(np.uint32))
    with pytest.raises(sb.SpmvError):
        sb.csr_to_format(rp, ci, v, rp.size - 1, x.size, int(rp[-1]), format="sell_c_s", sellcs_c=64,
                         sellcs_sigma=512, value_type="f32")


@pytest.mark.parametrize("block_nnz", [0, 256, 3072])
def test_fp32_packed_columns_match_dot2_oracle(sb, orc, block_nnz):
    """pack_cols=1: the kernel reads the column indices packed per staged block (smallest
    column + a fixed bit width; 1-bit to 31-bit fields, long rows as chunk runs); y is the
    sequential Dot2 oracle's bit for bit on every golden case and on a matrix whose blocks
    need every field width from 0 to 22 bits."""
    cases = [load_golden(n) for n in golden_names()]
    rng = np.random.default_rng(21)
    m, n = 3000, 4000000
    lens = rng.integers(0, 60, m)
    lens[::97] = rng.integers(500, 5000, lens[::97].size)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    spans = 2 ** rng.integers(0, 23, m)
    ci = np.concatenate([np.sort(rng.integers(0, max(1, min(n, s)), k)) + rng.integers(0, n - min(n, s) + 1)
                         for k, s in zip(lens, spans)]).astype(np.int32)
    cases.append(dict(row_ptr=rp, col_ind=ci, values=rng.uniform(-1, 1, ci.size), x=rng.uniform(-1, 1, n)))
    for g in cases:
        rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
        mf, y32, y64 = _run(sb, rp, ci, v, x, pack_cols=1, block_nnz=block_nnz)
        ref = orc.csr_f32_dot2(rp, ci, v.astype(np.float32), x.astype(np.float32))
        assert np.array_equal(y32.view(np.uint32), ref.view(np.uint32)), (rp.size - 1, block_nnz)
        assert np.array_equal(y64.astype(np.float32).view(np.uint32), y32.view(np.uint32))
        assert np.array_equal(mf.export("col_ind"), ci)


@pytest.mark.parametrize("kernel", [7, -1])
@pytest.mark.parametrize("case", ["long_rows", "empty_rows", "chunk_multiple", "one_long_row"])
def test_fp32_segmented_kernel_edge_cases(sb, orc, case, kernel):
    """Kernel 7 on rows across many 256-entry chunks, empty rows (leading, inner, trailing),
    nnz an exact multiple of the chunk, a single row spanning every chunk (and the default
    kernel on the same cases): within the error bound, empty rows zero."""
    rng = np.random.default_rng(len(case))
    if case == "long_rows":
        lens = rng.integers(0, 3000, 200)
    elif case == "empty_rows":
        lens = np.where(rng.random(3000) < 0.4, 0, rng.integers(1, 40, 3000))
        lens[:7] = 0
        lens[-11:] = 0
    elif case == "chunk_multiple":
        lens = np.full(1024, 64)                        # nnz = 65536 = 256 chunks of 256
    else:
        lens = np.array([5000])
    n = 8192
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32) \
        if lens.sum() else np.zeros(0, np.int32)
    v = rng.uniform(-1, 1, int(rp[-1]))
    x = rng.uniform(-1, 1, n)
    mf = sb.csr_to_format(rp, ci, v, rp.size - 1, n, int(rp[-1]), format="csr_naive", value_type="f32", kernel=kernel)
    y32 = mf.spmv(x.astype(np.float32), np.full(mf.m, 7.0, np.float32))
    gold, absy = orc.csr_gold(rp, ci, v, x)
    assert np.all(y32[lens == 0] == 0.0)
    assert rel_row_error(y32.astype(np.float64), gold, absy) <= TOL_F32


def test_fp32_device_path(sb, orc):
    import torch

    g = load_golden("gen_gamma_skew_2000")
    rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
    mf, y32, _ = _run(sb, rp, ci, v, x)
    xd = torch.from_numpy(x.astype(np.float32)).cuda()
    yd = torch.zeros(mf.m, dtype=torch.float32, device="cuda")
    mf.spmv(xd, yd)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy().view(np.uint32), y32.view(np.uint32))
