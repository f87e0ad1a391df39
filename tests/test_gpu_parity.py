"""GPU parity: conversions and y through the C ABI against the reference's own outputs
(golden fixtures) and the oracle restatement (full-size configs).

Bars:
  * every converted array (row_cluster_ptr, ja, a, permutations, thread ranges, row_order,
    slice widths/pointers, columns, values) bit-identical;
  * y bit-identical to the same format's reference y (each kernel sums a row in the
    reference format's own order: csr_naive split multiply/add, csr_vec 4 FMA lanes,
    sell / sell_sorted / sell_c_s one FMA per slice column);
  * every format within 1e-12 per row of the reference csr_naive y, relative to
    max(|y_i|, sum_j |a_ij x_j|) (the condition-aware tolerance).
"""
import numpy as np
import pytest

from conftest import assert_golden_array, golden_names, load_golden, rel_row_error

pytestmark = pytest.mark.gpu

TOL = 1e-12
T, V = 8, 4
REF_FORMATS = ["csr_naive", "csr_vec", "sell", "sell_sorted"]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def _eq_bits(a, b):
    a, b = np.ascontiguousarray(a, np.float64), np.ascontiguousarray(b, np.float64)
    bad = np.flatnonzero(_bits(a) != _bits(b))
    return bad


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the gpu tests need a CUDA device"
    return torch


def _mk(sb, g, fmt, **kw):
    rp, ci, v = g["row_ptr"], g["col_ind"], g["values"]
    return sb.csr_to_format(rp, ci, v, rp.size - 1, int(g["n"]), int(rp[-1]), format=fmt, **kw)


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("fmt", REF_FORMATS)
def test_format_matches_reference(sb, orc, name, fmt):
    g = load_golden(name)
    mf = _mk(sb, g, fmt, num_threads=T, vec_len=V)
    y = np.full(mf.m, 1.0)            # the reference's empty-row probe (bench_spmv.cpp:561-564)
    mf.spmv(g["x"], y)
    bad = _eq_bits(y, g[f"y_{fmt}"])
    assert bad.size == 0, f"{fmt}/{name}: {bad.size} rows differ from the reference, first {bad[:5]}"
    assert mf.mem_footprint == float(g[f"mem_{fmt}"])
    if fmt in ("sell", "sell_sorted"):
        keys = ["row_cluster_ptr", "ja", "a", "ranges"] + (["permutation", "rev_permutation"] if fmt == "sell_sorted" else [])
        for k in keys:
            assert_golden_array(g, f"{fmt}_{k}", mf.export(k))
    gold, absy = orc.csr_gold(g["row_ptr"], g["col_ind"], g["values"], g["x"])
    assert rel_row_error(y, g["y_csr_naive"], absy) <= TOL


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("C,sigma", [(32, 256), (64, 64)])
def test_sellcs_matches_reference(sb, orc, name, C, sigma):
    g = load_golden(name)
    mf = _mk(sb, g, "sell_c_s", sellcs_c=C, sellcs_sigma=sigma)
    pre = f"sellcs_{C}_{sigma}_"
    assert_golden_array(g, pre + "row_order", mf.export("row_order").astype(np.int64))
    assert_golden_array(g, pre + "slice_widths", mf.export("slice_widths").astype(np.int64))
    assert_golden_array(g, pre + "slice_pointers", mf.export("slice_pointers"))
    assert_golden_array(g, pre + "column_indices", mf.export("column_indices").astype(np.int64))
    assert_golden_array(g, pre + "values", mf.export("sellcs_values"))
    y = mf.spmv(g["x"], np.full(mf.m, 1.0))
    arr = orc.sellcs_convert(g["row_ptr"], g["col_ind"], g["values"], C, sigma)
    y_orc = orc.sellcs_spmv(arr, mf.m, C, g["x"])
    assert _eq_bits(y, y_orc).size == 0
    gold, absy = orc.csr_gold(g["row_ptr"], g["col_ind"], g["values"], g["x"])
    assert rel_row_error(y, g["y_csr_naive"], absy) <= TOL


@pytest.mark.parametrize("fmt", REF_FORMATS + ["sell_c_s"])
def test_device_path_equals_host_path(sb, torch_cuda, fmt):
    torch = torch_cuda
    g = load_golden("gen_gamma_skew_2000")
    mf = _mk(sb, g, fmt)
    y_host = mf.spmv(g["x"])
    xd = torch.from_numpy(g["x"]).cuda()
    yd = torch.full((mf.m,), 7.0, dtype=torch.float64, device="cuda")
    mf.spmv(xd, yd)
    torch.cuda.synchronize()
    assert _eq_bits(yd.cpu().numpy(), y_host).size == 0


@pytest.mark.parametrize("fmt", ["csr_naive", "csr_vec", "sell", "sell_sorted"])
@pytest.mark.parametrize("block_nnz,stages", [(64, 2), (256, 3), (8192, 4)])
def test_staging_geometry_does_not_change_results(sb, fmt, block_nnz, stages):
    """Tiny staging blocks force the long-unit path (rows / slices larger than a block)."""
    for name in ["long_rows_60", "gen_gamma_skew_2000", "empty_rows_333"]:
        g = load_golden(name)
        mf = _mk(sb, g, fmt, block_nnz=block_nnz, stages=stages)
        y = mf.spmv(g["x"], np.full(mf.m, 1.0))
        assert _eq_bits(y, g[f"y_{fmt}"]).size == 0, (name, fmt, block_nnz)


@pytest.mark.parametrize("fmt", ["csr_naive", "csr_vec", "sell", "sell_sorted", "sell_c_s"])
@pytest.mark.parametrize("threads,block_nnz,stages", [(256, 64, 2), (128, 256, 3), (256, 0, 0), (512, 2048, 4)])
def test_pipelined_kernel_matches_reference(sb, orc, fmt, threads, block_nnz, stages):
    """Kernel 3 (next block's gather overlapping this block's rows): same y bits as the
    reference for every golden case; tiny blocks force the long-unit path."""
    for name in golden_names():
        g = load_golden(name)
        mf = _mk(sb, g, fmt, kernel=3, threads=threads, block_nnz=block_nnz, stages=stages)
        y = mf.spmv(g["x"], np.full(mf.m, 1.0))
        if fmt == "sell_c_s":
            arr = orc.sellcs_convert(g["row_ptr"], g["col_ind"], g["values"], 32, 512)
            ref = orc.sellcs_spmv(arr, mf.m, 32, g["x"])
        else:
            ref = g[f"y_{fmt}"]
        assert _eq_bits(y, ref).size == 0, (name, fmt, threads, block_nnz, stages)


@pytest.mark.parametrize("fmt", ["csr_naive", "csr_vec", "sell", "sell_sorted", "sell_c_s"])
@pytest.mark.parametrize("threads,block_rows,block_nnz,stages",
                         [(0, 0, 0, 0), (96, 64, 64, 2), (256, 32, 256, 3), (512, 128, 2048, 4)])
def test_warp_specialised_kernel_matches_reference(sb, orc, fmt, threads, block_rows, block_nnz, stages):
    """Kernel 4 (gather warps + row warps): same y bits as the reference for every golden
    case; 64-entry blocks force the long-unit path of the row warps."""
    for name in golden_names():
        g = load_golden(name)
        mf = _mk(sb, g, fmt, kernel=4, threads=threads, block_rows=block_rows, block_nnz=block_nnz, stages=stages)
        y = mf.spmv(g["x"], np.full(mf.m, 1.0))
        if fmt == "sell_c_s":
            arr = orc.sellcs_convert(g["row_ptr"], g["col_ind"], g["values"], 32, 512)
            ref = orc.sellcs_spmv(arr, mf.m, 32, g["x"])
        else:
            ref = g[f"y_{fmt}"]
        assert _eq_bits(y, ref).size == 0, (name, fmt, threads, block_rows, block_nnz, stages)


def test_warp_specialised_kernel_rejects_bad_split(sb):
    g = load_golden("hand6")
    for kw in [dict(threads=64, block_rows=64), dict(threads=128, block_rows=48)]:
        with pytest.raises(sb.SpmvError):
            _mk(sb, g, "csr_naive", kernel=4, **kw)
    with pytest.raises(sb.SpmvError):       # slices of 32 rows need at least 32 row threads... and 64 > 32
        _mk(sb, g, "sell_c_s", kernel=4, threads=64, block_rows=32, sellcs_c=64, sellcs_sigma=64)


@pytest.mark.parametrize("fmt", ["csr_naive", "csr_vec", "sell", "sell_sorted", "sell_c_s"])
@pytest.mark.parametrize("threads,block_nnz,stages", [(256, 64, 2), (128, 0, 0), (512, 4096, 3)])
def test_own_gather_kernel_matches_reference(sb, orc, fmt, threads, block_nnz, stages):
    """Kernel 5 (row threads load their own x): same y bits as the reference for every
    golden case; 64-entry blocks force the long-unit path."""
    for name in golden_names():
        g = load_golden(name)
        mf = _mk(sb, g, fmt, kernel=5, threads=threads, block_nnz=block_nnz, stages=stages)
        y = mf.spmv(g["x"], np.full(mf.m, 1.0))
        if fmt == "sell_c_s":
            arr = orc.sellcs_convert(g["row_ptr"], g["col_ind"], g["values"], 32, 512)
            ref = orc.sellcs_spmv(arr, mf.m, 32, g["x"])
        else:
            ref = g[f"y_{fmt}"]
        assert _eq_bits(y, ref).size == 0, (name, fmt, threads, block_nnz, stages)


@pytest.mark.parametrize("fmt", ["sell", "sell_sorted", "sell_c_s", "csr_naive"])
@pytest.mark.parametrize("block_nnz,stages", [(64, 2), (0, 0), (1024, 4)])
def test_warp_own_gather_kernel_matches_reference(sb, orc, fmt, block_nnz, stages):
    """Kernel 6 (warp-autonomous, slice rows load their own x; CSR takes kernel 2's path):
    same y bits as the reference for every golden case; 64-entry chunks split long slices."""
    for name in golden_names():
        g = load_golden(name)
        mf = _mk(sb, g, fmt, kernel=6, block_nnz=block_nnz, stages=stages)
        y = mf.spmv(g["x"], np.full(mf.m, 1.0))
        if fmt == "sell_c_s":
            arr = orc.sellcs_convert(g["row_ptr"], g["col_ind"], g["values"], 32, 512)
            ref = orc.sellcs_spmv(arr, mf.m, 32, g["x"])
        else:
            ref = g[f"y_{fmt}"]
        assert _eq_bits(y, ref).size == 0, (name, fmt, block_nnz, stages)


def _sliced_ref(orc, g, fmt, C):
    rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
    m = rp.size - 1
    if fmt == "sell_c_s":
        return orc.sellcs_spmv(orc.sellcs_convert(rp, ci, v, C, 512), m, C, x)
    if fmt == "sell":
        return orc.sell_spmv(orc.sell_convert(rp, ci, v, C, T), m, C, x)
    return orc.sell_sorted_spmv(orc.sell_sorted_convert(rp, ci, v, C, T), m, C, x)


@pytest.mark.parametrize("fmt,C", [("sell_c_s", 32), ("sell_c_s", 64), ("sell", 8), ("sell_sorted", 16),
                                   ("sell", 32), ("sell_sorted", 32)])
@pytest.mark.parametrize("kernel,threads,block_rows,tiles,stages", [(8, 0, 0, 0, 0), (8, 96, 64, 1, 2), (8, 256, 128, 3, 3),
                                                                    (8, 512, 256, 8, 4), (9, 0, 0, 0, 0), (9, 0, 0, 1, 2),
                                                                    (9, 0, 0, 3, 4)])
def test_tiled_kernel_matches_reference(sb, orc, fmt, C, kernel, threads, block_rows, tiles, stages):
    """Kernel 8 (kernel 4 over the column indices in row-major 8-column tiles) and kernel 9
    (warp-owned slices over the same tiles, x transposed between lanes; slices of 32 rows,
    other heights fall back to kernel 8): same y bits as the reference SELL order for every
    golden case, slice heights 8..64 (SELL-C-sigma takes C in [32, 256]); one-tile blocks
    force long slices through chunk runs.  The exported arrays keep the reference layout."""
    kw = dict(sellcs_c=C, sellcs_sigma=512) if fmt == "sell_c_s" else dict(vec_len=C, num_threads=T)
    if threads:
        kw.update(threads=threads, block_rows=block_rows)
    if tiles:
        kw.update(block_nnz=tiles * 8 * C, stages=stages)
    for name in golden_names():
        g = load_golden(name)
        mf = _mk(sb, g, fmt, kernel=kernel, **kw)
        y = mf.spmv(g["x"], np.full(mf.m, 1.0))
        assert _eq_bits(y, _sliced_ref(orc, g, fmt, C)).size == 0, (name, fmt, C, kernel, threads, tiles, stages)
        if fmt == "sell_c_s" and name == golden_names()[0]:
            arr = orc.sellcs_convert(g["row_ptr"], g["col_ind"], g["values"], C, 512)
            assert np.array_equal(mf.export("column_indices"), arr["column_indices"])


def test_tiled_kernel_long_slices(sb, orc):
    """Kernels 8 and 9 on a skewed matrix (rows up to 3000 entries among rows of 0-40, empty rows):
    slices wider than a block run as chunks of whole tiles, narrower last tiles included."""
    rng = np.random.default_rng(8)
    m = n = 20000
    lens = rng.integers(0, 40, m)
    lens[rng.choice(m, 60, replace=False)] = rng.integers(200, 3000, 60)
    lens[rng.choice(m, 500, replace=False)] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32)
    v = rng.uniform(-1, 1, int(rp[-1]))
    x = rng.uniform(-1, 1, n)
    g = dict(row_ptr=rp, col_ind=ci, values=v, x=x, n=n)
    for C in (32, 64):
        ref = orc.sellcs_spmv(orc.sellcs_convert(rp, ci, v, C, 512), m, C, x)
        for kernel in (8, 9):
            for kw in [dict(), dict(block_nnz=8 * C, stages=2), dict(block_nnz=24 * C + 8)]:
                mf = _mk(sb, g, "sell_c_s", kernel=kernel, sellcs_c=C, sellcs_sigma=512, **kw)
                y = mf.spmv(x, np.full(m, 1.0))
                assert _eq_bits(y, ref).size == 0, (C, kernel, kw)


@pytest.mark.parametrize("stages,kw2", [(0, {}), (1, {}), (3, {}), (5, {}), (6, {}), (5, dict(block_rows=2)),
                                        (0, dict(block_rows=1, block_nnz=256)),
                                        (0, dict(block_rows=64, block_nnz=2048))])
@pytest.mark.parametrize("fmt,C,sigma", [("sell_c_s", 32, 512), ("sell_c_s", 32, 32), ("sell_c_s", 32, 4096),
                                         ("sell", 32, 0), ("sell_sorted", 32, 0), ("sell_c_s", 64, 512)])
def test_register_tiled_kernel_matches_reference(sb, orc, fmt, C, sigma, stages, kw2):
    """Kernel 10 (warp-claimed slices of 32 rows summed from registers, no shared memory; the
    lines two tiles ahead prefetched into L2, stages 3: into L1, 5: into L1 with items claimed
    one ahead and their first two tiles prefetched, 6: that form into L2, 1: none;
    block_rows / block_nnz: item size and prefetch distance, 256-entry items included):
    the reference's y bits on every golden case and on a skewed matrix whose heavy slices
    (rows up to 3,000 entries) are claimed first; slice heights other than 32 fall back to
    kernel 8.  Several launches in a row reuse the work queue, which each launch resets."""
    kw = dict(sellcs_c=C, sellcs_sigma=sigma) if fmt == "sell_c_s" else dict(vec_len=C, num_threads=T)
    cases = [load_golden(name) for name in golden_names()]
    rng = np.random.default_rng(10)
    m = n = 30000
    lens = rng.integers(0, 40, m)
    lens[rng.choice(m, 80, replace=False)] = rng.integers(200, 3000, 80)
    lens[rng.choice(m, 700, replace=False)] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32)
    cases.append(dict(row_ptr=rp, col_ind=ci, values=rng.uniform(-1, 1, int(rp[-1])), x=rng.uniform(-1, 1, n), n=n))
    for g in cases:
        ref = (orc.sellcs_spmv(orc.sellcs_convert(g["row_ptr"], g["col_ind"], g["values"], C, sigma),
                               g["row_ptr"].size - 1, C, g["x"]) if fmt == "sell_c_s" else _sliced_ref(orc, g, fmt, C))
        # slices of 64 rows fall back to kernel 8, whose staging blocks are checked apart
        mf = _mk(sb, g, fmt, kernel=10, stages=stages, **(kw2 if C == 32 else {}), **kw)
        for _ in range(3):
            y = mf.spmv(g["x"], np.full(mf.m, 1.0))
            assert _eq_bits(y, ref).size == 0, (fmt, C, sigma, g["row_ptr"].size - 1)


@pytest.mark.parametrize("block_nnz,stages", [(0, 0), (256, 3), (2048, 2)])
def test_packed_columns_csr_naive(sb, orc, block_nnz, stages):
    """pack_cols=1 on FP64 csr_naive (kernel 4 reads the columns packed per staged block):
    the reference's y bits on every golden case, including long rows as chunk runs and
    blocks whose columns span from 1 to 2^22 values."""
    for name in golden_names():
        g = load_golden(name)
        mf = _mk(sb, g, "csr_naive", pack_cols=1, block_nnz=block_nnz, stages=stages)
        y = mf.spmv(g["x"], np.full(mf.m, 1.0))
        assert _eq_bits(y, g["y_csr_naive"]).size == 0, (name, block_nnz)
        assert np.array_equal(mf.export("col_ind"), g["col_ind"])
    rng = np.random.default_rng(31)
    m, n = 4000, 4000000
    lens = rng.integers(0, 50, m)
    lens[::211] = rng.integers(800, 6000, lens[::211].size)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    spans = 2 ** rng.integers(0, 23, m)
    ci = np.concatenate([np.sort(rng.integers(0, max(1, min(n, s)), k)) + rng.integers(0, n - min(n, s) + 1)
                         for k, s in zip(lens, spans)]).astype(np.int32)
    v = rng.uniform(-1, 1, ci.size)
    x = rng.uniform(-1, 1, n)
    mf = sb.csr_to_format(rp, ci, v, m, n, int(rp[-1]), format="csr_naive", pack_cols=1, block_nnz=block_nnz,
                          stages=stages)
    assert _eq_bits(mf.spmv(x, np.full(m, 1.0)), orc.csr_spmv(rp, ci, v, x)).size == 0
    with pytest.raises(sb.SpmvError):
        _mk(sb, load_golden("hand6"), "csr_vec", pack_cols=1)


def test_tiled_kernel_rejects_small_blocks(sb):
    g = load_golden("hand6")
    with pytest.raises(sb.SpmvError):           # a block must hold one 8 x 32 tile
        _mk(sb, g, "sell_c_s", kernel=8, block_nnz=128, sellcs_c=32, sellcs_sigma=64)


def test_pipelined_kernel_rejects_oversized_blocks(sb):
    g = load_golden("hand6")
    with pytest.raises(sb.SpmvError):
        _mk(sb, g, "csr_naive", kernel=3, threads=64, block_nnz=1024)


def test_non_exact_long_rows_within_tolerance(sb, orc):
    g = load_golden("long_rows_60")
    mf = _mk(sb, g, "csr_naive", exact=0, block_nnz=512)
    y = mf.spmv(g["x"])
    gold, absy = orc.csr_gold(g["row_ptr"], g["col_ind"], g["values"], g["x"])
    assert rel_row_error(y, g["y_csr_naive"], absy) <= TOL


@pytest.mark.parametrize("Vw", [32, 64])
@pytest.mark.parametrize("fmt", ["sell", "sell_sorted"])
def test_wide_slices_match_restatement(sb, orc, fmt, Vw):
    g = load_golden("gen_diag_1500")
    rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
    mf = _mk(sb, g, fmt, vec_len=Vw)
    y = mf.spmv(x)
    if fmt == "sell":
        arr = orc.sell_convert(rp, ci, v, Vw, T)
        y_orc = orc.sell_spmv(arr, mf.m, Vw, x)
    else:
        arr = orc.sell_sorted_convert(rp, ci, v, Vw, T)
        y_orc = orc.sell_sorted_spmv(arr, mf.m, Vw, x)
    for k in ["row_cluster_ptr", "ja", "a"]:
        assert np.array_equal(mf.export(k).view(np.uint8), np.ascontiguousarray(arr[k]).view(np.uint8)), k
    assert _eq_bits(y, y_orc).size == 0


@pytest.mark.parametrize("threads", [1, 3, 64])
@pytest.mark.parametrize("fmt", ["sell", "sell_sorted"])
def test_thread_count_layouts(sb, orc, fmt, threads):
    g = load_golden("empty_rows_333")
    rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
    mf = _mk(sb, g, fmt, num_threads=threads)
    conv = orc.sell_convert if fmt == "sell" else orc.sell_sorted_convert
    arr = conv(rp, ci, v, V, threads)
    for k in arr:
        assert np.array_equal(mf.export(k), arr[k]), k


# ------------------------------------------------------------------ edge cases
def _rand_csr(m, n, seed, empty_frac=0.2, maxlen=9):
    rng = np.random.default_rng(seed)
    lens = rng.integers(1, maxlen + 1, m)
    lens[rng.random(m) < empty_frac] = 0
    lens = np.minimum(lens, n)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for k in lens] or [np.empty(0)]).astype(np.int32)
    v = rng.uniform(-1, 1, int(rp[-1]))
    return rp, ci, v


@pytest.mark.parametrize("m,n", [(1, 1), (5, 3), (3, 5), (7, 1000), (1001, 17)])
@pytest.mark.parametrize("fmt", REF_FORMATS + ["sell_c_s", "div_rf"])
def test_small_and_rectangular(sb, orc, fmt, m, n):
    rp, ci, v = _rand_csr(m, n, m * 31 + n)
    x = np.random.default_rng(1).uniform(-1, 1, n)
    mf = sb.csr_to_format(rp, ci, v, m, n, int(rp[-1]), format=fmt)
    y = mf.spmv(x, np.full(m, 1.0))
    if fmt == "csr_naive":
        ref = orc.csr_spmv(rp, ci, v, x)
    elif fmt == "csr_vec":
        ref = orc.csr_vec_spmv(rp, ci, v, x, V)
    elif fmt == "sell":
        ref = orc.sell_spmv(orc.sell_convert(rp, ci, v, V, T), m, V, x)
    elif fmt == "sell_sorted":
        ref = orc.sell_sorted_spmv(orc.sell_sorted_convert(rp, ci, v, V, T), m, V, x)
    elif fmt == "sell_c_s":
        ref = orc.sellcs_spmv(orc.sellcs_convert(rp, ci, v, 32, 512), m, 32, x)
    else:
        d = orc.div_convert(rp, ci, v, n, T, V, 16384, 0.0)
        assert np.array_equal(mf.export("div_data"), d["data"])
        gold, absy = orc.csr_gold(rp, ci, v, x)
        assert rel_row_error(y, gold, absy) <= TOL
        return
    assert _eq_bits(y, ref).size == 0


@pytest.mark.parametrize("fmt", REF_FORMATS + ["sell_c_s", "div_rf"])
def test_all_rows_empty_and_no_entries(sb, fmt):
    m, n = 50, 40
    rp = np.zeros(m + 1, np.int32)
    mf = sb.csr_to_format(rp, np.empty(0, np.int32), np.empty(0), m, n, 0, format=fmt)
    y = mf.spmv(np.ones(n), np.full(m, 1.0))
    assert np.all(y == 0.0)


def test_malformed_csr_is_rejected(sb):
    rp = np.array([0, 2, 1, 3], np.int32)
    with pytest.raises(sb.SpmvError) as e:
        sb.csr_to_format(rp, np.array([0, 1, 2], np.int32), np.ones(3), 3, 3, 3)
    assert e.value.status == 2
    rp = np.array([0, 1, 2], np.int32)
    with pytest.raises(sb.SpmvError) as e:
        sb.csr_to_format(rp, np.array([0, 9], np.int32), np.ones(2), 2, 3, 2)
    assert e.value.status == 2


# ------------------------------------------------------------------ DIV-RF
@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("pv,pre", [(16384, "div"), (1000, "div1000")])
def test_div_rf_matches_reference(sb, orc, name, pv, pre):
    """Packet bytes, packet-group offsets and thread ranges bit-identical to the reference's
    DIVArray; y within the tolerance of the reference's csr_naive y."""
    g = load_golden(name)
    mf = _mk(sb, g, "div_rf", num_threads=T, vec_len=V, div_packet_vals=pv)
    assert_golden_array(g, f"{pre}_data", mf.export("div_data"))
    assert_golden_array(g, f"{pre}_group_pos", mf.export("div_groups"))
    assert_golden_array(g, "div_ranges", mf.export("ranges"))
    if pre == "div":
        assert mf.mem_footprint == float(g["mem_div_rf"])
    y = mf.spmv(g["x"], np.full(mf.m, 1.0))
    gold, absy = orc.csr_gold(g["row_ptr"], g["col_ind"], g["values"], g["x"])
    assert rel_row_error(y, g["y_csr_naive"], absy) <= TOL
    ref_y = g["y_div_rf" if pre == "div" else "y_div_rf_1000"]
    assert rel_row_error(y, ref_y, absy) <= TOL


@pytest.mark.parametrize("name", ["gen_gamma_skew_2000", "dup_values_700", "long_dup_row_40", "empty_rows_333"])
@pytest.mark.parametrize("L,pv,threads", [(32, 2048, 8), (32, 512, 1), (8, 777, 5), (1, 100, 3)])
def test_div_rf_other_lane_counts(sb, orc, name, L, pv, threads):
    """GPU-native settings (32 lanes, smaller packets): bytes equal the restatement's and
    decode back to the input matrix (the reference's self-check, div.cpp:515-603)."""
    g = load_golden(name)
    rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
    mf = _mk(sb, g, "div_rf", num_threads=threads, vec_len=L, div_packet_vals=pv)
    data = mf.export("div_data")
    d = orc.div_convert(rp, ci, v, int(g["n"]), threads, L, pv, 0.0)
    assert np.array_equal(data, d["data"])
    assert np.array_equal(mf.export("div_groups"), d["group_pos"])
    nnz = int(rp[-1])
    r, c, val = orc.div_decode_coo(data, L, nnz)
    order = np.lexsort((c, r))
    assert np.array_equal(r[order], np.repeat(np.arange(rp.size - 1), np.diff(rp)))
    assert np.array_equal(c[order], ci)
    assert np.array_equal(val[order].view(np.uint64), v.view(np.uint64))
    y = mf.spmv(x, np.full(mf.m, 1.0))
    gold, absy = orc.csr_gold(rp, ci, v, x)
    assert rel_row_error(y, gold, absy) <= TOL
    # without the decoders' L1 prefetch of the coordinates
    y1 = _mk(sb, g, "div_rf", num_threads=threads, vec_len=L, div_packet_vals=pv, stages=1).spmv(x, np.full(mf.m, 1.0))
    assert rel_row_error(y1, gold, absy) <= TOL


@pytest.mark.parametrize("pv,threads", [(16384, 8), (4096, 8), (1000, 3), (64, 1)])
def test_div_rf_warp_decoder(sb, orc, pv, threads):
    """The 32-lane warp decoder (kernel 2: one warp per packet, one lane per lane stream)
    against the CTA decoder (kernel 0) on the same packets and against binary128 row sums,
    on every golden case (repeated values: rf > 1 groups; empty rows; long rows split over
    packets) and twice in a row (split rows are zeroed before each run)."""
    for name in golden_names():
        g = load_golden(name)
        rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
        gold, absy = orc.csr_gold(rp, ci, v, x)
        ys = {}
        # the warp decoder with its L1 prefetch (default, and 16 positions ahead) and without it
        # (and the form held to 64 registers, ctas_per_sm 4)
        for kernel, st, pd, cps in ((0, 0, 0, 0), (2, 0, 0, 0), (2, 1, 0, 0), (2, 0, 16, 0), (2, 0, 0, 4), (2, 4, 0, 0)):
            mf = _mk(sb, g, "div_rf", num_threads=threads, vec_len=32, div_packet_vals=pv, kernel=kernel, stages=st,
                     block_nnz=pd, ctas_per_sm=cps)
            for _ in range(2):
                ys[kernel, st, pd] = mf.spmv(x, np.full(mf.m, 1.0))
            assert rel_row_error(ys[kernel, st, pd], gold, absy) <= TOL, (name, pv, kernel, st, pd, cps)
        assert rel_row_error(ys[2, 0, 0], ys[0, 0, 0], absy) <= TOL
    with pytest.raises(sb.SpmvError):
        _mk(sb, load_golden("hand6"), "div_rf", vec_len=4, kernel=2)


@pytest.mark.parametrize("pv,threads,L", [(16384, 8, 4), (1000, 8, 4), (64, 3, 4), (512, 5, 32)])
def test_div_rf_packet_reordering_matches_reference(sb, orc, pv, threads, L, monkeypatch):
    """DIV_PACKET_REORDERING=1 (div.cpp:377-395, :455-498): packet bytes and packet-group
    offsets bit for bit against the reference compiled from its sources, with the same
    setting, on every golden case (small packets: many groups per thread, long rows split
    across packets, equal medians); y within 1e-12 and equal to the unordered layout's."""
    if not orc.ref_available("div_rf"):
        pytest.fail("the compiled reference for div_rf is missing (make -C oracle ref)")
    monkeypatch.setenv("DIV_PACKET_REORDERING", "1")
    monkeypatch.setenv("CSRCV_NUM_PACKET_VALS", str(pv))
    for name in golden_names():
        g = load_golden(name)
        rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
        continue_ref = L == 4        # the reference's x86 build has VEC_LEN = 4
        mf = _mk(sb, g, "div_rf", num_threads=threads, vec_len=L, div_packet_vals=pv, div_packet_reordering=1)
        if continue_ref:
            R = orc.RefFormat("div_rf", rp, ci, v, n=int(g["n"]), threads=threads)
            try:
                a = R.div_arrays()
            finally:
                R.close()
            assert np.array_equal(mf.export("div_data"), orc.div_zero_header_padding(a["data"], L)), name
            assert np.array_equal(mf.export("div_groups"), a["group_pos"]), name
        y = mf.spmv(x, np.full(mf.m, 1.0))
        gold, absy = orc.csr_gold(rp, ci, v, x)
        assert rel_row_error(y, gold, absy) <= TOL
        plain = _mk(sb, g, "div_rf", num_threads=threads, vec_len=L, div_packet_vals=pv)
        assert plain.export("div_data").size == mf.export("div_data").size
        assert rel_row_error(plain.spmv(x, np.full(mf.m, 1.0)), y, absy) <= TOL


def test_div_rf_reordering_normal100k(sb, orc, monkeypatch):
    """The 100k-row configuration with reordering, against the compiled reference."""
    if not orc.ref_available("div_rf"):
        pytest.fail("the compiled reference for div_rf is missing (make -C oracle ref)")
    monkeypatch.setenv("DIV_PACKET_REORDERING", "1")
    monkeypatch.setenv("CSRCV_NUM_PACKET_VALS", "16384")
    gm = sb.generate_artificial(100000, 100000, 10, 2, "normal", "random", 0.3, 0, 1.0, 0.5, 14)
    rp, ci, v = gm.row_ptr, gm.col_ind, 2.0 * gm.values - 1.0
    mf = sb.csr_to_format(rp, ci, v, format="div_rf", div_packet_reordering=1)
    R = orc.RefFormat("div_rf", rp, ci, v, threads=T)
    try:
        a = R.div_arrays()
    finally:
        R.close()
    assert np.array_equal(mf.export("div_data"), orc.div_zero_header_padding(a["data"], V))
    assert np.array_equal(mf.export("div_groups"), a["group_pos"])


@pytest.mark.parametrize("tol", [1e-6, 1e-3])
def test_div_rf_lossy_values(sb, orc, tol):
    """DIV_VC_TOLERANCE: rounded values, same bytes as the restatement, relative value
    error within the tolerance."""
    g = load_golden("gen_diag_1500")
    rp, ci, v, x = g["row_ptr"], g["col_ind"], g["values"], g["x"]
    mf = _mk(sb, g, "div_rf", div_tolerance=tol)
    d = orc.div_convert(rp, ci, v, int(g["n"]), T, V, 16384, tol)
    assert np.array_equal(mf.export("div_data"), d["data"])
    r, c, val = orc.div_decode_coo(d["data"], V, int(rp[-1]))
    order = np.lexsort((c, r))
    rel = np.abs(val[order] - v) / np.maximum(np.abs(v), 1e-300)
    assert rel.max() <= tol
