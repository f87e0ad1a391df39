"""Full-size parity on the benchmark matrices (normal100k: 100k rows, nnz 999,475;
gamma4m: 4M rows, nnz 80,469,735), generated by the native generator (itself pinned on
the reference generator) with values mapped v -> 2v - 1 and x ~ U[-1, 1).

Against the reference compiled from its own sources (oracle/_ref, the reference's
csr_to_format + Matrix_Format::spmv of each format, T = 8 threads): every converted array
and every y bit-identical at both sizes.  SELL-C-sigma's RVV kernel cannot run on x86, so
its y is compared with the oracle restatement (its arrays with the compiled reference
conversion).  Against binary128 row sums: within 1e-12.
"""
import numpy as np
import pytest

from conftest import rel_row_error

pytestmark = pytest.mark.gpu

TOL = 1e-12
T, V = 8, 4
CONFIGS = {
    "normal100k": (100000, 100000, 10, 2, "normal", "random", 0.3, 0, 1.0, 0.5, 14),
    "gamma4m": (4000000, 4000000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7),
}
_cache = {}


def matrix(sb, name):
    if name not in _cache:
        g = sb.generate_artificial(*CONFIGS[name])
        v = 2.0 * g.values - 1.0
        x = np.random.default_rng(12345).uniform(-1.0, 1.0, g.m)
        _cache[name] = (g.row_ptr, g.col_ind, v, x)
    return _cache[name]


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("cfg", ["normal100k", "gamma4m"])
def test_csr_naive_fullsize(sb, orc, cfg):
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format="csr_naive")
    assert mf.nnz == {"normal100k": 999475, "gamma4m": 80469735}[cfg]
    y = mf.spmv(x)
    assert np.array_equal(_bits(y), _bits(orc.csr_spmv(rp, ci, v, x)))
    gold, absy = orc.csr_gold(rp, ci, v, x)
    assert rel_row_error(y, gold, absy) <= TOL


@pytest.mark.parametrize("cfg", ["normal100k", "gamma4m"])
def test_csr_naive_packed_columns_fullsize(sb, orc, cfg):
    """csr_naive with packed columns, FP64 and the FP32 variant: the same y bits as the
    plain columns at both sizes."""
    rp, ci, v, x = matrix(sb, cfg)
    y = sb.csr_to_format(rp, ci, v, format="csr_naive", pack_cols=1).spmv(x)
    assert np.array_equal(_bits(y), _bits(orc.csr_spmv(rp, ci, v, x)))
    x32 = x.astype(np.float32)
    y32p = sb.csr_to_format(rp, ci, v, format="csr_naive", value_type="f32", pack_cols=1).spmv(x32)
    y32 = sb.csr_to_format(rp, ci, v, format="csr_naive", value_type="f32").spmv(x32)
    assert np.array_equal(y32p.view(np.uint32), y32.view(np.uint32))


@pytest.mark.parametrize("cfg,C,sigma", [("normal100k", 32, 256), ("gamma4m", 32, 512)])
def test_sellcs_fullsize(sb, orc, cfg, C, sigma):
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format="sell_c_s", sellcs_c=C, sellcs_sigma=sigma)
    arr = orc.sellcs_convert(rp, ci, v, C, sigma)
    assert np.array_equal(mf.export("row_order"), arr["row_order"])
    assert np.array_equal(mf.export("slice_pointers"), arr["slice_pointers"])
    assert np.array_equal(mf.export("column_indices"), arr["column_indices"])
    assert np.array_equal(_bits(mf.export("sellcs_values")), _bits(arr["values"]))
    y = mf.spmv(x)
    assert np.array_equal(_bits(y), _bits(orc.sellcs_spmv(arr, mf.m, C, x)))


@pytest.mark.parametrize("fmt", ["csr_vec", "sell", "sell_sorted"])
def test_other_formats_normal100k(sb, orc, fmt):
    rp, ci, v, x = matrix(sb, "normal100k")
    mf = sb.csr_to_format(rp, ci, v, format=fmt)
    y = mf.spmv(x)
    if fmt == "csr_vec":
        ref = orc.csr_vec_spmv(rp, ci, v, x, V)
    else:
        conv = orc.sell_convert if fmt == "sell" else orc.sell_sorted_convert
        arr = conv(rp, ci, v, V, T)
        for k in arr:
            assert np.array_equal(np.ascontiguousarray(mf.export(k)).view(np.uint8),
                                  np.ascontiguousarray(arr[k]).view(np.uint8)), k
        ref = (orc.sell_spmv if fmt == "sell" else orc.sell_sorted_spmv)(arr, mf.m, V, x)
    assert np.array_equal(_bits(y), _bits(ref))


@pytest.mark.parametrize("fmt", ["sell", "sell_sorted", "csr_vec"])
def test_other_formats_gamma4m_properties(sb, orc, fmt):
    """Config 2 at full size: y bit-identical to the restatement for csr_vec; for the SELL
    pair the layout invariants (pointer monotone, every nnz stored once) and y within the
    tolerance of the binary128 sums."""
    rp, ci, v, x = matrix(sb, "gamma4m")
    mf = sb.csr_to_format(rp, ci, v, format=fmt)
    y = mf.spmv(x)
    gold, absy = orc.csr_gold(rp, ci, v, x)
    assert rel_row_error(y, gold, absy) <= TOL
    if fmt == "csr_vec":
        assert np.array_equal(_bits(y), _bits(orc.csr_vec_spmv(rp, ci, v, x, V)))
    else:
        rcp = mf.export("row_cluster_ptr")
        assert np.all(np.diff(rcp) >= 0) and int(rcp[-1]) == mf.stored_elems
        a = mf.export("a")
        assert np.count_nonzero(a) == np.count_nonzero(v)
        assert np.isclose(np.sum(np.abs(a)), np.sum(np.abs(v)), rtol=1e-12)


def _need_ref(orc, fmt):
    if not orc.ref_available(fmt):
        pytest.fail(f"the compiled reference for {fmt} is missing (make -C oracle ref)")


@pytest.mark.parametrize("cfg", ["normal100k", "gamma4m"])
@pytest.mark.parametrize("fmt", ["csr_naive", "csr_vec", "sell", "sell_sorted"])
def test_against_compiled_reference(sb, orc, cfg, fmt):
    """Converted arrays (row_cluster_ptr, ja, a, thread ranges, permutations) and y bit for
    bit against the reference's own csr_to_format + spmv (csr.cpp, csr_vec.cpp,
    sell.cpp:95-280, sell_sorted.cpp:119-427), y probed with the bench's m + 64 buffer of
    ones (bench_spmv.cpp:561-564)."""
    _need_ref(orc, fmt)
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format=fmt)
    y = mf.spmv(x, np.full(mf.m, 1.0))
    R = orc.RefFormat(fmt, rp, ci, v, threads=T)
    try:
        y_ref = R.spmv(x)[:mf.m]
        if fmt in ("sell", "sell_sorted"):
            for k, a in R.sell_arrays().items():
                got = np.ascontiguousarray(mf.export(k))
                assert got.dtype == a.dtype and np.array_equal(got.view(np.uint8), a.view(np.uint8)), k
        assert mf.mem_footprint == R.mem_footprint
    finally:
        R.close()
    bad = np.flatnonzero(_bits(y) != _bits(y_ref))
    assert bad.size == 0, f"{bad.size} rows differ from the reference, first {bad[:5]}"


@pytest.mark.parametrize("cfg,C,sigma", [("normal100k", 32, 256), ("gamma4m", 32, 512)])
def test_sellcs_arrays_against_compiled_reference(sb, orc, cfg, C, sigma):
    """SELL-C-sigma conversion against the reference's own sellcs_format.c / radix_sort.c
    (get_order_by_row_size, csr_to_sellcs), compiled from its sources."""
    _need_ref(orc, "sellcs")
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format="sell_c_s", sellcs_c=C, sellcs_sigma=sigma)
    ref = orc.ref_sellcs_convert(rp, ci, v, C, sigma)
    names = {"row_order": "row_order", "slice_widths": "slice_widths", "slice_pointers": "slice_pointers",
             "column_indices": "column_indices", "values": "sellcs_values"}
    for k, a in ref.items():
        got = mf.export(names[k])
        if k == "values":
            assert np.array_equal(_bits(got), _bits(a)), k
        else:
            assert np.array_equal(got.astype(np.int64), a.astype(np.int64)), k


@pytest.mark.parametrize("cfg", ["normal100k", "gamma4m"])
def test_div_rf_against_compiled_reference(sb, orc, cfg):
    """DIV-RF packet bytes and packet-group offsets bit for bit against the reference's
    own compress_kernel_div (div.cpp:236-604, div_kernels_rf.h:538-919) at T = 8, L = 4,
    16384 values a packet; y within 1e-12 of the reference's decoder (its sums run in
    value-sorted order, as do ours, but the partial sums of split rows combine
    differently)."""
    _need_ref(orc, "div_rf")
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format="div_rf")
    data, groups = mf.export("div_data"), mf.export("div_groups")
    y = mf.spmv(x, np.full(mf.m, 1.0))
    R = orc.RefFormat("div_rf", rp, ci, v, threads=T)
    try:
        a = R.div_arrays()
        y_ref = R.spmv(x)[:mf.m]
    finally:
        R.close()
    assert np.array_equal(mf.export("div_thread_bytes"), a["thread_bytes"])
    ref_data = orc.div_zero_header_padding(a["data"], V)
    bad = np.flatnonzero(data != ref_data)
    assert data.size == ref_data.size and bad.size == 0, f"{bad.size} packet bytes differ, first {bad[:5]}"
    assert np.array_equal(groups, a["group_pos"])
    gold, absy = orc.csr_gold(rp, ci, v, x)
    assert rel_row_error(y, y_ref, absy) <= TOL
    assert rel_row_error(y, gold, absy) <= TOL


@pytest.mark.parametrize("cfg", ["normal100k", "gamma4m"])
def test_div_rf_fullsize(sb, orc, cfg):
    """Config 1: packet bytes identical to the restatement (itself pinned on the reference
    at this size); gamma4m: decode round trip of every packet and y within tolerance."""
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format="div_rf")
    data = mf.export("div_data")
    if cfg == "normal100k":
        d = orc.div_convert(rp, ci, v, mf.n, T, V, 16384, 0.0)
        assert np.array_equal(data, d["data"])
        assert np.array_equal(mf.export("div_groups"), d["group_pos"])
    else:
        r, c, val = orc.div_decode_coo(data, V, mf.nnz)
        order = np.lexsort((c, r))
        assert np.array_equal(r[order], np.repeat(np.arange(mf.m, dtype=np.int32), np.diff(rp)))
        assert np.array_equal(c[order], ci)
        assert np.array_equal(val[order].view(np.uint64), v.view(np.uint64))
    y = mf.spmv(x)
    gold, absy = orc.csr_gold(rp, ci, v, x)
    assert rel_row_error(y, gold, absy) <= TOL
