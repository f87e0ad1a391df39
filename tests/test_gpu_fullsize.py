"""Full-size parity on the benchmark configurations (config 1: 100k rows, nnz 999,475;
config 2: 4M rows, nnz 80,469,735), generated by the native generator (itself pinned on
the reference generator) with values mapped v -> 2v - 1 and x ~ U[-1, 1).

Against the oracle restatement (which is pinned on the reference): y bit-identical per
format, converted arrays bit-identical; against binary128 row sums: within 1e-12.
"""
import numpy as np
import pytest

from conftest import rel_row_error

pytestmark = pytest.mark.gpu

TOL = 1e-12
T, V = 8, 4
CONFIGS = {
    "config1": (100000, 100000, 10, 2, "normal", "random", 0.3, 0, 1.0, 0.5, 14),
    "config2": (4000000, 4000000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7),
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


@pytest.mark.parametrize("cfg", ["config1", "config2"])
def test_csr_naive_fullsize(sb, orc, cfg):
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format="csr_naive")
    assert mf.nnz == {"config1": 999475, "config2": 80469735}[cfg]
    y = mf.spmv(x)
    assert np.array_equal(_bits(y), _bits(orc.csr_spmv(rp, ci, v, x)))
    gold, absy = orc.csr_gold(rp, ci, v, x)
    assert rel_row_error(y, gold, absy) <= TOL


@pytest.mark.parametrize("cfg,C,sigma", [("config1", 32, 256), ("config2", 32, 512)])
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
def test_other_formats_config1(sb, orc, fmt):
    rp, ci, v, x = matrix(sb, "config1")
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
def test_other_formats_config2_properties(sb, orc, fmt):
    """Config 2 at full size: y bit-identical to the restatement for csr_vec; for the SELL
    pair the layout invariants (pointer monotone, every nnz stored once) and y within the
    tolerance of the binary128 sums."""
    rp, ci, v, x = matrix(sb, "config2")
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


@pytest.mark.parametrize("cfg", ["config1", "config2"])
def test_div_rf_fullsize(sb, orc, cfg):
    """Config 1: packet bytes identical to the restatement (itself pinned on the reference
    at this size); config 2: decode round trip of every packet and y within tolerance."""
    rp, ci, v, x = matrix(sb, cfg)
    mf = sb.csr_to_format(rp, ci, v, format="div_rf")
    data = mf.export("div_data")
    if cfg == "config1":
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
