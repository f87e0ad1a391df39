"""The drop-in: the reference's own bench driver (src/bench.cpp + src/bench_spmv.cpp)
linked with spmv-dare_b200/plugin/gpu_format.cpp runs unchanged on the GPU formats, and
the y that the plugin returns through the reference's Matrix_Format interface
(spmv_kernel.h:17,28) matches the reference format's own y.

The y check drives each plugin through dropin_check.cpp, which makes the bench's calls
with the bench's buffers (pageable aligned_alloc(64) x and y, y of m + 64 elements
pre-filled with 1.0, the CSR arrays overwritten and freed right after csr_to_format,
bench.cpp:622-651, bench_spmv.cpp:546-564).  The reference side is the reference's own
csr_to_format + spmv of the same format, compiled from its sources (oracle/_ref):
bit for bit for csr_naive, csr_vec, sell and sell_sorted; SELL-C-sigma's RVV kernel cannot
run on x86, so its y is compared with the oracle restatement bit for bit; DIV-RF within
1e-12 of the reference's decoder and of binary128 row sums."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_row_error

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "spmv-dare_b200", "plugin", "_build")
ENV = dict(USE_ARTIFICIAL_MATRICES="1", USE_PROCESSES="0", GPU_KERNEL="1", USE_RCM_REORDERING="0", COOLDOWN="0",
           CSRCV_NUM_PACKET_VALS="16384", DIV_VC_TOLERANCE="0", OMP_NUM_THREADS="8")
ARGV = ["100000", "100000", "10", "2", "normal", "random", "0.3", "0", "1.0", "0.5", "14"]
FORMATS = ["csr_naive", "csr_vec", "sell", "sell_sorted", "sell_c_s", "div_rf"]
SENTINEL = np.uint64(0x7ff8dead0000beef)


@pytest.mark.parametrize("fmt", FORMATS)
def test_reference_bench_driver_runs_gpu_format(fmt):
    exe = os.path.join(BUILD, f"spmv_gpu_{fmt}_d.exe")
    if not os.path.exists(exe):
        pytest.skip("drop-in executables not built (make -C spmv-dare_b200/plugin REF=...)")
    env = dict(os.environ, PROGG=f"gpu_{fmt}", **ENV)
    p = subprocess.run([exe] + ARGV, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    m = re.search(r"GFLOPS = ([0-9.]+)", p.stdout)
    assert m and float(m.group(1)) > 0
    assert "_B200" in p.stderr   # the CSV line carries the GPU format name


def _dropin_matrix(sb):
    """A 20k-row gamma / skewed matrix with empty rows, long rows and 50 columns past the
    last row (n > m): the 4M-row matrix's generator parameters at a size the reference runs in
    well under a second, plus a hand-made tail of every edge the formats pad or split."""
    g = sb.generate_artificial(20000, 20000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7)
    rp, ci = g.row_ptr.astype(np.int64), g.col_ind
    v = 2.0 * g.values - 1.0
    rows = np.diff(rp)
    rows[::97] = 0                                    # empty rows scattered through
    keep = np.ones(ci.size, bool)
    for r in range(0, rows.size, 97):
        keep[rp[r]:rp[r + 1]] = False
    ci, v = ci[keep], v[keep]
    rp = np.concatenate([[0], np.cumsum(rows)])
    n = 20050
    long_cols = np.arange(0, n, 3, dtype=np.int32)      # one row of 6,684 entries
    rp = np.concatenate([rp, [rp[-1] + long_cols.size, rp[-1] + long_cols.size]])   # then an empty last row
    ci = np.concatenate([ci, long_cols])
    v = np.concatenate([v, np.random.default_rng(5).uniform(-1, 1, long_cols.size)])
    return rp.astype(np.int32), ci.astype(np.int32), v, n


@pytest.mark.parametrize("fmt", FORMATS)
def test_dropin_y_matches_reference(sb, orc, fmt, tmp_path):
    exe = os.path.join(BUILD, f"dropin_check_{fmt}_d.exe")
    if not os.path.exists(exe):
        pytest.fail("drop-in check executables not built (make -C spmv-dare_b200/plugin REF=...)")
    rp, ci, v, n = _dropin_matrix(sb)
    m, nnz = rp.size - 1, ci.size
    x = np.random.default_rng(11).uniform(-1, 1, n)
    with open(tmp_path / "a.bin", "wb") as f:
        np.array([m, n, nnz], np.int64).tofile(f)
        rp.tofile(f)
        ci.tofile(f)
        v.tofile(f)
    x.tofile(tmp_path / "x.bin")
    env = dict(os.environ, OMP_NUM_THREADS="8", CSRCV_NUM_PACKET_VALS="16384", DIV_VC_TOLERANCE="0")
    p = subprocess.run([exe, str(tmp_path / "a.bin"), str(tmp_path / "x.bin"), str(tmp_path / "y.bin")], env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    yall = np.fromfile(tmp_path / "y.bin", np.float64)
    assert yall.size == m + 64
    assert np.all(yall[m:].view(np.uint64) == SENTINEL), "the plugin wrote past y[m-1]"
    y = yall[:m]
    bits = lambda a: np.ascontiguousarray(a).view(np.uint64)
    if fmt == "sell_c_s":
        y_ref = orc.sellcs_spmv(orc.sellcs_convert(rp, ci, v, 32, 512), m, 32, x)
    else:
        orc_fmt = fmt
        R = orc.RefFormat(orc_fmt, rp, ci, v, n=n, threads=8)
        try:
            y_ref = R.spmv(x)[:m]
            assert f"mem_footprint: {R.mem_footprint:.17g}" in p.stdout
        finally:
            R.close()
    if fmt == "div_rf":
        gold, absy = orc.csr_gold(rp, ci, v, x)
        assert rel_row_error(y, y_ref, absy) <= 1e-12
        assert rel_row_error(y, gold, absy) <= 1e-12
        assert np.all(y[np.diff(rp) == 0] == 0.0)
    else:
        bad = np.flatnonzero(bits(y) != bits(y_ref))
        assert bad.size == 0, f"{fmt}: {bad.size} rows differ from the reference, first {bad[:5]}"
