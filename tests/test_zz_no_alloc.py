"""Allocation-free entry point spmv_run_device_mixed_noalloc, called through the C ABI.

It serves callers that cannot let the library call cudaMalloc (a host program that owns
all device memory through its own pool, or a loop that cannot take the synchronisation an
allocation may cause).  Its scratch (x rounded to FP32, the FP32 y) lives in a static
device array instead of the handle's lazily allocated buffers; everything else is the FP32
Dot2 path that spmv_run takes with FP64 buffers.  Bar: y bit-identical to spmv_run on the
same handle (tolerance 0 ulp), for two calls in a row with different x, so a stale array
would show; with the default kernel and with the segmented kernel 7 (which zeroes empty
rows from a list and merges rows across chunks into y), on matrices with empty rows.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

ULP_TOL = 0   # same arithmetic as spmv_run on an FP32 handle: bit-identical


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream or 1   # 1 = cudaStreamLegacy


def _noalloc(lib, mf, xd, yd):
    import torch

    st = lib.spmv_run_device_mixed_noalloc(mf.handle, xd.data_ptr(), yd.data_ptr(), _stream())
    torch.cuda.synchronize()
    return st


def _ulps(a, b):
    return int(np.max(np.abs(a.view(np.int64) - b.view(np.int64)), initial=0))


@pytest.mark.parametrize("kernel", [-1, 7])
@pytest.mark.parametrize("name", ["gen_gamma_skew_2000", "long_rows_60", "dup_values_700", "empty_rows_333"])
def test_noalloc_matches_spmv_run_twice(sb, name, kernel):
    import torch

    g = load_golden(name)
    rp, ci, v = g["row_ptr"], g["col_ind"], g["values"]
    m, n = rp.size - 1, g["x"].size
    assert m + n <= sb._capi.NOALLOC_MAX_ELEMS
    mf = sb.csr_to_format(rp, ci, v, m, n, int(rp[-1]), format="csr_naive", value_type="f32", kernel=kernel)
    lib = sb.library()
    rng = np.random.default_rng(77)
    for call in range(2):
        x = g["x"] if call == 0 else rng.uniform(-1.0, 1.0, n)
        ref = mf.spmv(x, np.full(m, 1.0))                     # existing entry: spmv_run
        xd = torch.from_numpy(x).cuda()
        yd = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
        assert _noalloc(lib, mf, xd, yd) == 0, lib.spmv_last_error()
        assert lib.spmv_sync(mf.handle) == 0
        assert _ulps(yd.cpu().numpy(), ref) <= ULP_TOL, f"call {call}"


def test_noalloc_rejects_oversize_and_f64(sb):
    import torch

    lib = sb.library()
    cap = sb._capi.NOALLOC_MAX_ELEMS
    m = cap // 2 + 1                          # n + m = cap + 2 > cap
    rp = np.arange(m + 1, dtype=np.int32)
    ci = np.arange(m, dtype=np.int32)
    v = np.ones(m)
    big = sb.csr_to_format(rp, ci, v, m, m, m, format="csr_naive", value_type="f32")
    xd = torch.zeros(m, dtype=torch.float64, device="cuda")
    yd = torch.zeros(m, dtype=torch.float64, device="cuda")
    st = _noalloc(lib, big, xd, yd)
    assert st == sb._capi.SPMV_ERR_ARG and b"exceeds" in lib.spmv_last_error()
    f64 = sb.csr_to_format(rp[:101], ci[:100], v[:100], 100, 100, 100, format="csr_naive")
    assert _noalloc(lib, f64, xd, yd) == sb._capi.SPMV_ERR_ARG
    # a rejected call launched nothing: the last valid call's result still stands
    g = load_golden("gen_gamma_skew_2000")
    mf = sb.csr_to_format(g["row_ptr"], g["col_ind"], g["values"], format="csr_naive", value_type="f32")
    x = g["x"]
    xd2 = torch.from_numpy(x).cuda()
    yd2 = torch.empty(mf.m, dtype=torch.float64, device="cuda")
    assert _noalloc(lib, mf, xd2, yd2) == 0
    assert _ulps(yd2.cpu().numpy(), mf.spmv(x, np.full(mf.m, 1.0))) <= ULP_TOL


def test_noalloc_takes_no_device_memory(sb):
    """After the first call on the device (which resolves the static array's address),
    further calls leave the device's free memory unchanged."""
    import torch

    g = load_golden("gen_gamma_skew_2000")
    mf = sb.csr_to_format(g["row_ptr"], g["col_ind"], g["values"], format="csr_naive", value_type="f32")
    lib = sb.library()
    xd = torch.from_numpy(g["x"]).cuda()
    yd = torch.empty(mf.m, dtype=torch.float64, device="cuda")
    assert _noalloc(lib, mf, xd, yd) == 0
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _noalloc(lib, mf, xd, yd) == 0
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_other_current_device(sb):
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    g = load_golden("gen_gamma_skew_2000")
    with torch.cuda.device(0):
        mf = sb.csr_to_format(g["row_ptr"], g["col_ind"], g["values"], format="csr_naive", value_type="f32")
    with torch.cuda.device(1):
        xd = torch.from_numpy(g["x"]).cuda()
        yd = torch.empty(mf.m, dtype=torch.float64, device="cuda")
        st = sb.library().spmv_run_device_mixed_noalloc(mf.handle, xd.data_ptr(), yd.data_ptr(), 1)
    assert st == sb._capi.SPMV_ERR_ARG
