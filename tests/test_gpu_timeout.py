"""Bounded device waits, exercised without a fault.

A handle created with debug_flags = SPMV_DEBUG_WITHHOLD_HANDOFF runs the warp-specialised
kernels (4, 8 and the FP32 default) with gather warps that never hand a stage to the row
warps: the row warps' wait on the hand-off runs out after wait_limit_us, they record the
timeout, their issuing thread waits for the bulk copies it has in flight, and every warp
leaves.  Nothing is faulted: every copy still lands, no barrier waits on a thread that
left, and the CUDA context stays usable.  The test checks that spmv_sync() then reports
SPMV_ERR_TIMEOUT and that a fresh handle on the same matrix gives the reference's y.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPMV_ERR_TIMEOUT = 6
WITHHOLD = 1
WAIT_US = 2000


def _matrix(sb):
    g = sb.generate_artificial(50000, 50000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7)
    x = np.random.default_rng(4).uniform(-1, 1, g.m)
    return g.row_ptr, g.col_ind, 2.0 * g.values - 1.0, x


@pytest.mark.parametrize("fmt,kw", [
    ("csr_naive", {}),                                  # kernel 4, the csr_naive default
    ("csr_vec", {}),                                    # kernel 4, FMA lanes
    ("sell_c_s", dict(sellcs_c=32, sellcs_sigma=512, kernel=8)),  # kernel 8 over tiled columns
    ("csr_naive", dict(value_type="f32")),              # the FP32 warp-specialised kernel
])
def test_withheld_handoff_times_out_then_fresh_handle_is_exact(sb, orc, fmt, kw):
    import time

    rp, ci, v, x = _matrix(sb)
    held = sb.csr_to_format(rp, ci, v, format=fmt, wait_limit_us=WAIT_US, debug_flags=WITHHOLD, **kw)
    t0 = time.perf_counter()
    with pytest.raises(sb.SpmvError) as e:
        held.spmv(x)
    assert e.value.status == SPMV_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 5.0            # a few wait limits, not the 2 s default
    with pytest.raises(sb.SpmvError) as e:             # the error word is sticky on its handle
        held.sync()
    assert e.value.status == SPMV_ERR_TIMEOUT
    held.destroy()

    fresh = sb.csr_to_format(rp, ci, v, format=fmt, wait_limit_us=WAIT_US, **kw)
    y = fresh.spmv(x, np.full(fresh.m, 1.0))
    if kw.get("value_type") == "f32":
        v32, x32 = v.astype(np.float32), x.astype(np.float32)
        ref = orc.csr_f32_dot2(rp, ci, v32, x32).astype(np.float64)
    elif fmt == "csr_naive":
        ref = orc.csr_spmv(rp, ci, v, x)
    elif fmt == "csr_vec":
        ref = orc.csr_vec_spmv(rp, ci, v, x, 4)
    else:
        ref = orc.sellcs_spmv(orc.sellcs_convert(rp, ci, v, 32, 512), fresh.m, 32, x)
    assert np.array_equal(np.ascontiguousarray(y).view(np.uint64), np.ascontiguousarray(ref).view(np.uint64))
    fresh.sync()


def test_debug_flags_are_validated(sb):
    rp = np.array([0, 1], np.int32)
    with pytest.raises(sb.SpmvError):
        sb.csr_to_format(rp, np.array([0], np.int32), np.array([1.0]), format="csr_naive", debug_flags=2)
    with pytest.raises(sb.SpmvError):
        sb.csr_to_format(rp, np.array([0], np.int32), np.array([1.0]), format="csr_naive", wait_limit_us=-1)
