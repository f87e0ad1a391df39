"""The C-ABI library loads and exports every entry point include/spmv_b200.h declares;
host-side argument handling (no GPU compute)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "spmv_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(spmv_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = _declared_functions()
    for must in ["spmv_create", "spmv_run", "spmv_run_device", "spmv_destroy", "spmv_export", "spmv_get_info",
                 "spmv_last_error", "spmv_format_desc_init", "spmv_artgen_create"]:
        assert must in names


def test_library_exports_every_declared_symbol(sb):
    lib = sb.library()
    for name in _declared_functions():
        assert hasattr(lib, name), f"{name} declared in include/spmv_b200.h but not exported"


def test_python_bindings_cover_the_header(sb):
    from spmv_dare_b200 import _capi

    assert set(_declared_functions()) <= set(_capi.SIGNATURES)


def test_desc_defaults_are_the_reference_defaults(sb):
    d = sb.format_defaults("div_rf")
    assert d["num_threads"] == 8 and d["vec_len"] == 4 and d["div_packet_vals"] == 16384
    assert d["div_tolerance"] == 0.0 and d["exact"] == 1
    d = sb.format_defaults("sell_c_s")
    assert (d["sellcs_c"], d["sellcs_sigma"]) == (32, 512)


def test_symmetric_unexpanded_is_rejected(sb):
    rp = np.array([0, 1], np.int32)
    with pytest.raises(sb.SpmvError) as e:
        sb.csr_to_format(rp, np.array([0], np.int32), np.array([1.0]), 1, 1, 1, symmetric=1, symmetry_expanded=0)
    assert e.value.status == 5


@pytest.mark.parametrize("params,status", [
    (dict(format="sell_c_s", sellcs_c=48), 1),
    (dict(format="sell_c_s", sellcs_c=32, sellcs_sigma=100), 1),
    (dict(format="csr_vec", vec_len=3), 1),
    (dict(format="div_rf", div_tolerance=1.5), 1),
    (dict(format="csr_naive", num_threads=0), 1),
    (dict(format="csr_naive", kernel=7), 1),                      # the segmented kernel is FP32 only
    (dict(format="csr_naive", kernel=8, value_type="f32"), 1),    # the tiled kernels are FP64 only
    (dict(format="csr_naive", kernel=9, value_type="f32"), 1),
    (dict(format="sell_c_s", kernel=11), 1),
    (dict(format="sell_c_s", kernel=10, value_type="f32"), 1),   # kernel 10 is FP64 slices
    (dict(format="csr_naive", wait_limit_us=-5), 1),
    (dict(format="csr_naive", debug_flags=4), 1),
    (dict(format="csr_naive", row_assign=2, value_type="f32"), 1),
    (dict(format="csr_naive", row_assign=1), 1),                 # FP32 variant only
])
def test_invalid_parameters_are_rejected_before_any_device_work(sb, params, status):
    rp = np.array([0, 1], np.int32)
    with pytest.raises(sb.SpmvError) as e:
        sb.csr_to_format(rp, np.array([0], np.int32), np.array([1.0]), 1, 1, 1, **params)
    assert e.value.status == status


def test_no_device_reports_status_not_fallback(sb):
    if has_gpu():
        pytest.skip("a GPU is present")
    rp = np.array([0, 1], np.int32)
    with pytest.raises(sb.SpmvError) as e:
        sb.csr_to_format(rp, np.array([0], np.int32), np.array([1.0]), 1, 1, 1)
    assert e.value.status in (3, 8)


def test_statistics_labels(sb):
    assert sb.statistics_print_labels().startswith(",gpu_format")


def test_struct_sizes_match_the_binding(sb):
    """The library's spmv_format_desc / spmv_info are the binding's (checked at load too)."""
    import ctypes

    from spmv_dare_b200 import _capi

    L = sb.library()
    assert L.spmv_format_desc_size() == ctypes.sizeof(_capi.FormatDesc)
    assert L.spmv_info_size() == ctypes.sizeof(_capi.Info)


def test_dropin_executable_is_built_against_this_header(tmp_path):
    """The drop-in driver checks its structs against the library before any GPU work: without
    a GPU it stops at the device, not at a header mismatch."""
    import os
    import subprocess

    from conftest import ROOT

    exe = os.path.join(ROOT, "spmv-dare_b200", "plugin", "_build", "dropin_check_csr_naive_d.exe")
    if not os.path.exists(exe):
        pytest.skip("drop-in executables not built (make -C spmv-dare_b200/plugin REF=...)")
    if has_gpu():
        pytest.skip("a GPU is present (the GPU tests run the driver)")
    with open(tmp_path / "a.bin", "wb") as f:
        np.array([2, 2, 2], np.int64).tofile(f)
        np.array([0, 1, 2], np.int32).tofile(f)
        np.array([0, 1], np.int32).tofile(f)
        np.array([1.0, 2.0]).tofile(f)
    np.array([1.0, 1.0]).tofile(tmp_path / "x.bin")
    p = subprocess.run([exe, str(tmp_path / "a.bin"), str(tmp_path / "x.bin"), str(tmp_path / "y.bin")],
                       capture_output=True, text=True, timeout=120)
    out = p.stdout + p.stderr
    assert p.returncode != 0 and "header and library differ" not in out
    assert "spmv_b200:" in out and "device" in out.lower(), out[-500:]
