"""Shared fixtures of the test suite.

Markers: tests marked ``gpu`` need a CUDA device (run with ``-m gpu`` on a B200); every
other test runs on the CPU (``-m "not gpu"``).
"""
from __future__ import annotations

import glob
import hashlib
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_package():
    """Imports the package directory spmv-dare_b200/ as module `spmv_dare_b200`."""
    if "spmv_dare_b200" in sys.modules:
        return sys.modules["spmv_dare_b200"]
    pkg = os.path.join(ROOT, "spmv-dare_b200")
    spec = importlib.util.spec_from_file_location("spmv_dare_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["spmv_dare_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def sb():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    return oracle


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


_golden_cache = {}


def load_golden(name):
    if name not in _golden_cache:
        with np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False) as z:
            _golden_cache[name] = {k: z[k] for k in z.files}
    return _golden_cache[name]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def assert_golden_array(g, key, actual):
    """Compares an array bit for bit with a golden array (stored in full or as a digest)."""
    actual = np.ascontiguousarray(actual)
    if key in g:
        exp = g[key]
        assert actual.shape == exp.shape, f"{key}: shape {actual.shape} != {exp.shape}"
        if exp.dtype.kind == "f":
            bad = np.flatnonzero(actual.view(np.uint64 if exp.itemsize == 8 else np.uint32) !=
                                 exp.view(np.uint64 if exp.itemsize == 8 else np.uint32))
        else:
            bad = np.flatnonzero(actual != exp.astype(actual.dtype))
        assert bad.size == 0, f"{key}: {bad.size} entries differ, first at {bad[:5]}"
    else:
        assert ("sha256_" + key) in g, f"golden has no {key}"
        assert actual.size == int(g["size_" + key]), f"{key}: size {actual.size} != {int(g['size_' + key])}"
        assert digest(actual) == str(g["sha256_" + key]), f"{key}: content digest differs"


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def rel_row_error(y, y_ref, absy):
    """max_i |y_i - y_ref_i| / max(|y_ref_i|, sum_j |a_ij x_j|): the condition-aware per-row
    relative error used for every tolerance test (0 where both are 0)."""
    den = np.maximum(np.abs(y_ref), absy)
    num = np.abs(y - y_ref)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(den > 0, num / np.where(den > 0, den, 1), np.where(num > 0, np.inf, 0))
    return float(r.max()) if r.size else 0.0
