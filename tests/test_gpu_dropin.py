"""The drop-in: the reference's own bench driver (src/bench.cpp + src/bench_spmv.cpp)
linked with spmv-dare_b200/plugin/gpu_format.cpp runs unchanged on the GPU formats."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "spmv-dare_b200", "plugin", "_build")
ENV = dict(USE_ARTIFICIAL_MATRICES="1", USE_PROCESSES="0", GPU_KERNEL="1", USE_RCM_REORDERING="0", COOLDOWN="0",
           CSRCV_NUM_PACKET_VALS="16384", DIV_VC_TOLERANCE="0", OMP_NUM_THREADS="8")
ARGV = ["100000", "100000", "10", "2", "normal", "random", "0.3", "0", "1.0", "0.5", "14"]


@pytest.mark.parametrize("fmt", ["csr_naive", "csr_vec", "sell", "sell_sorted", "sell_c_s", "div_rf"])
def test_reference_bench_driver_runs_gpu_format(fmt):
    exe = os.path.join(BUILD, f"spmv_gpu_{fmt}_d.exe")
    if not os.path.exists(exe):
        pytest.skip("drop-in executables not built (make -C spmv-dare_b200/plugin)")
    env = dict(os.environ, PROGG=f"gpu_{fmt}", **ENV)
    p = subprocess.run([exe] + ARGV, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    m = re.search(r"GFLOPS = ([0-9.]+)", p.stdout)
    assert m and float(m.group(1)) > 0
    assert "_B200" in p.stderr   # the CSV line carries the GPU format name
