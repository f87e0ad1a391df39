"""bench.py --impl reference (the reference's own csr_naive, compiled from its sources, on the
host cores) prints one JSON line of the bench contract; run here on a 20k-row instance of
the 4M-row matrix's generator parameters."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_prints_the_contract_line():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_csr_naive.so")):
        pytest.skip("reference build (oracle/_ref) not present")
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--rows", "20000", "--steps", "3",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-1500:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "GB/s" and d["value"] > 0 and d["steps"] == 3
    assert d["n_gpus"] == 1 and d["higher_is_better"] is True and d["dtype"] == "f64"
    assert d["config"]["m"] == 20000 and d["config"]["format"] == "csr_naive"
    assert set(d["config"]) == {"workload", "format", "m", "n", "nnz", "bytes_per_spmv", "l2", "parallelism",
                                "format_params"}
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert "20000-row" in d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun with N > 1 only rank 0 runs and prints; the others exit 0 at once."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--rows", "20000", "--steps", "3",
                        "--warmup", "3", "--gpus", "2"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-1500:]
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]


def test_bench_bytes_and_workload_names():
    """Algorithmic bytes of one SpMV on the 4M-row matrix (csr_mem_footprint + x + y) and of
    the FP32 variant; workload names carry no configuration numbering."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.algorithmic_bytes(4000000, 4000000, 80469735) == 1045636824
    assert bench.algorithmic_bytes(100000, 100000, 999475) == 13993704
    assert 80469735 * 8 + 4000001 * 4 + 4000000 * 4 + 4000000 * 4 == 691757884
    assert "4Mx4M" in bench.WORKLOAD and "config" not in bench.WORKLOAD.lower()
    assert bench.batch_workload(128).startswith("batch: 128 artificial matrices, seeds 1000-1127")
