"""Host logic of the batch autotuner (tuning.batch_plan): an all-csr_naive batch runs as one
block-diagonal SpMV, so the plan keeps csr_naive everywhere unless the matrices' own best
classes save more than the tolerance; and the committed batch database gives that plan."""
import os

import numpy as np

from conftest import ROOT


def _tuning(sb):
    import importlib

    return importlib.import_module("spmv_dare_b200.tuning")


def test_batch_plan_rule(sb):
    T = _tuning(sb)
    nan = np.nan
    t = np.full((3, len(T.CLASSES)), nan)
    t[:, 0] = [1.0, 1.0, 1.0]
    t[:, 13] = [0.9, 1.2, 1.1]                       # one matrix 10% faster in sell: 3.3% overall
    assert list(T.batch_plan(t)) == [0, 0, 0]
    t[:, 13] = [0.5, 0.6, 1.1]                       # 37% overall: each matrix's own best
    assert list(T.batch_plan(t)) == [13, 13, 0]
    t[0, 0] = np.inf                                 # a failed class is never chosen
    assert T.batch_plan(t)[0] == 13


def test_committed_batch_database_plan(sb):
    T = _tuning(sb)
    with np.load(os.path.join(ROOT, "spmv-dare_b200", "data", "tune_batch.npz")) as z:
        times, seeds = z["times_ms"], z["seeds"]
    assert times.shape == (512, len(T.CLASSES)) and seeds[0] == 1000 and seeds[-1] == 1511
    plan = T.batch_plan(times)
    assert np.all(plan == T.DEFAULT_CLASS)
    assert set(np.flatnonzero(~np.isnan(times[0]))) == set(T.BATCHABLE)   # timed (inf: refused)
