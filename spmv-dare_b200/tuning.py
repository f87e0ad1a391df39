"""Exhaustive autotuner over the format / parameter classes of the selector.

A class is one format with its parameters: the CSR kernel and its staging geometry, the
lanes of csr_vec, the slice height of sell / sell_sorted, C and sigma of SELL-C-sigma.  For a matrix, every
class is converted on the GPU and timed with CUDA events on the launching stream: warm-up
runs, then `reps` single SpMVs each preceded by an L2 flush (a 256 MB write), median kept.
A class whose conversion fails (e.g. a slice table beyond 32 bits) scores infinity.
The tuning cost of a matrix is the wall time of all conversions and timing runs.
"""
from __future__ import annotations

import statistics
import time

import numpy as np


def _ws(threads, rows, block, stages):
    return {"format": "csr_naive", "kernel": 4, "threads": threads, "block_rows": rows, "block_nnz": block,
            "stages": stages}


def _cta(threads, block):
    return {"format": "csr_naive", "kernel": 0, "threads": threads, "block_nnz": block, "stages": 2}


# 29 classes: the CSR kernel and its staging geometry (threads, row threads, entries per
# block, stages) -- the choice that depends most on the matrix with these kernels -- and
# the other formats with their own parameters (lanes, slice height, C and sigma), each with
# the kernel it is timed with.  New classes are appended, so a database's class indices keep
# their meaning (of the last five only SELL with 32-row slices adds a batch descriptor to
# BATCHABLE, below: the others repeat earlier descriptors, or the batch engine does not run
# the format).
CLASSES = [
    _ws(160, 64, 768, 3),          # the csr_naive default
    _ws(160, 64, 256, 4),
    _ws(160, 64, 512, 3),
    _ws(192, 64, 1024, 3),
    _ws(256, 64, 1536, 3),
    _ws(224, 96, 1024, 3),
    _ws(128, 32, 384, 4),
    _ws(320, 128, 2048, 3),
    _cta(256, 768),
    _cta(128, 256),
    _cta(512, 2048),
    {"format": "csr_vec", "vec_len": 4},
    {"format": "csr_vec", "vec_len": 8},
    {"format": "sell", "vec_len": 4},
    {"format": "sell", "vec_len": 8},
    {"format": "sell_sorted", "vec_len": 4},
    {"format": "sell_c_s", "sellcs_c": 8, "sellcs_sigma": 256, "kernel": 0},
    {"format": "sell_c_s", "sellcs_c": 16, "sellcs_sigma": 512, "kernel": 0},
    {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 32, "kernel": 0},
    {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 512, "kernel": 0},
    {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 4096, "kernel": 0},
    {"format": "sell_c_s", "sellcs_c": 64, "sellcs_sigma": 1024, "kernel": 0},
    {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 512, "kernel": 4},
    {"format": "div_rf"},
    # the later kernels: SELL-C-sigma on kernels 8 and 10, SELL with 32-row slices on kernel
    # 10, DIV-RF with 32 lanes (the warp decoder)
    {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 512, "kernel": 8},
    {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 512, "kernel": 10},
    {"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 4096, "kernel": 10},
    {"format": "sell", "vec_len": 32, "kernel": 10},
    {"format": "div_rf", "vec_len": 32},
]
DEFAULT_CLASS = 0      # what the library picks without a selector


def batch_desc(i):
    """The batch descriptor dict of class i: its format and slice parameters (the batch
    kernel has one staging geometry for all matrices)."""
    return {k: v for k, v in CLASSES[i].items() if k in ("format", "vec_len", "sellcs_c", "sellcs_sigma")}


# one class per distinct batch descriptor of the formats the batched kernel runs
BATCHABLE = []
for _i, _c in enumerate(CLASSES):
    if _c["format"] in ("csr_naive", "sell", "sell_sorted", "sell_c_s") and \
            all(batch_desc(_i) != batch_desc(_j) for _j in BATCHABLE):
        BATCHABLE.append(_i)


def batch_plan(times, tol=0.05):
    """Per-matrix classes of a batch from its matrices' exhaustive timings (times[i][k], ms):
    csr_naive (the default class) for every matrix when the sum of its times is within `tol`
    of the per-matrix best sum, since an all-csr_naive batch runs as one block-diagonal
    SpMV on the warp-specialised kernel, about twice the throughput of the mixed-format
    work queue; otherwise each matrix's own best class."""
    t = np.where(np.isfinite(times), times, np.inf)
    best = np.argmin(t, axis=1)
    if np.sum(t[:, DEFAULT_CLASS]) <= (1.0 + tol) * np.sum(t[np.arange(t.shape[0]), best]):
        return np.full(t.shape[0], DEFAULT_CLASS)
    return best


def class_name(i):
    c = CLASSES[i]
    rest = ",".join(f"{k}={v}" for k, v in c.items() if k != "format")
    return c["format"] + (f"({rest})" if rest else "")


class Timer:
    """CUDA-event timing of single SpMVs with an L2 flush before each."""

    def __init__(self, torch, device, flush_bytes=256 << 20):
        self.torch = torch
        self.flush = torch.empty(flush_bytes // 4, dtype=torch.float32, device=device)

    def time(self, mf, xd, yd, reps=7, warmup=2):
        torch = self.torch
        stream = torch.cuda.current_stream()
        for _ in range(warmup):
            mf.spmv(xd, yd)
        per = []
        for _ in range(reps):
            self.flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            mf.spmv(xd, yd)
            e1.record(stream)
            e1.synchronize()
            per.append(e0.elapsed_time(e1))
        return statistics.median(per)


def exhaustive(sb, timer, rp, ci, v, m, n, classes=None, reps=7):
    """Times every class on one matrix: (ms per class, best class, tuning wall seconds)."""
    torch = timer.torch
    classes = list(range(len(CLASSES))) if classes is None else list(classes)
    xd = torch.empty(n, dtype=torch.float64, device="cuda").uniform_(-1.0, 1.0)
    yd = torch.empty(m, dtype=torch.float64, device="cuda")
    nnz = int(ci.numel()) if getattr(ci, "is_cuda", False) else int(rp[-1])
    times = {}
    t0 = time.perf_counter()
    for i in classes:
        try:
            mf = sb.csr_to_format(rp, ci, v, m, n, nnz, **CLASSES[i])
            times[i] = timer.time(mf, xd, yd, reps=reps)
            mf.destroy()
        except sb.SpmvError:
            times[i] = float("inf")
    torch.cuda.synchronize()
    cost = time.perf_counter() - t0
    best = min(times, key=lambda k: times[k])
    return times, best, cost


def ratio_to_best(times, chosen):
    """Throughput of the chosen class relative to the best class (1.0 = the best)."""
    best = min(times.values())
    t = times.get(chosen, float("inf"))
    return best / t if np.isfinite(t) and t > 0 else 0.0
