"""Synthetic matrix workloads of the batched and learned-selector benchmarks.

Every matrix comes from the native restatement of the reference's artificial generator
(artificial-matrix-generator/artificial_matrix_generation.c) with parameters drawn by a
seeded numpy PCG64 stream keyed by the matrix seed, so a seed always names the same matrix.
Values are mapped v -> 2v - 1 (U[-1, 1)), x ~ U[-1, 1) from the same stream.

batch_params (512 matrices, seeds 1000-1511):
    rows = cols log-uniform in [1e3, 2e5]; avg_row U[5, 60]; std = U[0.1, 1.0] x avg;
    distribution normal / gamma (50/50); skew U[0, 200]; avg_bw U[0.01, 0.5];
    placement random; neighbours U[1.0, 2.0] and cross-row similarity U[0.3, 0.5]
    (the range the 100k- and 4M-row configurations span).
selector_params: the same ranges with rows log-uniform in [rows_lo, rows_hi].
"""
from __future__ import annotations

import math

import numpy as np


def _draw(seed, rows_lo, rows_hi):
    r = np.random.Generator(np.random.PCG64(seed))
    rows = int(round(math.exp(r.uniform(math.log(rows_lo), math.log(rows_hi)))))
    avg = float(r.uniform(5.0, 60.0))
    std = float(r.uniform(0.1, 1.0)) * avg
    dist = "normal" if r.uniform() < 0.5 else "gamma"
    skew = float(r.uniform(0.0, 200.0))
    bw = float(r.uniform(0.01, 0.5))
    neigh = float(r.uniform(1.0, 2.0))
    cross = float(r.uniform(0.3, 0.5))
    return dict(rows=rows, cols=rows, avg=avg, std=std, distribution=dist, placement="random", bw=bw, skew=skew,
                neigh=neigh, cross=cross, seed=int(seed))


def batch_params(seed):
    """Generator parameters of one matrix of the 512-matrix batch."""
    return _draw(seed, 1e3, 2e5)


def selector_params(seed, rows_lo=1e4, rows_hi=3e5):
    """Generator parameters of one training / held-out matrix of the learned selector."""
    return _draw(seed, rows_lo, rows_hi)


def generate(sb, p):
    """(row_ptr, col_ind, values, x) of the matrix named by parameter dict p."""
    g = sb.generate_artificial(p["rows"], p["cols"], p["avg"], p["std"], p["distribution"], p["placement"], p["bw"],
                               p["skew"], p["neigh"], p["cross"], p["seed"])
    v = 2.0 * g.values - 1.0
    x = np.random.Generator(np.random.PCG64(p["seed"] + 7919)).uniform(-1.0, 1.0, p["cols"])
    return g.row_ptr, g.col_ind, v, x


def generate_device(sb, p):
    """(row_ptr, col_ind, values) CUDA tensors of the matrix named by p, generated on the GPU
    (distribution-equivalent to generate(); values mapped v -> 2v - 1)."""
    rp, ci, v = sb.generate_artificial_device(p["rows"], p["cols"], p["avg"], p["std"], p["distribution"],
                                              p["placement"], p["bw"], p["skew"], p["neigh"], p["cross"], p["seed"])
    return rp, ci, 2.0 * v - 1.0
