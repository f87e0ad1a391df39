"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

Run here, where the reference checkout is present and `make -C oracle ref` has compiled
it from its own sources into oracle/_ref/:

    python tests/golden/make_golden.py

Each fixture (an .npz) holds one CSR matrix, an x vector, and what the reference's own
code produced for it with 8 OpenMP threads on its x86 AVX2 build (VEC_LEN = 4):
  * y of csr_naive, csr_vec, sell, sell_sorted and div_rf (Matrix_Format::spmv, y
    pre-filled with 1.0 as bench_spmv.cpp:561-564 does);
  * the converted arrays of sell / sell_sorted (row_cluster_ptr, ja, a, permutations,
    thread ranges), of SELL-C-sigma (sellcs_format.c, two (C, sigma) settings) and of
    DIV-RF (every thread's packet stream and packet-group offsets, 16384 values/packet,
    plus one small-packet setting that splits rows across packets; the two padding bytes
    of each packet header, which the reference never writes, are stored as zero);
  * for generated matrices, the generator's own CSR (the native generator is pinned on it).
The reference has no shipped golden vectors or tests; these fixtures are its outputs.
"""
from __future__ import annotations

import os
import sys

import hashlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

T = 8
BIG = 40000                     # arrays above this many elements are stored as digests
KEEP = {"row_ptr", "col_ind", "values", "x"}   # the inputs are always stored in full


def hand6():
    # 6x6 with an empty row (row 3) and a full row; hand-checkable.
    rows = [[(0, 1.0), (2, 2.0)], [(1, -3.0)], [(0, 0.5), (3, 4.0), (5, -1.0)], [], [(4, 2.5), (5, 1.5)],
            [(0, 1.0), (1, 1.0), (2, 1.0), (3, 1.0), (4, 1.0), (5, 1.0)]]
    rp = [0]
    ci, v = [], []
    for r in rows:
        for c, a in r:
            ci.append(c)
            v.append(a)
        rp.append(len(ci))
    x = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float64), 6, x, None


def generated(args, seed_x):
    rows, cols = args[0], args[1]
    rp, ci, v, st = O.ref_generate(*args, threads=T)
    v = 2.0 * v - 1.0                      # values U[-1, 1): v -> 2v - 1 (exact in binary64)
    x = np.random.default_rng(seed_x).uniform(-1.0, 1.0, cols)
    return rp, ci, v, cols, x, dict(args=np.array([str(a) for a in args]))


def random_csr(m, n, density, empty_frac, seed, long_rows=()):
    rng = np.random.default_rng(seed)
    rp = [0]
    ci, v = [], []
    for i in range(m):
        if i in long_rows:
            k = long_rows[i]
        elif rng.random() < empty_frac:
            k = 0
        else:
            k = int(rng.poisson(density * n)) + 1
        k = min(k, n)
        cols = np.sort(rng.choice(n, size=k, replace=False))
        ci.extend(cols.tolist())
        v.extend(rng.uniform(-1, 1, k).tolist())
        rp.append(len(ci))
    x = rng.uniform(-1, 1, n)
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float64), n, x, None


def with_duplicates(seed):
    # values drawn from a small set, so DIV-RF sees replication factors > 1
    rp, ci, v, n, x, _ = random_csr(700, 900, 0.02, 0.1, seed)
    rng = np.random.default_rng(seed + 1)
    pool = rng.uniform(-1, 1, 37)
    v = pool[rng.integers(0, pool.size, v.size)]
    return rp, ci, v, n, x, None


def long_dup_row(seed):
    # single-row packets with replicated values and odd unique counts (DIV-RF row_bits == 0)
    rp, ci, v, n, x, _ = random_csr(40, 30000, 0.0004, 0.1, seed, long_rows={2: 5003, 17: 1999})
    rng = np.random.default_rng(seed + 1)
    pool = rng.uniform(-1, 1, 301)
    v = pool[rng.integers(0, pool.size, v.size)]
    return rp, ci, v, n, x, None


FIXTURES = {
    "hand6": hand6,
    "gen_normal_400": lambda: generated((400, 400, 10, 2, "normal", "random", 0.3, 0, 1.0, 0.5, 14), 1),
    "gen_gamma_skew_2000": lambda: generated((2000, 2000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7), 2),
    "gen_diag_1500": lambda: generated((1500, 1800, 12, 6, "gamma", "diagonal", 0.2, 30, 1.4, 0.6, 21), 3),
    "empty_rows_333": lambda: random_csr(333, 500, 0.01, 0.35, 4),
    "long_rows_60": lambda: random_csr(60, 40000, 0.0005, 0.1, 5, long_rows={3: 17000, 41: 2500}),
    "dup_values_700": lambda: with_duplicates(6),
    "long_dup_row_40": lambda: long_dup_row(8),
}


def make(name, fn):
    rp, ci, v, n, x, extra = fn()
    m = rp.size - 1
    out = dict(row_ptr=rp, col_ind=ci, values=v, n=np.int64(n), x=x)
    if extra:
        out.update({f"gen_{k}" if not k.startswith("gen_") else k: val for k, val in extra.items()})
    for fmt in ["csr_naive", "csr_vec", "sell", "sell_sorted", "div_rf"]:
        R = O.RefFormat(fmt, rp, ci, v, n=n, threads=T)
        out[f"y_{fmt}"] = R.spmv(x)[:m].copy()
        out[f"mem_{fmt}"] = np.float64(R.mem_footprint)
        if fmt in ("sell", "sell_sorted"):
            for k, a in R.sell_arrays().items():
                out[f"{fmt}_{k}"] = a
        if fmt == "div_rf":
            d = R.div_arrays()
            out["div_data"] = O.div_zero_header_padding(d["data"], 4)
            out["div_thread_bytes"] = d["thread_bytes"]
            out["div_group_pos"] = d["group_pos"]
            out["div_ranges"] = d["ranges"]
    for C, s in [(32, 256), (64, 64)]:
        a = O.ref_sellcs_convert(rp, ci, v, C, s)
        for k, arr in a.items():
            out[f"sellcs_{C}_{s}_{k}"] = arr
    # a small packet size (splits long rows across packets, several packets per group)
    os.environ["CSRCV_NUM_PACKET_VALS"] = "1000"
    try:
        R = O.RefFormat("div_rf", rp, ci, v, n=n, threads=T)
        d = R.div_arrays()
        out["div1000_data"] = O.div_zero_header_padding(d["data"], 4)
        out["div1000_group_pos"] = d["group_pos"]
        out["div1000_ranges"] = d["ranges"]
        out["y_div_rf_1000"] = R.spmv(x)[:m].copy()
    finally:
        os.environ["CSRCV_NUM_PACKET_VALS"] = "16384"
    # Large arrays are kept as SHA-256 digests only (the tests hash the GPU export and
    # compare; the oracle restatement, itself pinned on these digests, locates mismatches).
    for k in list(out):
        a = out[k]
        if isinstance(a, np.ndarray) and a.dtype != np.dtype("U") and a.size > BIG and k not in KEEP:
            out["sha256_" + k] = np.array(hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest())
            out["size_" + k] = np.int64(a.size)
            del out[k]
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    return path, m, int(rp[-1])


def main():
    if not O.ref_available("div_rf"):
        raise SystemExit("reference build missing: run `make -C oracle ref` first")
    for name, fn in FIXTURES.items():
        path, m, nnz = make(name, fn)
        print(f"{name}: m={m} nnz={nnz} -> {os.path.relpath(path, ROOT)} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
