"""Builds an autotuning database: for each seed, the matrix's GPU features and the CUDA-event
time of every format / parameter class (tuning.CLASSES), one JSON line per matrix.

    python spmv-dare_b200/tune_db.py --set selector --seeds 0:600 --out db.jsonl
    python spmv-dare_b200/tune_db.py --set batch --seeds 1000:1512 --classes batchable --out db.jsonl
    python spmv-dare_b200/tune_db.py --npz db.jsonl data/tune_x.npz     # compact arrays (data/)

Lines are written as each matrix finishes (an interrupted run keeps what it measured);
an existing output file is resumed (seeds already present are skipped).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def load_package():
    if "spmv_dare_b200" in sys.modules:
        return sys.modules["spmv_dare_b200"]
    spec = importlib.util.spec_from_file_location("spmv_dare_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["spmv_dare_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


PARAM_KEYS = ["rows", "avg", "std", "skew", "bw", "neigh", "cross"]


def to_npz(src, dst, num_classes=None):
    """The JSON lines of `src` as compact arrays (sorted by seed; NaN = class not timed,
    inf = class failed)."""
    import numpy as np

    if num_classes is None:
        load_package()
        from spmv_dare_b200 import tuning

        num_classes = len(tuning.CLASSES)

    R = sorted((json.loads(l) for l in open(src)), key=lambda r: r["seed"])
    times = np.full((len(R), num_classes), np.nan)
    for i, r in enumerate(R):
        for k, v in r["times_ms"].items():
            times[i, int(k)] = np.inf if v is None else v
    np.savez_compressed(dst, seeds=np.array([r["seed"] for r in R]), m=np.array([r["m"] for r in R]),
                        nnz=np.array([r["nnz"] for r in R]), features=np.array([r["features"] for r in R]),
                        times_ms=times, best=np.array([r["best"] for r in R]), tune_s=np.array([r["tune_s"] for r in R]),
                        features_s=np.array([r["features_s"] for r in R]),
                        gamma=np.array([r["params"]["distribution"] == "gamma" for r in R]),
                        params=np.array([[r["params"][k] for k in PARAM_KEYS] for r in R]),
                        param_names=np.array(PARAM_KEYS))


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if argv and argv[0] == "--npz":
        return to_npz(argv[1], argv[2])
    ap = argparse.ArgumentParser()
    ap.add_argument("--set", choices=["selector", "batch"], default="selector")
    ap.add_argument("--seeds", default="0:100", help="first:end (end exclusive)")
    ap.add_argument("--classes", default="all", choices=["all", "batchable"])
    ap.add_argument("--rows-lo", type=float, default=1e4)
    ap.add_argument("--rows-hi", type=float, default=3e5)
    ap.add_argument("--reps", type=int, default=7)
    ap.add_argument("--device-gen", action="store_true",
                    help="generate each matrix on the GPU and convert it from device memory")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    import torch

    sb = load_package()
    from spmv_dare_b200 import selector, tuning, workloads

    s0, s1 = (int(t) for t in a.seeds.split(":"))
    done = set()
    if os.path.exists(a.out):
        with open(a.out) as f:
            for line in f:
                try:
                    done.add(json.loads(line)["seed"])
                except Exception:
                    pass
    classes = tuning.BATCHABLE if a.classes == "batchable" else list(range(len(tuning.CLASSES)))
    timer = tuning.Timer(torch, "cuda")
    with open(a.out, "a") as out:
        for seed in range(s0, s1):
            if seed in done:
                continue
            p = workloads.batch_params(seed) if a.set == "batch" else workloads.selector_params(seed, a.rows_lo, a.rows_hi)
            if a.device_gen:
                rp, ci, v = workloads.generate_device(sb, p)
                m, n, nnz = p["rows"], p["cols"], int(ci.numel())
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                F = selector.features_device(rp, ci, m, n, nnz)
            else:
                rp, ci, v, _ = workloads.generate(sb, p)
                m, n, nnz = rp.size - 1, p["cols"], int(rp[-1])
                t0 = time.perf_counter()
                F = selector.features(rp, ci, m, n)
            feat_s = time.perf_counter() - t0
            times, best, cost = tuning.exhaustive(sb, timer, rp, ci, v, m, n, classes, reps=a.reps)
            rec = {"seed": seed, "params": p, "m": m, "n": n, "nnz": nnz, "features": F.tolist(),
                   "features_s": feat_s, "times_ms": {str(k): (None if t == float("inf") else t) for k, t in times.items()},
                   "best": best, "tune_s": cost}
            out.write(json.dumps(rec) + "\n")
            out.flush()
            print(f"seed {seed} m {m} nnz {nnz} best {tuning.class_name(best)} {times[best]:.4f} ms tune {cost:.2f}s",
                  flush=True)


if __name__ == "__main__":
    sys.exit(main())
