"""Benchmark of the SpMV hot path on B200 (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--format csr_naive] [--impl ours|reference]

Workload: the 4M x 4M configuration of the reference's artificial generator (gamma row
lengths, skew 100, seed 7; nnz 80,469,735), generated natively, values mapped to U[-1, 1),
x ~ U[-1, 1).  A step is one SpMV y = A x over the whole matrix.

Metric: SpMV GB/s over the algorithmic bytes of one SpMV,
    B = nnz * (8 + 4) + (m + 1) * 4 + n * 8 + m * 8
(the reference's csr_mem_footprint, spmv_kernel.h:23, plus x read once and y written once),
and GFLOP/s = 2 nnz / t (bench_spmv.cpp:358).  `value` is measured on device-resident
inputs with CUDA events around exactly K steps (after W warm-up steps); the inputs (1.05 GB)
exceed the 126 MB L2, so no flush is needed between steps.  `e2e` is the same metric
through the public API with host buffers: x copied host->device and y device->host inside
every timed step.  Every format of the reference is converted and timed (`per_format`);
the headline `value` is --format.

--impl reference times the reference's own CPU implementation of the same format, compiled
from its sources (oracle/_ref), on all host cores.

--workload batch: the batched engine on 512 artificial matrices (seeds 1000-1511, rows
log-uniform in [1e3, 2e5], parameters from spmv-dare_b200/workloads.py), each in the format
the batch autotuner picked for it from the matrices' exhaustive timings
(spmv-dare_b200/data/tune_batch.npz, tuning.batch_plan; --retune re-runs the timings here).  A step is one SpMV of every matrix: one CUDA-graph replay of
the persistent work-queue kernel (`value`), beside the same batch launched directly and the
512 matrices launched one by one with their own handles.  Metric: the aggregate algorithmic
bytes of the 512 SpMVs over the step time.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import signal
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
CONFIG2 = (4000000, 4000000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7)
WORKLOAD = "4M-row artificial gamma matrix: 4Mx4M, avg 20, std 15, gamma, random, bw 0.05, skew 100, neigh 2.0, cross 0.3, seed 7"
FORMATS = ["csr_naive", "csr_vec", "sell", "sell_sorted", "sell_c_s", "div_rf"]
FORMAT_PARAMS = {
    "sell_c_s": dict(sellcs_c=32, sellcs_sigma=512),
}
FALLBACK_HBM = 6650.0
# "tuned" settings timed beside each format's plain (reference-default) one: the GPU-native
# choices of slice height, sorting window, kernel, lane count and packet size.  A setting
# that changes the operation order (csr_vec lanes, slice heights) is held to the stated
# tolerance against csr_naive instead of bit parity.
TUNED = {
    "csr_naive": [dict(pack_cols=1), dict(kernel=4, threads=192, block_rows=64, block_nnz=1024, stages=3),
                  dict(kernel=4, threads=160, block_rows=64, block_nnz=512, stages=3)],
    "csr_vec": [dict(vec_len=8), dict(vec_len=2)],
    "sell": [dict(vec_len=16), dict(vec_len=32), dict(vec_len=32, stages=5)],
    "sell_sorted": [dict(vec_len=16), dict(vec_len=32), dict(vec_len=32, stages=5)],
    "sell_c_s": [dict(sellcs_c=32, sellcs_sigma=512, stages=5), dict(sellcs_c=32, sellcs_sigma=4096),
                 dict(sellcs_c=32, sellcs_sigma=32), dict(sellcs_c=64, sellcs_sigma=1024)],
    "div_rf": [dict(vec_len=32), dict(vec_len=32, div_packet_vals=4096), dict(vec_len=32, div_packet_vals=2048),
               dict(vec_len=32, div_packet_vals=1024)],
}
TUNED_TOL = 1e-12
# FP32 variant settings timed (the first is the library default); every one sums each row
# as the same sequential Dot2 chain, so y is the same bits
FP32_SETTINGS = [dict(), dict(row_assign=1), dict(format="sell_c_s", sellcs_c=32, sellcs_sigma=512),
                 dict(pack_cols=1), dict(threads=256, block_rows=96, block_nnz=1536)]


def load_package():
    if "spmv_dare_b200" in sys.modules:
        return sys.modules["spmv_dare_b200"]
    pkg = os.path.join(ROOT, "spmv-dare_b200")
    spec = importlib.util.spec_from_file_location("spmv_dare_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["spmv_dare_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def algorithmic_bytes(m, n, nnz, vsize=8, xsize=8):
    return nnz * (vsize + 4) + (m + 1) * 4 + n * xsize + m * xsize


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def ncu_traffic(fmt):
    """dram bytes per launch of the format's kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"spmv_{fmt}_gamma4m.md")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = os.path.join("/tmp", f"spmv_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        # nvidia-smi's start-up (seconds on a freshly booted node) can hold the driver and
        # stall this process's launches: time only once its first sample is written
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 15.0:
            if os.path.getsize(self.path) > 0 or self.p.poll() is not None:
                break
            time.sleep(0.05)
        time.sleep(0.3)

    def stop(self):
        if self.p is None:
            return None
        self.p.send_signal(signal.SIGTERM)
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.remove(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


class stdout_to_stderr:
    """The reference's CPU code prints progress to stdout; keep stdout for the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, v):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def config_tuple(args):
    """Config 2, optionally with fewer rows/cols (--rows, for profiling captures)."""
    if args.rows:
        return (args.rows, args.rows) + CONFIG2[2:]
    return CONFIG2


def generate(sb, args):
    g = sb.generate_artificial(*config_tuple(args))
    v = 2.0 * g.values - 1.0
    x = np.random.default_rng(12345).uniform(-1.0, 1.0, g.m)
    return g.row_ptr, g.col_ind, v, x


def make_config(args, fmt, m, n, nnz, B, world):
    """The `config` object of both arms (same keys, so the two lines compare key by key)."""
    return {"workload": WORKLOAD if not args.rows else WORKLOAD.replace("4Mx4M", f"{m}x{n}"),
            "format": fmt, "m": m, "n": n, "nnz": nnz, "bytes_per_spmv": B,
            "l2": "no flush: inputs (1.05 GB/SpMV) exceed the 126 MB L2",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "format_params": FORMAT_PARAMS.get(fmt, {})}


def convert_median(sb, rp, ci, v, m, n, nnz, fmt, reps=3, **params):
    """Converts `reps` times and keeps the handle of the median conversion time; returns
    (handle, {convert_ms, alloc_ms, copy_in_ms} of that conversion, all conversion times)."""
    runs = []
    for _ in range(reps):
        mf = sb.csr_to_format(rp, ci, v, m, n, nnz, format=fmt, **params)
        runs.append(mf)
    runs.sort(key=lambda h: h.convert_ms)
    keep = runs[len(runs) // 2]
    allms = sorted(h.convert_ms for h in runs)
    for h in runs:
        if h is not keep:
            h.destroy()
    return keep, {"convert_ms": keep.convert_ms, "convert_alloc_ms": keep.alloc_ms,
                  "convert_copy_in_ms": keep.copy_in_ms}, allms


def time_device(mf, xd, yd, steps, warmup, torch):
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        mf.spmv(xd, yd)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    ev[0].record(stream)
    for k in range(steps):
        mf.spmv(xd, yd)
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
    total = ev[0].elapsed_time(ev[steps])
    return total, per


def run_ours(args):
    import torch

    world, rank, local = dist_setup(args)
    sb = load_package()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rp, ci, v, x = generate(sb, args)
    m, n, nnz = rp.size - 1, rp.size - 1, int(rp[-1])
    f32 = args.value_type == "f32"
    B = algorithmic_bytes(m, n, nnz, 4, 4) if f32 else algorithmic_bytes(m, n, nnz)
    flops = 2.0 * nnz
    peak, peak_kind = hbm_peak()

    formats = [args.format] + [f for f in FORMATS if f != args.format] if args.all_formats else [args.format]
    per_format = {}
    head = None
    for fmt in formats:
        try:
            mf, conv, conv_all = convert_median(sb, rp, ci, v, m, n, nnz, fmt, **FORMAT_PARAMS.get(fmt, {}))
        except sb.SpmvError as e:
            per_format[fmt] = {"error": str(e)}
            continue
        if args.value_type == "f32" and fmt == args.format:
            xd = torch.from_numpy(x.astype(np.float32)).to(dev)
            yd = torch.empty(m, dtype=torch.float32, device=dev)
        else:
            xd = torch.from_numpy(x).to(dev)
            yd = torch.empty(m, dtype=torch.float64, device=dev)
        sampler = ClockSampler(local) if fmt == args.format else None
        barrier(world)
        if sampler:
            sampler.start()
        total_ms, per = time_device(mf, xd, yd, args.steps, args.warmup, torch)
        clocks = sampler.stop() if sampler else None
        barrier(world)
        total_ms = max_over_ranks(world, total_ms)
        ms = total_ms / args.steps
        med = statistics.median(per)
        rec = {"ms_per_step": ms, "ms_median": med, "gbs": B * 1e-9 / (ms * 1e-3),
               "gflops": flops * 1e-9 / (ms * 1e-3), "hbm_frac": B * 1e-9 / (med * 1e-3) / peak,
               **conv, "convert_ms_all": [round(t, 2) for t in conv_all],
               "mem_footprint": mf.mem_footprint, "stored_elems": mf.stored_elems,
               "kernels_per_spmv": mf.kernels_per_run}
        per_format[fmt] = rec
        if fmt == args.format:
            head = dict(rec, clocks=clocks, mf=mf, xd=xd, yd=yd, per=per)
        else:
            del mf
        torch.cuda.empty_cache()

    if head is None:
        raise SystemExit(f"format {args.format} failed: {per_format.get(args.format)}")
    if args.all_formats and not args.no_tuned:
        tuned_legs(sb, torch, dev, rp, ci, v, x, per_format, B, peak, args)
    if args.all_formats:
        per_format["csr_f32_dot2"] = fp32_variant(sb, torch, dev, rp, ci, v, x, args, per_format)

    # e2e: public API with pinned host buffers; x H2D and y D2H inside every step
    mf = head["mf"]
    xh = torch.from_numpy(x.astype(np.float32) if f32 else x).pin_memory().numpy()
    yh = torch.empty(m, dtype=torch.float32 if f32 else torch.float64).pin_memory().numpy()
    for _ in range(args.warmup):
        mf.spmv(xh, yh)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        mf.spmv(xh, yh)
    e2e_s = (time.perf_counter() - t0) / args.steps
    e2e_s = max_over_ranks(world, e2e_s)

    value = world * B * 1e-9 / (head["ms_per_step"] * 1e-3)
    achieved = B * 1e-9 / (statistics.median(head["per"]) * 1e-3)
    traffic = ncu_traffic("csr_f32_dot2" if f32 else args.format)
    out = {
        "metric": "SpMV GB/s (algorithmic bytes / time; % of HBM peak in roofline)",
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(head["ms_per_step"], 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if f32 else "f64",
        "data": "synthetic (the reference's artificial generator restated natively, the 4M-row gamma matrix; values 2v-1, x U[-1,1))",
        "config": make_config(args, args.format, m, n, nnz, B, world),
        "gflops": round(head["gflops"], 2),
        "e2e": {"value": round(world * B * 1e-9 / e2e_s, 2), "unit": "GB/s",
                "h2d_bytes_per_step": int((max(0, mf.x_span[1] - mf.x_span[0] + 1) + mf.x_col0) * xh.itemsize),
                "d2h_bytes_per_step": int(yh.nbytes), "ms_per_step": round(e2e_s * 1e3, 4),
                "x_copied": {"span": list(mf.x_span), "x0": mf.x_col0}},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured"
                     else "fallback 6.65 TB/s"},
        "gpu_launches": args.steps * mf.kernels_per_run,
        "clocks": head["clocks"],
        "per_format": {k: {kk: (float(f"{vv:.5g}") if isinstance(vv, float) else vv) for kk, vv in r.items()}
                       for k, r in per_format.items()},
    }
    if args.all_formats and not args.no_batch:
        del head, mf
        torch.cuda.empty_cache()
        out["batch"] = batch_block(sb, torch, dev, args, world, peak)
        torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with stdout_to_stderr():
            out["cpu_baseline"] = cpu_baseline(args.format, rp, ci, v, x, B, sample_s=args.cpu_seconds)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def reference_rows(sb, torch, dev, rp, ci, v, x):
    """FP64 csr_naive y (the reference's bits) and sum_j |a_ij x_j| per row, on the GPU."""
    m, n, nnz = rp.size - 1, x.size, int(rp[-1])
    m64 = sb.csr_to_format(rp, ci, v, m, n, nnz, format="csr_naive")
    y64 = torch.empty(m, dtype=torch.float64, device=dev)
    m64.spmv(torch.from_numpy(x).to(dev), y64)
    mabs = sb.csr_to_format(rp, ci, np.abs(v), m, n, nnz, format="csr_naive")
    absy = torch.empty(m, dtype=torch.float64, device=dev)
    mabs.spmv(torch.from_numpy(np.abs(x)).to(dev), absy)
    torch.cuda.synchronize()
    m64.destroy()
    mabs.destroy()
    return y64, absy


def tuned_legs(sb, torch, dev, rp, ci, v, x, per_format, B, peak, args):
    """Each format's TUNED settings, timed like the plain line; the fastest one whose y is
    within TUNED_TOL of csr_naive (relative to max(|y|, sum |a x|)) becomes the format's
    `tuned` entry."""
    m, n, nnz = rp.size - 1, x.size, int(rp[-1])
    y64, absy = reference_rows(sb, torch, dev, rp, ci, v, x)
    den = torch.maximum(y64.abs(), absy).clamp_min(1e-300)
    xd = torch.from_numpy(x).to(dev)
    yd = torch.empty(m, dtype=torch.float64, device=dev)
    steps = max(5, args.steps // 2)
    for fmt, cands in TUNED.items():
        rec = per_format.get(fmt)
        if not rec or "error" in rec:
            continue
        best, tried = None, []
        for params in cands:
            try:
                mf = sb.csr_to_format(rp, ci, v, m, n, nnz, format=fmt, **params)
            except sb.SpmvError as e:
                tried.append({"params": params, "error": str(e)[:120]})
                continue
            _, per = time_device(mf, xd, yd, steps, args.warmup, torch)
            med = statistics.median(per)
            err = float(((yd - y64).abs() / den).max().item())
            entry = {"params": params, "ms_median": round(med, 5), "gbs": round(B * 1e-9 / (med * 1e-3), 1),
                     "hbm_frac": round(B * 1e-9 / (med * 1e-3) / peak, 4), "max_rel_err_vs_csr": err,
                     "convert_ms": round(mf.convert_ms, 2), "stored_elems": mf.stored_elems}
            tried.append({"params": params, "ms_median": entry["ms_median"], "max_rel_err_vs_csr": err})
            if err <= TUNED_TOL and (best is None or med < best["ms_median"]):
                best = entry
            mf.destroy()
            torch.cuda.empty_cache()
        if best is not None and best["ms_median"] < rec["ms_median"]:
            rec["tuned"] = best
        else:
            rec["tuned"] = {"params": "plain (no faster setting within tolerance)", "ms_median": rec["ms_median"],
                            "hbm_frac": rec["hbm_frac"]}
        rec["tuned_tried"] = tried


def mixed_classes(count):
    """Batch formats dealt round robin over sell, sell_sorted, sell_c_s (C=32, sigma=512) and
    csr_naive: a batch that runs the persistent work-queue kernel."""
    from spmv_dare_b200 import tuning

    pool = [tuning.CLASSES.index({"format": "sell", "vec_len": 4}),
            tuning.CLASSES.index({"format": "sell_sorted", "vec_len": 4}),
            tuning.CLASSES.index({"format": "sell_c_s", "sellcs_c": 32, "sellcs_sigma": 512, "kernel": 0}), 0]
    return [pool[i % 4] for i in range(count)]


def batch_block(sb, torch, dev, args, world, peak):
    """The 512-matrix batch (C4) inside the default line: the autotuned batch (every matrix
    csr_naive with these kernels: one block-diagonal SpMV, CUDA-graph replay) and the same
    matrices with formats dealt round robin over csr_naive / sell / sell_sorted / sell_c_s,
    which runs the persistent work-queue kernel; y of each against the matrices' own
    handles, bit for bit."""
    from spmv_dare_b200 import tuning

    mats, classes, xs, B = batch_matrices(sb, args.batch_count, False)
    xh = np.concatenate(xs)
    xd = torch.from_numpy(xh).to(dev)
    out = {"workload": batch_workload(len(mats)), "matrices": len(mats), "bytes_per_step": B,
           "nnz_total": sum(int(mt[0][-1]) for mt in mats)}
    steps = max(5, args.steps // 2)
    legs = [("tuned", classes), ("mixed", mixed_classes(len(mats)))]
    for name, cls in legs:
        batch = sb.Batch(mats, [tuning.batch_desc(c) for c in cls])
        yd = torch.empty(batch.total_y, dtype=torch.float64, device=dev)
        barrier(world)
        ms, per = time_events(lambda: batch.spmv(xd, yd, graph=True), steps, args.warmup, torch)
        barrier(world)
        ms = max_over_ranks(world, ms)
        y_batch = yd.cpu().numpy().copy()
        # the same matrices, each through its own handle of the same format
        ident = True
        for i, ((rp, ci, v, m, n), c) in enumerate(zip(mats, cls)):
            h = sb.csr_to_format(rp, ci, v, m, n, int(rp[-1]), **tuning.batch_desc(c))
            xo, yo = int(batch.x_offsets[i]), int(batch.y_offsets[i])
            yv = torch.empty(m, dtype=torch.float64, device=dev)
            h.spmv(xd[xo:xo + n], yv)
            ident = ident and bool(np.array_equal(yv.cpu().numpy().view(np.uint64),
                                                  y_batch[yo:yo + m].view(np.uint64)))
            h.destroy()
        med = statistics.median(per)
        counts = {}
        for c in cls:
            counts[tuning.class_name(c)] = counts.get(tuning.class_name(c), 0) + 1
        out[name] = {"graph_ms": round(ms, 4), "gbs": round(world * B * 1e-9 / (ms * 1e-3), 1),
                     "hbm_frac": round(B * 1e-9 / (med * 1e-3) / peak, 4), "formats": counts,
                     "path": "block-diagonal csr_naive SpMV (warp-specialised kernel)" if batch.num_blocks == 0 or
                     all(tuning.CLASSES[c]["format"] == "csr_naive" for c in cls) else "persistent work-queue batch_kernel",
                     "y_identical_to_per_matrix": ident, "steps": steps}
        batch.destroy()
        del yd
        torch.cuda.empty_cache()
    return out


def fp32_variant(sb, torch, dev, rp, ci, v, x, args, per_format):
    """Config 3: FP32 values (rounded once), exact int32 indices, FP32 x/y, Dot2-compensated
    rows.  Bytes: 8 nnz + 4 (m+1) + 4 n + 4 m.  Error against the FP64 csr_naive result
    (bit-identical to the reference's), relative to max(|y|, sum |a x|) and plain |dy|/|y|."""
    m, n, nnz = rp.size - 1, rp.size - 1, int(rp[-1])
    B32 = nnz * 8 + (m + 1) * 4 + n * 4 + m * 4
    xd = torch.from_numpy(x.astype(np.float32)).to(dev)
    yd = torch.empty(m, dtype=torch.float32, device=dev)
    legs = {}
    for i, params in enumerate(FP32_SETTINGS):
        kw = dict(params)
        fmt = kw.pop("format", "csr_naive")      # FP32 values on CSR, or on 32-row SELL-C-sigma slices
        try:
            mf = sb.csr_to_format(rp, ci, v, m, n, nnz, format=fmt, value_type="f32", **kw)
        except sb.SpmvError:
            continue
        _, per = time_device(mf, xd, yd, args.steps, args.warmup, torch)
        legs[i] = (statistics.median(per), mf)
    pack = min(legs, key=lambda k: legs[k][0])
    med, mf = legs[pack]
    # FP64 reference and sum |a_ij x_j| on the GPU (csr_naive handles)
    m64 = sb.csr_to_format(rp, ci, v, m, n, nnz, format="csr_naive")
    y64 = torch.empty(m, dtype=torch.float64, device=dev)
    m64.spmv(torch.from_numpy(x).to(dev), y64)
    mabs = sb.csr_to_format(rp, ci, np.abs(v), m, n, nnz, format="csr_naive")
    absy = torch.empty(m, dtype=torch.float64, device=dev)
    mabs.spmv(torch.from_numpy(np.abs(x)).to(dev), absy)
    torch.cuda.synchronize()
    d = (yd.double() - y64).abs()
    cond = (d / torch.maximum(y64.abs(), absy).clamp_min(1e-300)).cpu().numpy()
    nz = y64.abs() > 0
    plain = (d[nz] / y64.abs()[nz]).cpu().numpy()
    t64 = per_format.get("csr_naive", {}).get("ms_median")
    return {"ms_median": med, "gbs": B32 * 1e-9 / (med * 1e-3), "gflops": 2.0 * nnz * 1e-9 / (med * 1e-3),
            "bytes_per_spmv": B32, "speedup_vs_fp64_csr": (t64 / med) if t64 else None,
            "max_rel_err_cond": float(cond.max()), "mean_rel_err_cond": float(cond.mean()),
            "max_rel_err_plain": float(plain.max()) if plain.size else 0.0,
            "mean_rel_err_plain": float(plain.mean()) if plain.size else 0.0,
            "convert_ms": mf.convert_ms, "params": FP32_SETTINGS[pack],
            "plain_ms_median": round(legs[0][0], 5) if 0 in legs else None,
            "tried": [{"params": FP32_SETTINGS[k], "ms_median": round(t, 5)} for k, (t, _) in legs.items()]}


def cpu_baseline(fmt, rp, ci, v, x, B, sample_s=10.0):
    """The reference's own CPU implementation (compiled from its sources into oracle/_ref),
    all host cores, timed like bench_spmv.cpp:316-358 (median iteration)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    cores = len(os.sched_getaffinity(0))
    name = fmt if fmt in ("csr_naive", "csr_vec", "sell", "sell_sorted", "div_rf") else "csr_naive"
    if not O.ref_available(name):
        return {"value": None, "unit": "GB/s", "cores": cores, "kind": "reference",
                "sample": f"unavailable: oracle/_ref/libref_{name}.so not built"}
    R = O.RefFormat(name, rp, ci, v, threads=cores)
    y = np.ones(R.m + 64)
    R.spmv(x, y)
    times = []
    t_end = time.perf_counter() + sample_s
    while time.perf_counter() < t_end or len(times) < 5:
        t0 = time.perf_counter()
        R.spmv(x, y)
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": round(B * 1e-9 / med, 3), "unit": "GB/s", "cores": cores, "kind": "reference",
            "format": name, "ms_median": round(med * 1e3, 3),
            "sample": f"the full 4M-row matrix, {len(times)} SpMV iterations over ~{sample_s:.0f} s, median"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    name = args.format if args.format in ("csr_naive", "csr_vec", "sell", "sell_sorted", "div_rf") else "csr_naive"
    if not O.ref_available(name) or not O.ref_available("gen"):
        print(json.dumps({"impl": "reference", "unavailable": f"reference build oracle/_ref/libref_{name}.so missing"}))
        return
    cores = len(os.sched_getaffinity(0))
    cfg = config_tuple(args)
    with stdout_to_stderr():
        rp, ci, v, st = O.ref_generate(*cfg, threads=cores)
    v = 2.0 * v - 1.0
    m = n = rp.size - 1
    nnz = int(rp[-1])
    x = np.random.default_rng(12345).uniform(-1.0, 1.0, n)
    B = algorithmic_bytes(m, n, nnz)
    with stdout_to_stderr():
        R = O.RefFormat(name, rp, ci, v, threads=cores)
        y = np.ones(m + 64)
        for _ in range(args.warmup):
            R.spmv(x, y)
        per = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            R.spmv(x, y)
            per.append(time.perf_counter() - t0)
    ms = 1e3 * sum(per) / len(per)
    val = B * 1e-9 / (ms * 1e-3)
    out = {
        "metric": "SpMV GB/s (algorithmic bytes / time; % of HBM peak in roofline)",
        "value": round(val, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (the reference's own generator, the 4M-row gamma matrix; values 2v-1, x U[-1,1))",
        "config": make_config(args, name, m, n, nnz, B, world),
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": cores, "kind": "reference",
                         "sample": f"the {'full 4M-row' if not args.rows else f'{m}-row'} matrix, {args.steps} timed "
                                   f"SpMV steps after {args.warmup} warm-up"},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


BATCH_SEEDS = (1000, 1512)
BATCH_WORKLOAD = ("batch: {count} artificial matrices, seeds 1000-{last}, rows log-uniform [1e3, 2e5], avg U[5,60], "
                  "std U[0.1,1]xavg, normal/gamma, skew U[0,200], bw U[0.01,0.5], random placement")


def batch_workload(count):
    return BATCH_WORKLOAD.format(count=count, last=BATCH_SEEDS[0] + count - 1)


def batch_matrices(sb, count, retune=False):
    """(matrices, per-matrix class, x vectors, total bytes) of the batched workload."""
    pkg = os.path.join(ROOT, "spmv-dare_b200")
    sys.path.insert(0, pkg)
    from spmv_dare_b200 import tuning, workloads

    times = {}
    db_path = os.path.join(pkg, "data", "tune_batch.npz")
    if not retune and os.path.exists(db_path):
        with np.load(db_path) as z:
            times = dict(zip(z["seeds"].tolist(), z["times_ms"]))
    timer = None
    mats, rows, xs, B = [], [], [], 0
    for seed in range(BATCH_SEEDS[0], BATCH_SEEDS[0] + count):
        p = workloads.batch_params(seed)
        rp, ci, v, x = workloads.generate(sb, p)
        m = n = p["rows"]
        if seed not in times:
            import torch

            timer = timer or tuning.Timer(torch, "cuda")
            t, _, _ = tuning.exhaustive(sb, timer, rp, ci, v, m, n, tuning.BATCHABLE, reps=5)
            times[seed] = np.array([t.get(k, np.nan) for k in range(len(tuning.CLASSES))])
        mats.append((rp, ci, v, m, n))
        rows.append(times[seed])
        xs.append(x)
        B += algorithmic_bytes(m, n, int(rp[-1]))
    # the batch-level choice over the matrices' exhaustive timings (tuning.batch_plan)
    classes = [int(k) for k in tuning.batch_plan(np.array(rows))]
    return mats, classes, xs, B


def time_events(fn, steps, warmup, torch):
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    ev[0].record(stream)
    for k in range(steps):
        fn()
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    return ev[0].elapsed_time(ev[steps]) / steps, [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]


def run_batch(args):
    import torch

    world, rank, local = dist_setup(args)
    sb = load_package()
    from spmv_dare_b200 import tuning

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    mats, classes, xs, B = batch_matrices(sb, args.batch_count, args.retune)
    if args.batch_formats == "mixed":
        classes = mixed_classes(len(mats))
    nnz_total = sum(int(mt[0][-1]) for mt in mats)
    batch = sb.Batch(mats, [tuning.batch_desc(c) for c in classes])
    xh = np.concatenate(xs)
    xd = torch.from_numpy(xh).to(dev)
    yd = torch.empty(batch.total_y, dtype=torch.float64, device=dev)
    peak, peak_kind = hbm_peak()

    sampler = ClockSampler(local)
    barrier(world)
    sampler.start()
    ms_graph, per = time_events(lambda: batch.spmv(xd, yd, graph=True), args.steps, args.warmup, torch)
    clocks = sampler.stop()
    barrier(world)
    ms_graph = max_over_ranks(world, ms_graph)
    y_batch = yd.cpu().numpy().copy()
    ms_direct, _ = time_events(lambda: batch.spmv(xd, yd, graph=False), args.steps, args.warmup, torch)

    # the same matrices one launch each, with their own handles (each class's full tuning)
    handles = []
    for (rp, ci, v, m, n), c in zip(mats, classes):
        handles.append(sb.csr_to_format(rp, ci, v, m, n, int(rp[-1]), **tuning.CLASSES[c]))
    xo, yo = batch.x_offsets, batch.y_offsets
    views = [(xd[int(xo[i]):int(xo[i]) + mats[i][4]], yd[int(yo[i]):int(yo[i]) + mats[i][3]]) for i in range(len(mats))]

    def per_matrix():
        for h, (xv, yv) in zip(handles, views):
            h.spmv(xv, yv)

    ms_loop, _ = time_events(per_matrix, max(3, args.steps // 5), 3, torch)
    y_loop = yd.cpu().numpy()
    identical = bool(np.array_equal(y_batch.view(np.uint64), y_loop.view(np.uint64)))
    for h in handles:
        h.destroy()

    # e2e: host x in (pinned), one graph replay, host y out, every step
    xp = torch.from_numpy(xh).pin_memory()
    yp = torch.empty(batch.total_y, dtype=torch.float64).pin_memory()

    def e2e():
        xd.copy_(xp, non_blocking=True)
        batch.spmv(xd, yd, graph=True)
        yp.copy_(yd, non_blocking=True)

    for _ in range(args.warmup):
        e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(world, (time.perf_counter() - t0) / args.steps)

    achieved = B * 1e-9 / (statistics.median(per) * 1e-3)
    fmt_counts = {}
    for c in classes:
        fmt_counts[tuning.class_name(c)] = fmt_counts.get(tuning.class_name(c), 0) + 1
    out = {
        "metric": "batched SpMV GB/s (aggregate algorithmic bytes of all matrices / step time)",
        "value": round(world * B * 1e-9 / (ms_graph * 1e-3), 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_graph, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the reference's artificial generator restated natively; values 2v-1, x U[-1,1))",
        "config": {"workload": batch_workload(len(mats)), "matrices": len(mats), "nnz_total": nnz_total, "bytes_per_step": B,
                   "formats": fmt_counts, "tuning": "exhaustive autotuner over the batchable classes",
                   "l2": f"no flush: inputs ({B / 1e9:.2f} GB/step) exceed the 126 MB L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": {"value": round(world * B * 1e-9 / e2e_s, 2), "unit": "GB/s", "h2d_bytes_per_step": int(xh.nbytes),
                "d2h_bytes_per_step": int(batch.total_y * 8), "ms_per_step": round(e2e_s * 1e3, 4)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured"
                     else "fallback 6.65 TB/s"},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "batch": {"graph_ms": round(ms_graph, 4), "direct_ms": round(ms_direct, 4), "per_matrix_launches_ms": round(ms_loop, 4),
                  "graph_gbs": round(B * 1e-9 / (ms_graph * 1e-3), 1), "direct_gbs": round(B * 1e-9 / (ms_direct * 1e-3), 1),
                  "per_matrix_gbs": round(B * 1e-9 / (ms_loop * 1e-3), 1), "y_identical_to_per_matrix": identical,
                  "blocks": int(batch.num_blocks)},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with stdout_to_stderr():
            out["cpu_baseline"] = batch_cpu_baseline(mats, xs, args.cpu_seconds)
    batch.destroy()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def ref_batch_pass(mats, xs, reps, cores):
    """Seconds of one pass of the reference's csr_naive (compiled from its sources, all host
    cores) over the matrices: each converted, its SpMV timed `reps` times (mean), freed --
    the reference holds per-thread state in globals, one converted matrix at a time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    total = 0.0
    for (rp, ci, v, m, n), x in zip(mats, xs):
        R = O.RefFormat("csr_naive", rp, ci, v, threads=cores)
        y = np.ones(m + 64)
        R.spmv(x, y)
        t0 = time.perf_counter()
        for _ in range(reps):
            R.spmv(x, y)
        total += (time.perf_counter() - t0) / reps
        R.close()
    return total


def batch_cpu_baseline(mats, xs, sample_s=10.0):
    """The reference's csr_naive on all host cores, one pass over every batch matrix."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    cores = len(os.sched_getaffinity(0))
    if not O.ref_available("csr_naive"):
        return {"value": None, "unit": "GB/s", "cores": cores, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libref_csr_naive.so not built"}
    B = sum(algorithmic_bytes(m, n, int(rp[-1])) for (rp, ci, v, m, n) in mats)
    reps = 3
    t = ref_batch_pass(mats, xs, reps, cores)
    return {"value": round(B * 1e-9 / t, 3), "unit": "GB/s", "cores": cores, "kind": "reference",
            "format": "csr_naive", "ms_per_pass": round(t * 1e3, 3),
            "sample": f"all {len(mats)} batch matrices, SpMV time of each = mean of {reps} after 1 warm-up, summed"}


def run_reference_batch(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sb = load_package()
    with stdout_to_stderr():
        mats, classes, xs, B = batch_matrices(sb, args.batch_count, retune=False)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if not O.ref_available("csr_naive"):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libref_csr_naive.so missing"}))
        return
    cores = len(os.sched_getaffinity(0))
    with stdout_to_stderr():
        ref_batch_pass(mats[:2], xs[:2], args.warmup, cores)                 # warm-up
        t = ref_batch_pass(mats, xs, args.steps, cores)
    per = [t]
    ms = 1e3 * sum(per) / len(per)
    val = B * 1e-9 / (ms * 1e-3)
    print(json.dumps({
        "metric": "batched SpMV GB/s (aggregate algorithmic bytes of all matrices / step time)",
        "value": round(val, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the reference's artificial generator restated natively; values 2v-1, x U[-1,1))",
        "config": {"workload": batch_workload(len(mats)), "matrices": len(mats), "bytes_per_step": B, "format": "csr_naive"},
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": cores, "kind": "reference",
                         "sample": f"all {len(mats)} matrices per step; each matrix converted, its SpMV timed "
                                   f"{args.steps} times (mean), freed; step = sum over matrices"},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--format", default="csr_naive", choices=FORMATS)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--all-formats", dest="all_formats", action="store_true", default=True)
    ap.add_argument("--only-format", dest="all_formats", action="store_false")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--rows", type=int, default=0, help="the 4M-row gamma matrix with this many rows/cols (profiling)")
    ap.add_argument("--workload", default="gamma4m", choices=["gamma4m", "batch"])
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--retune", action="store_true", help="batch: re-run the autotuner instead of its database")
    ap.add_argument("--no-batch", action="store_true", help="leave the batch block out of the default line")
    ap.add_argument("--no-tuned", action="store_true", help="time only the plain settings of each format")
    ap.add_argument("--params", default="", help="JSON object of descriptor fields for --format (profiling)")
    ap.add_argument("--batch-formats", default="tuned", choices=["tuned", "mixed"],
                    help="--workload batch: the autotuner's formats, or four formats dealt round robin")
    ap.add_argument("--value-type", default="f64", choices=["f64", "f32"],
                    help="headline line of csr_naive with FP32 values and FP32 vectors (the FP32 variant)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.params:
        FORMAT_PARAMS[args.format] = dict(FORMAT_PARAMS.get(args.format, {}), **json.loads(args.params))
    if args.value_type == "f32":
        if args.format != "csr_naive" or args.all_formats:
            raise SystemExit("--value-type f32 times csr_naive alone (with --only-format)")
        FORMAT_PARAMS["csr_naive"] = dict(FORMAT_PARAMS.get("csr_naive", {}), value_type="f32")
    if args.workload == "batch":
        (run_reference_batch if args.impl == "reference" else run_batch)(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
