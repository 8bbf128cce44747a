"""Benchmark driver: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|single|multi] [--nrows N]

Workloads (seeded synthetic data on the device; no dataset is read):
  batched  1e8 rows x 4 uint32 columns (zipf 1.1, 1.3, 1.5 over 2^20
           values and a rounded normal), 1024 queries touching 1-4 columns
           with log-uniform selectivity in [0.01%, 90%]; one step = one
           batched pass answering all queries (bitmaps + counts).
  single   1e8 rows x 1 uniform column, one 10%-selectivity range; one step
           = one fused scan launch.
  multi    1e8 rows x 4 uniform columns, one conjunctive query with
           per-column selectivity in [5%, 50%]; fused vs separate passes.

Under torchrun each rank scans its own rows (weak scaling, no collective on
the data path); `value` is the aggregate over ranks.  Timing: W warm-up
steps, then K steps between CUDA events on the launching stream, barrier +
synchronize on both sides, max over ranks.  Inputs are larger than L2.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched range-scan GB/s & queries/s vs HBM peak; served query p50/p99 ms"


# ----------------------------------------------------------------------------
# environment
# ----------------------------------------------------------------------------

def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


# ----------------------------------------------------------------------------
# synthetic columns on the device
# ----------------------------------------------------------------------------

def gpu_column(torch, kind: str, n: int, seed: int, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if kind == "uniform":
        x = torch.randint(0, 1 << 32, (n,), generator=g, device=device, dtype=torch.int64)
        return x.to(torch.int32)  # two's-complement wrap keeps the uint32 bit pattern
    if kind.startswith("zipf"):
        s = float(kind[4:])
        distinct = 1 << 20
        ranks = torch.arange(1, distinct + 1, device=device, dtype=torch.float64)
        cdf = torch.cumsum(ranks.pow(-s), 0)
        cdf /= cdf[-1].clone()
        out = torch.empty(n, dtype=torch.int32, device=device)
        chunk = 1 << 24
        for i in range(0, n, chunk):
            m = min(chunk, n - i)
            u = torch.rand(m, generator=g, device=device, dtype=torch.float64)
            out[i:i + m] = torch.clamp(torch.searchsorted(cdf, u, right=True), max=distinct - 1).to(torch.int32)
        return out
    if kind == "normal":
        out = torch.empty(n, dtype=torch.int32, device=device)
        chunk = 1 << 24
        for i in range(0, n, chunk):
            m = min(chunk, n - i)
            x = torch.randn(m, generator=g, device=device, dtype=torch.float64) * (2.0 ** 28) + 2.0 ** 31
            out[i:i + m] = torch.clamp(torch.round(x), 0, 4294967295).to(torch.int64).to(torch.int32)
        return out
    raise ValueError(kind)


def host_sample(torch, col, m=1 << 20, seed=0):
    g = torch.Generator(device=col.device)
    g.manual_seed(seed)
    idx = torch.randint(0, col.numel(), (m,), generator=g, device=col.device)
    return np.sort(col[idx].cpu().numpy().view(np.uint32))


# ----------------------------------------------------------------------------
# CPU baseline: the reference's own CPU BinDex (oracle/_ref) when it was
# built, else the oracle's C restatement; timed on this host.
# ----------------------------------------------------------------------------

REF_N = 1 << 24


def reference_binary():
    p = os.path.join(ROOT, "oracle", "_ref", f"ref_bindex_{REF_N}")
    return p if os.access(p, os.X_OK) else None


def cpu_reference_run(cols_np, queries, repeats=3, max_seconds=60.0):
    """Time the reference BinDex query loop (build excluded) on a sample of
    REF_N rows; returns (seconds per query, kind, cores, detail)."""
    from rtscan_b200 import datagen as D
    ncols = len(cols_np)
    binary = reference_binary()
    if binary:
        with tempfile.TemporaryDirectory() as td:
            data = os.path.join(td, "cols.bin")
            D.write_columns(data, cols_np)
            cmdf = os.path.join(td, "cmd.txt")
            with open(cmdf, "w") as f:
                f.write(D.to_scan_cmd(queries, ncols))
            t0 = time.time()
            r = subprocess.run([binary, "-f", data, "-b", str(ncols), "-p", cmdf, "-r", str(repeats)],
                               capture_output=True, text=True, timeout=max_seconds + 240)
            if r.returncode != 0:
                raise RuntimeError("reference harness failed: " + r.stderr[-500:])
            ms = [float(l.split()[-1]) for l in r.stdout.splitlines() if l.startswith("query ")]
            eq = [l.split()[8] == "1" for l in r.stdout.splitlines() if l.startswith("query ")]
            return (sum(ms) / 1e3 / len(ms), "reference", 20,
                    {"queries": len(ms), "all_equal_scalar": all(eq), "wall_s": round(time.time() - t0, 1)})
    # fall back to the restated scalar filter (single thread)
    from oracle import oracle as O
    t0 = time.time()
    done = 0
    for q in queries:
        O.range_scan([cols_np[c] for c, _, _ in q], [t[1] for t in q], [t[2] for t in q])
        done += 1
        if time.time() - t0 > max_seconds:
            break
    return (time.time() - t0) / done, "port", 1, {"queries": done}


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------

def run(args):
    import torch
    import torch.distributed as dist

    import rtscan_b200 as R
    from rtscan_b200 import datagen as D

    world, rank, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = R.Context(local)
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream
    hbm_peak, peak_kind = peaks()

    n = args.nrows
    wl = args.workload
    if wl == "single":
        kinds = ["uniform"]
    elif wl == "multi":
        kinds = ["uniform"] * 4
    else:
        kinds = ["zipf1.1", "zipf1.3", "zipf1.5", "normal"]
    cols = [gpu_column(torch, k, n, 1000 * (rank + 1) + i, dev) for i, k in enumerate(kinds)]
    ctx.attach_columns([c.data_ptr() for c in cols], n)
    samples = [host_sample(torch, c, seed=7 + i) for i, c in enumerate(cols)]
    words = R.bitmap_words(n)
    stride = (words + 31) // 32 * 32

    rng = np.random.default_rng(42)
    if wl == "single":
        queries = [[(0, *D.range_for_selectivity(samples[0], 0.10))]]
    elif wl == "multi":
        q = []
        for c in range(4):
            sel = rng.uniform(0.05, 0.5)
            q.append((c, *D.range_for_selectivity(samples[c], sel, rng.uniform(sel / 2, 1 - sel / 2))))
        queries = [q]
    else:
        queries = D.batch_queries([s_ for s_ in samples], args.queries, seed=42)  # sample-based bounds
    nq = len(queries)
    out = torch.empty(nq * stride, dtype=torch.int32, device=dev)
    cnt = torch.zeros(nq, dtype=torch.int64, device=dev)

    used_cols = sorted({c for q in queries for c, _, _ in q})
    if wl == "batched":
        bytes_step = 4 * n * len(used_cols) + nq * n / 8
        launch = lambda: ctx.scan_batch_async(queries, out.data_ptr(), stride, cnt.data_ptr(), s)
    else:
        bytes_step = 4 * n * len(used_cols) + n / 8
        launch = lambda: ctx.scan_async(queries[0], out.data_ptr(), cnt.data_ptr(), s)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        launch()
    barrier()
    l0 = ctx.launches
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    barrier()
    ev[0].record(stream)
    for i in range(args.steps):
        launch()
        ev[i + 1].record(stream)
    barrier()
    clk = clocks.stop()
    launches = ctx.launches - l0
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item()) / args.steps

    # dominant kernel: the step is one launch of it on this stream
    kern_ms = statistics.median(per)
    achieved = bytes_step / (kern_ms * 1e-3) / 1e9

    # comparisons on rank 0's device
    extra = {}
    if wl == "multi":
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            ctx.scan_separate_async(queries[0], out.data_ptr(), cnt.data_ptr(), s)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.scan_separate_async(queries[0], out.data_ptr(), cnt.data_ptr(), s)
        e1.record(stream)
        torch.cuda.synchronize()
        sep_ms = e0.elapsed_time(e1) / args.steps
        extra["separate_passes_ms"] = round(sep_ms, 4)
        extra["fused_speedup_vs_separate"] = round(sep_ms / ms_step, 3)

    # e2e through the C-ABI with host buffers: columns uploaded from pinned
    # host memory and the result bitmap read back, every step.
    e2e_s = float("nan")
    if not args.no_e2e:
        host_cols = [c.cpu().pin_memory() for c in cols]
        host_np = [h.numpy().view(np.uint32) for h in host_cols]
        e2e_steps = max(2, min(args.steps, 5))
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ctx.load_columns(host_np)
            for q in queries[: (1 if wl != "batched" else nq)]:
                ctx.scan(q)
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        ctx.attach_columns([c.data_ptr() for c in cols], n)
    h2d = 4 * n * len(cols)
    d2h = (nq if wl == "batched" else 1) * (words * 4 + 8)

    gbs_total = bytes_step * world / (ms_step * 1e-3) / 1e9
    line = {
        "metric": METRIC,
        "value": round(gbs_total, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded, generated on device)",
        "config": {"workload": {"batched": "batched 1e8x4 skewed, 1024 queries", "single": "single-column 1e8 scan 10%",
                                "multi": "multi-column 1e8x4 conjunctive"}[wl],
                   "nrows_per_gpu": n, "ncols": len(cols), "queries_per_step": nq, "l2": "inputs larger than L2"},
        "queries_per_s": round(nq * world / (ms_step * 1e-3), 1),
        "rows_per_s": round(n * world / (ms_step * 1e-3), 1),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": None, "peak_kind": peak_kind},
        "e2e": {"value": round(bytes_step / e2e_s / 1e9 * world, 3), "unit": "GB/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "queries_per_s": round((nq if wl == 'batched' else 1) * world / e2e_s, 2)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    line.update(extra)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        m = REF_N
        cols_np = [c[:m].cpu().numpy().view(np.uint32).copy() for c in cols]
        qs = queries[: min(len(queries), 8)]
        sec, kind, cores, detail = cpu_reference_run(cols_np, qs)
        used = len({c for q in qs for c, _, _ in q})
        cpu_bytes = 4 * m * used / len(qs) * 0 + sum(4 * m * len({c for c, _, _ in q}) + m / 8 for q in qs) / len(qs)
        line["cpu_baseline"] = {"value": round(cpu_bytes / sec / 1e9, 3), "unit": "GB/s", "cores": cores,
                                "kind": kind, "queries_per_s": round(1.0 / sec, 2),
                                "sample": f"{m} rows x {len(cols)} cols, {len(qs)} queries of this workload",
                                **detail}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    """--impl reference: the reference's CPU path on this host (rank 0 only)."""
    world, rank, local = dist_env()
    if rank != 0:
        return
    import torch

    from rtscan_b200 import datagen as D
    m = REF_N
    wl = args.workload
    kinds = {"single": ["uniform"], "multi": ["uniform"] * 4}.get(wl, ["zipf1.1", "zipf1.3", "zipf1.5", "normal"])
    cols = [D.column(k, m, 1000 + i) for i, k in enumerate(kinds)]
    samples = [np.sort(c[np.random.default_rng(7).integers(0, m, size=1 << 18)]) for c in cols]
    rng = np.random.default_rng(42)
    if wl == "single":
        queries = [[(0, *D.range_for_selectivity(samples[0], 0.10))]]
    elif wl == "multi":
        queries = [[(c, *D.range_for_selectivity(samples[c], 0.2)) for c in range(4)]]
    else:
        queries = D.batch_queries(samples, 1024, seed=42)
    per_step = min(len(queries), 8)
    vals = []
    kind = cores = None
    for step in range(args.warmup + args.steps):
        qs = [queries[(step * per_step + i) % len(queries)] for i in range(per_step)]
        sec, kind, cores, detail = cpu_reference_run(cols, qs, repeats=1)
        if step >= args.warmup:
            b = sum(4 * m * len({c for c, _, _ in q}) + m / 8 for q in qs) / len(qs)
            vals.append((b / sec / 1e9, 1.0 / sec, sec))
        if step >= args.warmup + 1 and sum(v[2] for v in vals) * per_step > 120:
            break
    v = statistics.median(x[0] for x in vals)
    qps = statistics.median(x[1] for x in vals)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "GB/s", "n_gpus": world,
            "steps": len(vals), "warmup": args.warmup, "ms_per_step": round(1e3 * per_step / qps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded)",
            "config": {"workload": wl, "nrows": m, "ncols": len(cols), "queries_per_step": per_step},
            "queries_per_s": round(qps, 2),
            "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "kind": kind, "cores": cores,
                             "sample": f"{m} rows x {len(cols)} cols, {per_step} queries per step"},
            "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "single", "multi"])
    ap.add_argument("--nrows", type=int, default=100_000_000)
    ap.add_argument("--queries", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
