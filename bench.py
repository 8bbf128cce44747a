"""Benchmark driver: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|single|multi|q6] [--nrows N] [--queries Q]

Workloads (seeded synthetic data generated on the device; no dataset is read):
  batched  (default) 1e8 rows x 4 uint32 columns (zipf 1.1, 1.3, 1.5 over 2^20
           values and a rounded normal, mean 2^31, sd 2^28), 1024 queries
           touching 1-4 columns with log-uniform selectivity in [0.01%, 90%];
           one step = one batched call answering all queries (1024 bitmaps
           + counts).  Compared with one fused-scan launch per query, and at
           256 concurrent 4-column queries.
  single   1e8 rows x 1 uniform column, one 10%-selectivity range; one step
           = one fused scan launch.
  multi    1e8 rows x 4 uniform columns, one conjunctive query with
           per-column selectivity in [5%, 50%]; fused vs separate passes.
  q6       1e8 rows x 4 integer-coded columns shaped like TPC-H Q6
           (shipdate, discount, quantity, extendedprice); one step = one
           fused scan-and-aggregate (count and sum of price x discount over
           shipdate in 1994, discount 5-7, quantity < 24), no bitmap.
           Compared with the scan followed by the masked sum, and with the
           compaction of its bitmap to row ids.

The default batched line also carries the other configurations of the
scan, each timed with CUDA events on the launching stream beside its own
roofline fraction: `single_1e8` (the plain one-column 1e8-row scan at 10 %),
`sweep_1e8` (one-column queries at 0.1-90 % selectivity on a uniform 2^32
column and on 2^8- and 2^6-value columns, fused scan and BinDex) and
`multi_1e8` (2-, 3- and 4-column conjunctions, fused against separate
per-column passes plus AND).

`--gpus N` runs N ranks, one per GPU: under torchrun (WORLD_SIZE set) it
must equal the world size; without it, bench.py starts itself under
torch.distributed.run with N processes.  Each rank scans its own rows
(weak scaling, no collective on the data path) and answers the same
queries (rank 0's, broadcast); `value` is the aggregate over ranks and the
counts of the first query are summed over ranks with one all-reduce.
Timing: W warm-up steps, then K steps between CUDA events on the launching
stream, barrier + synchronize on both sides, max over ranks.  Inputs are
larger than L2 (400 MB per column).
"""
from __future__ import annotations

import argparse
import json
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
Q6_METRIC = "fused scan-and-aggregate GB/s vs HBM peak"
BATCH_KINDS = ["zipf1.1", "zipf1.3", "zipf1.5", "normal"]
# TPC-H Q6 shape, integer-coded: shipdate (yyyymmdd-like), discount (%),
# quantity, extendedprice (cents)
Q6_KINDS = ["range:19920101:19990101", "range:0:11", "range:1:51", "range:90000:10500000"]
Q6_TERMS = [(0, 19940101, 19950100), (1, 5, 7), (2, 0, 23)]


# ----------------------------------------------------------------------------
# environment
# ----------------------------------------------------------------------------

def dist_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def free_port():
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def launch_command(gpus, argv):
    """The torch.distributed.run command that runs this script as `gpus`
    ranks on one node (rendezvous on 127.0.0.1)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)] + list(argv)


def check_world(gpus):
    """None when this process is the run itself; else the command that
    starts `gpus` ranks.  A world size that disagrees with --gpus is an
    error, so that a line never reports fewer GPUs than were asked for."""
    if "WORLD_SIZE" in os.environ:
        world = int(os.environ["WORLD_SIZE"])
        if world != gpus:
            raise SystemExit(f"bench.py: --gpus {gpus} but WORLD_SIZE={world}")
        return None
    return launch_command(gpus, sys.argv[1:]) if gpus > 1 else None


def agree_queries(queries, world):
    """Rank 0's queries on every rank (one broadcast): all ranks answer the
    same queries on their own rows."""
    if world == 1:
        return queries
    import torch.distributed as dist
    box = [queries]
    dist.broadcast_object_list(box, src=0)
    return [[(int(c), int(lo), int(hi)) for c, lo, hi in q] for q in box[0]]


def host_info():
    """Host cores and CPU model of this machine (for the CPU baselines)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"host_cpus": os.cpu_count(), "cpu_model": model}


# DRAM traffic of a step from one ncu capture each (dram__bytes_read.sum +
# dram__bytes_write.sum of every launch of one step) beside that step's
# algorithmic bytes (columns read once, one bitmap written per query).  The
# timed workload's step is credited with the same traffic-to-bytes ratio
# (its launches read the columns and write the bitmaps in proportion) and
# `traffic` is that per launch, like `achieved`.  The batched step is the
# shared-position pre-pass and two 512-query passes: the pre-pass writes
# 8 B per row and pass (16 B) that the passes read back, traffic above the
# algorithmic bytes by design.
NCU_TRAFFIC = {
    "batched": {"kernels": "pre_kernel<4,1> + 2 x batch4_kernel<4,16,16,true>",
                "capture": "2e7 rows x 4 columns, 1024 queries: the three launches of one step",
                "bytes": (320.09e6 + 275.12e6) + (160.21e6 + 1221.65e6) + (160.61e6 + 1223.99e6),
                "step_bytes": 4 * 4 * 2e7 + 1024 * 2e7 / 8},
    "single": {"kernels": "scan_fused_kernel<1,1>", "capture": "1e8 rows x 1 column, one launch",
               "bytes": 408.9e6, "step_bytes": 4 * 1e8 + 1e8 / 8},
}


def step_traffic(wl, bytes_step, launches):
    """Traffic of the timed workload's step scaled from its capture."""
    cap = NCU_TRAFFIC.get(wl)
    if cap is None:
        return None
    t = cap["bytes"] / cap["step_bytes"] * bytes_step
    return {"bytes": round(t / launches / 1e9, 3), "unit": "GB per launch", "GB_per_step": round(t / 1e9, 3),
            "algorithmic_GB_per_step": round(bytes_step / 1e9, 3), "kernels": cap["kernels"],
            "capture": cap["capture"]}


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
# synthetic columns on the device (same distributions as rtscan_b200.datagen)
# ----------------------------------------------------------------------------

def gpu_column(torch, kind: str, n: int, seed: int, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if kind == "uniform":
        x = torch.randint(0, 1 << 32, (n,), generator=g, device=device, dtype=torch.int64)
        return x.to(torch.int32)  # two's-complement wrap keeps the uint32 bit pattern
    if kind.startswith("range:"):  # uniform integers in [a, b)
        a, b = (int(x) for x in kind.split(":")[1:])
        return torch.randint(a, b, (n,), generator=g, device=device, dtype=torch.int64).to(torch.int32)
    out = torch.empty(n, dtype=torch.int32, device=device)
    chunk = 1 << 24
    if kind.startswith("zipf"):
        s = float(kind[4:])
        distinct = 1 << 20
        ranks = torch.arange(1, distinct + 1, device=device, dtype=torch.float64)
        cdf = torch.cumsum(ranks.pow(-s), 0)
        cdf /= cdf[-1].clone()
        for i in range(0, n, chunk):
            m = min(chunk, n - i)
            u = torch.rand(m, generator=g, device=device, dtype=torch.float64)
            out[i:i + m] = torch.clamp(torch.searchsorted(cdf, u, right=True), max=distinct - 1).to(torch.int32)
        return out
    if kind == "normal":
        for i in range(0, n, chunk):
            m = min(chunk, n - i)
            x = torch.randn(m, generator=g, device=device, dtype=torch.float64) * (2.0 ** 28) + 2.0 ** 31
            out[i:i + m] = torch.clamp(torch.round(x), 0, 4294967295).to(torch.int64).to(torch.int32)
        return out
    raise ValueError(kind)


def host_sample(torch, col, m=1 << 18, seed=0):
    g = torch.Generator(device=col.device)
    g.manual_seed(seed)
    idx = torch.randint(0, col.numel(), (m,), generator=g, device=col.device)
    return np.sort(col[idx].cpu().numpy().view(np.uint32))


def make_queries(D, wl, samples, nq, seed=42):
    rng = np.random.default_rng(seed)
    if wl == "single":
        return [[(0, *D.range_for_selectivity(samples[0], 0.10))]]
    if wl == "q6":
        return [list(Q6_TERMS)]
    if wl == "multi":
        q = []
        for c in range(len(samples)):
            sel = rng.uniform(0.05, 0.5)
            q.append((c, *D.range_for_selectivity(samples[c], sel, rng.uniform(sel / 2, 1 - sel / 2))))
        return [q]
    return D.batch_queries(samples, nq, seed=seed)


def row_query_bytes(n, queries):
    """Algorithmic bytes of a workload per row and query: its step bytes
    (columns once per batch, one bitmap per query) over rows x queries.  A
    CPU sample of k of its queries over m rows is credited k * m times this,
    its share of the workload's bytes, so that GB/s compare like for like
    with the batched arm however small the sample."""
    return step_bytes(n, queries) / (n * len(queries))


def step_bytes(n, queries):
    """Algorithmic bytes of one step: every referenced column read once plus
    one bitmap written per query."""
    used = {c for q in queries for c, _, _ in q}
    return 4 * n * len(used) + len(queries) * n / 8


# ----------------------------------------------------------------------------
# CPU baseline: the reference's own CPU BinDex (oracle/_ref, compiled from
# the reference sources) when present, else the oracle's C restatement.
# ----------------------------------------------------------------------------

REF_N = 1 << 24      # rows of the CPU sample in the GPU arm's cpu_baseline
REF_THREADS = 20     # the reference's thread count (THREAD_NUM, bindex.cpp:27)


def reference_binary(n=REF_N):
    p = os.path.join(ROOT, "oracle", "_ref", f"ref_bindex_{n}")
    return p if os.access(p, os.X_OK) else None


def run_reference_harness(binary, cols_np, queries, checked=1, repeats=1, timeout=1800):
    """The reference's own CPU path once over `queries`: its BinDex build of
    every column, then its query loop (sieve + refine + AND merge per
    query, timed per query like the reference's timer 11).  The scalar
    filter checks the first `checked` queries.  Returns (build_ms, [scan_ms
    per query], [bindex == scalar for the checked queries])."""
    from rtscan_b200 import datagen as D
    with tempfile.TemporaryDirectory() as td:
        data = os.path.join(td, "cols.bin")
        D.write_columns(data, cols_np)
        cmdf = os.path.join(td, "cmd.txt")
        with open(cmdf, "w") as f:
            f.write(D.to_scan_cmd(queries, len(cols_np)))
        r = subprocess.run([binary, "-f", data, "-b", str(len(cols_np)), "-p", cmdf, "-r", str(repeats),
                            "-c", str(checked)], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference harness failed: " + r.stderr[-500:])
    build_ms = next(float(l.split()[1]) for l in r.stdout.splitlines() if l.startswith("build_ms"))
    q = [l.split() for l in r.stdout.splitlines() if l.startswith("query ")]
    if len(q) != len(queries):
        raise RuntimeError(f"reference harness answered {len(q)} of {len(queries)} queries")
    return build_ms, [float(x[-1]) for x in q], [x[7] == "1" for x in q if x[7] != "-1"]


def cpu_reference_run(cols_np, queries, max_seconds=60.0):
    """Seconds per query of the reference BinDex query loop (index build
    excluded) on REF_N-row columns; returns (seconds, kind, cores, detail)."""
    binary = reference_binary(len(cols_np[0]))
    if binary:
        t0 = time.time()
        build_ms, ms, eq = run_reference_harness(binary, cols_np, queries, checked=1, repeats=3)
        return (sum(ms) / 1e3 / len(ms), "reference", REF_THREADS,
                {"queries": len(ms), "reference_bindex_equals_scalar": all(eq), "index_build_ms": round(build_ms),
                 "wall_s": round(time.time() - t0, 1)})
    from oracle import oracle as O
    t0 = time.time()
    done = 0
    for q in queries:
        O.range_scan([cols_np[c] for c, _, _ in q], [t[1] for t in q], [t[2] for t in q])
        done += 1
        if time.time() - t0 > max_seconds:
            break
    return (time.time() - t0) / done, "port", 1, {"queries": done}


def cpu_sample_columns(kinds, m):
    from rtscan_b200 import datagen as D
    out = []
    for i, k in enumerate(kinds):
        if k.startswith("range:"):
            a, b = (int(x) for x in k.split(":")[1:])
            out.append(np.random.default_rng(1000 + i).integers(a, b, m).astype(np.uint32))
        else:
            out.append(D.column(k, m, 1000 + i))
    return out


def q6_cpu_port(kinds, terms):
    """The q6 step restated in numpy (one thread) on REF_N rows: the
    reference has no aggregate step to time."""
    cols = cpu_sample_columns(kinds, REF_N)
    t0 = time.perf_counter()
    reps = 0
    while True:
        hit = np.ones(REF_N, bool)
        for c, lo, hi in terms:
            hit &= (cols[c] >= lo) & (cols[c] <= hi)
        total = int(np.sum(cols[3][hit].astype(np.uint64) * cols[1][hit].astype(np.uint64)))
        reps += 1
        if time.perf_counter() - t0 > 3.0:
            break
    sec = (time.perf_counter() - t0) / reps
    return {"value": round(4 * REF_N * len(cols) / sec / 1e9, 3), "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": f"{REF_N} rows x {len(cols)} columns, numpy restatement of the q6 step "
                      f"({reps} repetitions; sum {total})"}


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------

def run(args):
    import torch
    import torch.distributed as dist

    import rtscan_b200 as R
    from rtscan_b200 import datagen as D

    world, rank, local = dist_env()
    if world > 1:
        import datetime
        # NCCL's communicator log shows the ranks of a scaling run
        os.environ.setdefault("NCCL_DEBUG", "INFO")
        os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = R.Context(local)
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream
    hbm_peak, peak_kind = peaks()

    n = args.nrows
    wl = args.workload
    kinds = {"single": ["uniform"], "multi": ["uniform"] * 4, "q6": Q6_KINDS}.get(wl, BATCH_KINDS)
    cols = [gpu_column(torch, k, n, 1000 * (rank + 1) + i, dev) for i, k in enumerate(kinds)]
    ctx.attach_columns([c.data_ptr() for c in cols], n)
    samples = [host_sample(torch, c, seed=7 + i) for i, c in enumerate(cols)]
    # host copy of the first rows of every column: the CPU baseline's sample
    cpu_cols = [c[:min(REF_N, n)].cpu().numpy().view(np.uint32).copy() for c in cols] \
        if rank == 0 and world == 1 and not args.no_cpu_baseline and wl != "q6" else None
    queries = agree_queries(make_queries(D, wl, samples, args.queries), world)
    pq = R.prepare(queries)
    nq = len(queries)
    words = R.bitmap_words(n)
    stride = (words + 31) // 32 * 32
    out = torch.empty(nq * stride, dtype=torch.int32, device=dev)
    cnt = torch.zeros(nq, dtype=torch.int64, device=dev)
    bytes_step = step_bytes(n, queries) if wl != "q6" else 4 * n * len(cols)
    agg_cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    agg_sum = torch.zeros(2, dtype=torch.int64, device=dev)
    tuned = None
    if wl == "batched" and not args.no_autotune:
        tuned = ctx.autotune_batch(pq)  # launch shape for this table and batch (outside the timed region)
    if wl == "batched":
        launch = lambda: ctx.scan_batch_async(pq, out.data_ptr(), stride, cnt.data_ptr(), s)
    elif wl == "q6":
        launch = lambda: ctx.scan_aggregate_async(queries[0], 3, 1, agg_cnt.data_ptr(), agg_sum.data_ptr(), s)
    else:
        launch = lambda: ctx.scan_async(queries[0], out.data_ptr(), cnt.data_ptr(), s)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def timed(fn, steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record(stream)
        for i in range(steps):
            fn()
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        return [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)], ev[0].elapsed_time(ev[-1])

    for _ in range(args.warmup):
        launch()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = ctx.launches
    barrier()
    per, total_ms = timed(launch, args.steps)
    barrier()
    launches = ctx.launches - l0
    clk = clocks.stop()
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item()) / args.steps
    kern_launches = max(1, launches // args.steps)
    ms_launch = statistics.median(per) / kern_launches
    achieved = (bytes_step / kern_launches) / (ms_launch * 1e-3) / 1e9
    tr = step_traffic(wl, bytes_step, kern_launches)

    extra = {}
    if wl == "multi":
        for _ in range(3):
            ctx.scan_separate_async(queries[0], out.data_ptr(), cnt.data_ptr(), s)
        per_sep, _ = timed(lambda: ctx.scan_separate_async(queries[0], out.data_ptr(), cnt.data_ptr(), s), args.steps)
        sep_ms = statistics.median(per_sep)
        extra["separate_passes_ms"] = round(sep_ms, 4)
        extra["fused_speedup_vs_separate"] = round(sep_ms / statistics.median(per), 3)
    if wl == "batched":
        # the same batch prepared once and replayed as one CUDA graph per step
        pb = ctx.prepare_batch(pq, out.data_ptr(), stride, cnt.data_ptr())
        pb.launch(s)
        per_g, _ = timed(lambda: pb.launch(s), args.steps)
        extra["graph_replay_ms_per_step"] = round(statistics.median(per_g), 4)
        pb.release()
    if wl == "q6":
        extra.update(q6_legs(torch, R, ctx, queries[0], n, out, cnt, s, timed, statistics.median(per)))
    if world > 1:
        from rtscan_b200 import shard as SH
        extra["global_match_count_q0"] = int(SH.all_reduce_counts(cnt[:1].cpu().numpy())[0])
    if wl == "batched" and not args.no_compare:
        each = lambda: ctx.scan_each_async(pq, out.data_ptr(), stride, cnt.data_ptr(), s)
        each()
        per_each, _ = timed(each, 2)
        each_ms = statistics.median(per_each)
        extra["one_query_per_launch_ms"] = round(each_ms, 3)
        extra["batched_speedup_vs_one_per_launch"] = round(each_ms / statistics.median(per), 2)
        # north-star comparison: 256 concurrent 4-column queries
        q4 = D.batch_queries(samples, 256, seed=7, min_cols=4, max_cols=4)
        pq4 = R.prepare(q4)
        b4 = lambda: ctx.scan_batch_async(pq4, out.data_ptr(), stride, cnt.data_ptr(), s)
        e4 = lambda: ctx.scan_each_async(pq4, out.data_ptr(), stride, cnt.data_ptr(), s)
        b4(); e4()
        pb4, _ = timed(b4, 3)
        pe4, _ = timed(e4, 2)
        mb4, me4 = statistics.median(pb4), statistics.median(pe4)
        extra["q256x4col"] = {"batched_ms": round(mb4, 3), "one_per_launch_ms": round(me4, 3),
                              "batched_qps": round(256 / (mb4 * 1e-3), 1),
                              "one_per_launch_qps": round(256 / (me4 * 1e-3), 1),
                              "speedup": round(me4 / mb4, 2)}

    if wl == "batched" and not args.no_legs:
        lclk = ClockSampler(local)
        lclk.start()
        extra["single_1e8"] = single_leg(torch, R, D, dev, args.nrows, hbm_peak)
        extra["multi_1e8"] = multi_leg(torch, R, D, dev, args.nrows, hbm_peak)
        extra["sweep_1e8"] = sweep_leg(torch, R, D, dev, args.nrows, hbm_peak)
        extra["legs_clocks"] = lclk.stop()

    # e2e through the C-ABI with host buffers: the step's columns uploaded
    # from pinned host memory and every result bitmap + count read back.
    e2e = None
    if not args.no_e2e and wl == "q6":
        e2e = q6_e2e(torch, R, local, cols, queries[0], bytes_step, world, dev, barrier)
    elif not args.no_e2e:
        host_cols = [c.cpu().pin_memory() for c in cols]
        host_np = [h.numpy().view(np.uint32) for h in host_cols]
        hb = torch.empty((nq, stride), dtype=torch.int32).pin_memory()
        hb_np = hb.numpy().view(np.uint32)
        ctx.scan_batch_host(host_np, pq, hb_np, stride)  # warm-up (allocates device buffers)
        reps = 5
        barrier()
        calls = []
        for _ in range(reps):  # each call blocks until its bitmaps and counts are on the host
            t0 = time.perf_counter()
            _, counts = ctx.scan_batch_host(host_np, pq, hb_np, stride)
            calls.append(time.perf_counter() - t0)
        e2e_s = statistics.median(calls)
        et = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e2e_s = float(et.item())
        h2d_b, d2h_b = ctx.host_transfer_bytes()
        e2e = {"value": round(bytes_step * world / e2e_s / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": int(h2d_b), "d2h_bytes_per_step": int(d2h_b),
               "dense_d2h_bytes_per_step": int(nq * (R.bitmap_words(n) * 4 + 8)),
               "queries_per_s": round(nq * world / e2e_s, 2), "ms_per_step": round(e2e_s * 1e3, 2),
               "calls_ms": [round(c * 1e3, 1) for c in calls], "timing": "median of 5 calls after one warm-up",
               "api": "rts_scan_batch_host"}
        # the box's own pinned device-to-host copy rate (the e2e step's floor:
        # its bitmaps cannot leave the device faster)
        m = min(out.numel(), hb.numel(), 1 << 29)
        src, dst = out.view(-1)[:m], hb.view(-1)[:m]
        dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        d2h = 3 * 4 * m / (e0.elapsed_time(e1) * 1e-3) / 1e9
        e2e["pinned_d2h_GB_s"] = round(d2h, 2)
        e2e["d2h_floor_ms"] = round(e2e["d2h_bytes_per_step"] / d2h / 1e6, 2)
        del hb, host_cols

    gbs_total = bytes_step * world / (ms_step * 1e-3) / 1e9
    line = {
        "metric": METRIC if wl != "q6" else Q6_METRIC,
        "value": round(gbs_total, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "step_ms": {"min": round(min(per), 4), "median": round(statistics.median(per), 4), "max": round(max(per), 4)},
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded, generated on device)",
        "config": workload_config(wl, n, nq, kinds),
        "queries_per_s": round(nq * world / (ms_step * 1e-3), 1),
        "rows_per_s": round(n * world / (ms_step * 1e-3), 1),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4),
                     "traffic": (tr or {}).get("bytes"), "traffic_unit": "GB per launch", "traffic_detail": tr,
                     "peak_kind": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                     "kernel_launches_per_step": kern_launches},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if wl == "batched":
        line["batch_config"] = ctx.batch_config()
        line["batch_config"]["source"] = "autotuned" if tuned else "default"
        if tuned:
            line["batch_config"]["autotune"] = ctx.autotune_report()
    line.update(extra)

    if args.bindex_io and rank == 0:
        line["bindex_io"] = bindex_io_leg(torch, R, dev, args.bindex_io)
    if args.bindex_query and rank == 0:
        line["bindex_query"] = sweep_leg(torch, R, D, dev, args.bindex_query, hbm_peak)

    if wl == "batched" and args.pass_sweep:
        line["pass_sweep"] = pass_sweep(torch, R, D, dev, rank, args.pass_sweep)

    if wl == "batched" and not args.no_serve:
        del out, cnt
        ctx.attach_columns([c.data_ptr() for c in cols[:1]], n)
        del cols
        torch.cuda.empty_cache()
        line["served"] = served_leg(torch, R, D, ctx, dev, rank, args)
        rates = line["served"]["rates"]
        ref = min(rates, key=lambda r: abs(r["offered_qps"] - 5000)) if rates else None
        if ref:
            line["served_p50_ms"] = ref["p50_ms"]
            line["served_p99_ms"] = ref["p99_ms"]
            line["served_at_qps"] = ref["offered_qps"]

    if rank == 0 and world == 1 and not args.no_cpu_baseline and wl == "q6":
        line["cpu_baseline"] = q6_cpu_port(kinds, queries[0])
    elif rank == 0 and world == 1 and not args.no_cpu_baseline:
        m = min(REF_N, n)
        cols_np = cpu_cols
        qs = queries[:16]
        sec, kind, cores, detail = cpu_reference_run(cols_np, qs)
        bprq = row_query_bytes(n, queries)
        line["cpu_baseline"] = {"value": round(m * bprq / sec / 1e9, 3), "unit": "GB/s", "cores": cores,
                                "kind": kind, "queries_per_s": round(m / n / sec, 3),
                                "queries_per_s_sample": round(1.0 / sec, 2),
                                "sample": f"the first {m} rows of this workload's {len(cols_np)} columns and its "
                                          f"first {len(qs)} queries (reference BinDex query loop, "
                                          f"{cores} threads, index build excluded); credited {bprq:.4f} B per "
                                          "row and query, the workload's bytes share; queries_per_s scaled "
                                          "to the workload's rows (the full-size reference run is "
                                          "`--impl reference`)",
                                **host_info(), **detail}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def bindex_io_leg(torch, R, dev, n, K=128):
    """BinDex of one n-row zipf 1.3 column: build on the device vs save to a
    file and load it back (the load checks checksums and the sorted order
    against the column)."""
    col = gpu_column(torch, "zipf1.3", n, 99, dev)
    c = R.Context(dev.index or 0)
    c.attach_columns([col.data_ptr()], n)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    c.build_bindex(0, K)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "col0.bdx")
        t0 = time.perf_counter()
        c.save_bindex(0, path)
        save_s = time.perf_counter() - t0
        size = os.path.getsize(path)
        c.drop_bindex(0)
        t0 = time.perf_counter()
        c.load_bindex(0, path)
        load_s = time.perf_counter() - t0
    c.close()
    return {"rows": n, "K": K, "file_MB": round(size / 1e6, 1), "build_ms": round(build_s * 1e3, 1),
            "save_ms": round(save_s * 1e3, 1), "load_ms": round(load_s * 1e3, 1),
            "load_GB_s": round(size / load_s / 1e9, 2)}


def event_median(torch, fn, reps=9, warm=3):
    """Median CUDA-event time (ms) of fn() on the current stream, each
    repetition bracketed by its own events and a synchronize."""
    st = torch.cuda.current_stream()
    for _ in range(warm):
        fn()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def graph_per_call(torch, fn_on, calls=20, reps=7):
    """Device time (ms) per call of fn_on(stream handle) with `calls` calls
    captured in one CUDA graph (after the caller's warm-up calls) and the
    graph replayed between two CUDA events: the calls' kernels back to back
    without host work or launch gaps between them, median over `reps`."""
    st = torch.cuda.current_stream()
    cs = torch.cuda.Stream()
    cs.wait_stream(st)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=cs):
        for _ in range(calls):
            fn_on(cs.cuda_stream)
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        g.replay()
        e1.record(st)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / calls)
    del g
    return statistics.median(ts)


def stream_per_call(torch, fn, calls=20, reps=5):
    """Device time (ms) per call of fn() issued `calls` times back to back
    between two CUDA events (host planning overlaps the device work, as in
    a stream of queries), median over `reps` such runs."""
    st = torch.cuda.current_stream()
    for _ in range(3):
        fn()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(calls):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / calls)
    return statistics.median(ts)


def single_leg(torch, R, D, dev, n, hbm_peak):
    """The plain single-query scan: one uniform 2^32 column of n rows, one
    range at 10 % selectivity ([q45, q55] of a sample), one fused-scan launch.
    Bytes: 4 B per row read + the bitmap written (+ the 8-byte count)."""
    col = gpu_column(torch, "uniform", n, 42, dev)
    c = R.Context(dev.index or 0)
    c.attach_columns([col.data_ptr()], n)
    terms = [(0, *D.range_for_selectivity(host_sample(torch, col), 0.10))]
    bm = torch.empty(R.bitmap_words(n), dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    ms = event_median(torch, lambda: c.scan_async(terms, bm.data_ptr(), cnt.data_ptr(), s), reps=15)
    nbytes = 4 * n + R.bitmap_words(n) * 4 + 8
    gbs = nbytes / (ms * 1e-3) / 1e9
    out = {"workload": f"{n:.3g} rows x 1 uniform column, one 10 % range", "kernel": "scan_fused_kernel<1,1>",
           "launches": 1, "lo": terms[0][1], "hi": terms[0][2], "selectivity": round(int(cnt.item()) / n, 5),
           "ms": round(ms, 4), "rows_per_s": round(n / (ms * 1e-3), 1), "bytes": nbytes,
           "GB_s": round(gbs, 1), "frac": round(gbs / hbm_peak, 4), "peak": hbm_peak}
    c.close()
    return out


def multi_leg(torch, R, D, dev, n, hbm_peak, seed=3):
    """Conjunctions over the first 2, 3 and 4 of four independently seeded
    uniform 2^32 columns, per-column selectivity uniform in [5 %, 50 %]:
    the fused scan (one launch: every column read once, one bitmap write)
    against separate per-column passes plus AND passes, bitmaps compared.
    Bytes: fused 4cN + N/8; separate c(4N + N/8) + (c-1) 3N/8."""
    cols = [gpu_column(torch, "uniform", n, 61 + i, dev) for i in range(4)]
    smp = [host_sample(torch, x, seed=3 + i) for i, x in enumerate(cols)]
    c = R.Context(dev.index or 0)
    c.attach_columns([x.data_ptr() for x in cols], n)
    rng = np.random.default_rng(seed)
    words = R.bitmap_words(n)
    a = torch.empty(words, dtype=torch.int32, device=dev)
    b = torch.empty(words, dtype=torch.int32, device=dev)
    ca = torch.zeros(1, dtype=torch.int64, device=dev)
    cb = torch.zeros(1, dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    res = []
    for k in (2, 3, 4):
        terms = []
        for col in range(k):
            sel = rng.uniform(0.05, 0.5)
            terms.append((col, *D.range_for_selectivity(smp[col], sel, rng.uniform(sel / 2, 1 - sel / 2))))
        tf = event_median(torch, lambda: c.scan_async(terms, a.data_ptr(), ca.data_ptr(), s))
        ts = event_median(torch, lambda: c.scan_separate_async(terms, b.data_ptr(), cb.data_ptr(), s))
        fb = 4 * k * n + words * 4
        sb = k * (4 * n + words * 4) + (k - 1) * 3 * words * 4
        res.append({"columns": k, "selectivity": round(int(ca.item()) / n, 6),
                    "fused_ms": round(tf, 4), "fused_GB_s": round(fb / (tf * 1e-3) / 1e9, 1),
                    "fused_frac": round(fb / (tf * 1e-3) / 1e9 / hbm_peak, 4),
                    "separate_ms": round(ts, 4), "separate_GB_s": round(sb / (ts * 1e-3) / 1e9, 1),
                    "fused_speedup_vs_separate": round(ts / tf, 3),
                    "equal": bool(torch.equal(a, b)) and int(ca.item()) == int(cb.item())})
    c.close()
    return {"workload": f"{n:.3g} rows x 2-4 uniform columns, one conjunctive query", "queries": res}


SWEEP_SELS = (0.001, 0.01, 0.10, 0.50, 0.90)


def domain_range(domain, sel):
    """The central run of values of a uniform [0, domain) column whose share
    is nearest to `sel` (at least one value)."""
    w = max(1, min(domain, int(round(sel * domain))))
    lo = (domain - w) // 2
    return lo, lo + w - 1


def sweep_leg(torch, R, D, dev, n, hbm_peak, K=128):
    """One-column queries of the selectivity sweep, each through the fused
    scan and through the BinDex (built once per column, K areas), bitmaps
    compared: a uniform 2^32 column at 0.1/1/10/50/90 % (bounds at sample
    quantiles) and columns of 256 and 64 distinct values (central value runs
    nearest those shares; the achieved selectivity is reported).  Times are
    the device time per query in a stream of 20 back-to-back calls (`_us`,
    the basis of GB/s and frac), the latency of one call alone
    (`_latency_us`, which includes the host's planning and launch of that
    call while the device waits), and for the BinDex the device time per
    query of 20 calls replayed as one CUDA graph (`bindex_graph_us` and its
    `bindex_graph_frac`: the query's kernels without the gaps between
    launches from the host, which a stream of sub-20-us queries shows).  Fused bytes: 4N + N/8.  BinDex bytes are those of the plan its planner picks,
    from exact ranks, costed as bindex_query (csrc/bindex.cu) costs it: the
    result write, every filter vector read, and 12 B per re-tested row (its
    row id, its gathered value and its result word); a query whose matches
    are cheaper to re-test than to sieve starts from zero and re-tests those
    rows only (refine_only)."""
    s = torch.cuda.current_stream()
    words = R.bitmap_words(n)
    bm = torch.empty(words, dtype=torch.int32, device=dev)
    ref = torch.empty_like(bm)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    res = {"rows": n, "K": K, "queries": []}
    fused_bytes = 4 * n + words * 4
    for kind, seed in (("uniform", 31), ("range:0:256", 41), ("range:0:64", 51)):
        col = gpu_column(torch, kind, n, seed, dev)
        c = R.Context(dev.index or 0)
        c.attach_columns([col.data_ptr()], n)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c.build_bindex(0, K)
        torch.cuda.synchronize()
        build_ms = (time.perf_counter() - t0) * 1e3
        srt = torch.sort(col.to(torch.int64) & 0xFFFFFFFF).values
        lower = lambda v: int(torch.searchsorted(srt, torch.tensor([v], device=dev)).item())
        fr = [lower(int(srt[k * (n // K)].item())) for k in range(K)]  # rank of area k's start value

        def nearest(est):  # the planner's filter vector (or constant) nearest to rank est
            best, bd = (-1, 0), est
            if n - est < bd:
                best, bd = (K - 1, n), n - est
            for j in range(1, K):
                if abs(fr[j] - est) < bd:
                    best, bd = (j - 1, fr[j]), abs(fr[j] - est)
            return best

        if kind == "uniform":
            smp = host_sample(torch, col)
            qs = [(sel, *D.range_for_selectivity(smp, sel)) for sel in SWEEP_SELS]
        else:
            dom = int(kind.split(":")[2])
            qs = [(sel, *domain_range(dom, sel)) for sel in SWEEP_SELS]
            qs = [q for i, q in enumerate(qs) if i == 0 or q[1:] != qs[i - 1][1:]]
        for sel, lo, hi in qs:
            terms = [(0, lo, hi)]
            r_lo = lower(lo) if lo > 0 else 0
            r_hi = lower(hi + 1) if hi < 0xFFFFFFFF else n
            refine, fv_reads = 0, 0
            for has, r in ((lo > 0, r_lo), (hi < 0xFFFFFFFF, r_hi)):
                if has:
                    k, rk = nearest(r)
                    refine += abs(rk - r)
                    fv_reads += 0 <= k < K - 1
            match = max(0, r_hi - r_lo)
            sieve_cost = n / 8 * (1 + fv_reads) + refine * 40.0
            cand_cost = n / 8 + (match + 2048) * 40.0
            refine_only = cand_cost < sieve_cost
            nbytes = n / 8 + match * 12 if refine_only else n / 8 * (1 + fv_reads) + refine * 12
            bq_on = lambda st: c.bindex_scan_async(terms, bm.data_ptr(), cnt.data_ptr(), st)
            bq = lambda: bq_on(s.cuda_stream)
            fq = lambda: c.scan_async(terms, ref.data_ptr(), cnt.data_ptr(), s.cuda_stream)
            lat_b = event_median(torch, bq, reps=7)
            t_b = stream_per_call(torch, bq)
            g_b = graph_per_call(torch, bq_on)
            hits = int(cnt.item())
            lat_f = event_median(torch, fq, reps=7)
            t_f = stream_per_call(torch, fq)
            fgbs = fused_bytes / (t_f * 1e-3) / 1e9
            res["queries"].append({
                "column": kind, "target": sel, "lo": lo, "hi": hi, "selectivity": round(hits / n, 5),
                "fused_us": round(t_f * 1e3, 1), "fused_latency_us": round(lat_f * 1e3, 1),
                "fused_GB_s": round(fgbs, 1), "fused_frac": round(fgbs / hbm_peak, 4),
                "bindex_us": round(t_b * 1e3, 1), "bindex_latency_us": round(lat_b * 1e3, 1),
                "bindex_rows_per_s": round(n / (t_b * 1e-3), 1),
                "bindex_plan": "refine_only" if refine_only else "sieve",
                "bindex_refined_rows": match if refine_only else refine, "bindex_bytes_MB": round(nbytes / 1e6, 2),
                "bindex_GB_s": round(nbytes / (t_b * 1e-3) / 1e9, 1),
                "bindex_frac": round(nbytes / (t_b * 1e-3) / 1e9 / hbm_peak, 4),
                "bindex_graph_us": round(g_b * 1e3, 1),
                "bindex_graph_frac": round(nbytes / (g_b * 1e-3) / 1e9 / hbm_peak, 4),
                "equal": bool(torch.equal(bm, ref)) and hits == int(cnt.item())})
        res.setdefault("bindex_build_ms", {})[kind] = round(build_ms, 1)
        c.close()
        del col, srt
        torch.cuda.empty_cache()
    return res


def q6_legs(torch, R, ctx, terms, n, out, cnt, s, timed, fused_ms):
    """The q6 step the long way (scan to a bitmap, then the masked sum), and
    the compaction of that bitmap to row ids, each timed like the step."""
    dev = out.device
    sm = torch.zeros(2, dtype=torch.int64, device=dev)
    rc = torch.zeros(1, dtype=torch.int64, device=dev)
    bm = out.data_ptr()

    def two_pass():
        ctx.scan_async(terms, bm, cnt.data_ptr(), s)
        ctx.bitmap_sum_async(bm, 3, 1, sm.data_ptr(), s)
    two_pass()
    per2, _ = timed(two_pass, 5)
    hits = int(cnt[0].item())
    rows = torch.empty(max(1, hits), dtype=torch.int32, device=dev)
    compact = lambda: ctx.bitmap_rows_async(bm, n, rows.data_ptr(), hits, rc.data_ptr(), s)
    compact()
    perc, _ = timed(compact, 5)
    msum = lambda: ctx.bitmap_sum_async(bm, 3, 1, sm.data_ptr(), s)
    msum()
    pers, _ = timed(msum, 5)
    m2, mc, ms = statistics.median(per2), statistics.median(perc), statistics.median(pers)
    words = (n + 31) // 32
    return {"hits": hits,
            "scan_then_masked_sum_ms": round(m2, 4), "fused_speedup_vs_two_pass": round(m2 / fused_ms, 3),
            "masked_sum": {"ms": round(ms, 4), "GB_s": round((words * 4 + 8 * n) / (ms * 1e-3) / 1e9, 1),
                           "bytes": "bitmap + 2 columns"},
            "bitmap_to_rows": {"ms": round(mc, 4), "rows": hits,
                               "GB_s": round((2 * words * 4 + 4 * hits) / (mc * 1e-3) / 1e9, 1),
                               "bytes": "bitmap twice + 4 per row id"}}


def q6_e2e(torch, R, local, cols, terms, bytes_step, world, dev, barrier):
    """q6 through the public API from host memory: upload the 4 pinned
    columns into a context, run the fused scan-and-aggregate, read the count
    and sum back."""
    host = [c.cpu().pin_memory().numpy().view(np.uint32) for c in cols]
    c2 = R.Context(local)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    sm = torch.zeros(2, dtype=torch.int64, device=dev)

    def step():
        c2.load_columns(host)
        c2.scan_aggregate_async(terms, 3, 1, cnt.data_ptr(), sm.data_ptr(), 0)
        return cnt.cpu(), sm.cpu()
    step()
    reps = 3
    barrier()
    t0 = time.perf_counter()
    for _ in range(reps):
        step()
    e_s = (time.perf_counter() - t0) / reps
    c2.close()
    return {"value": round(bytes_step * world / e_s / 1e9, 3), "unit": "GB/s",
            "h2d_bytes_per_step": int(bytes_step), "d2h_bytes_per_step": 24,
            "ms_per_step": round(e_s * 1e3, 2), "api": "rts_load_columns + rts_scan_aggregate_async"}


SERVE_KINDS = ["uniform", "uniform", "zipf1.3", "zipf1.3"]


def pass_sweep(torch, R, D, dev, rank, n, sizes=(1, 4, 16, 64, 128, 256, 512)):
    """Kernel time of one pass of each size over an n-row table of the served
    kinds (one server segment): a prepared batch (CUDA graph) replayed 7
    times, median CUDA-event time on the launching stream."""
    cols = [gpu_column(torch, k, n, 7000 * (rank + 1) + i, dev) for i, k in enumerate(SERVE_KINDS)]
    samples = [host_sample(torch, c, seed=21 + i) for i, c in enumerate(cols)]
    ctx = R.Context(dev.index or 0)
    ctx.attach_columns([c.data_ptr() for c in cols], n)
    stride = (R.bitmap_words(n) + 31) // 32 * 32
    s = torch.cuda.current_stream()
    out = []
    for nq in sizes:
        qs = D.batch_queries(samples, nq, seed=nq)
        bm = torch.empty(nq * stride, dtype=torch.int32, device=dev)
        cnt = torch.zeros(nq, dtype=torch.int64, device=dev)
        pb = ctx.prepare_batch(qs, bm.data_ptr(), stride, cnt.data_ptr())
        for _ in range(3):
            pb.launch(s.cuda_stream)
        ts = []
        for _ in range(7):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            pb.launch(s.cuda_stream)
            e1.record(s)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        pb.release()
        ms = statistics.median(ts)
        out.append({"queries": nq, "us": round(1e3 * ms, 1), "us_per_query": round(1e3 * ms / nq, 2)})
        del bm, cnt
    ctx.close()
    del cols
    return {"rows": n, "kinds": SERVE_KINDS, "passes": out}


def served_leg(torch, R, D, ctx, dev, rank, args):
    """Served scan: a resident 2^28-row x 4-column table
    (2 uniform + 2 zipf 1.3 columns, 4 GiB), open-loop Poisson arrivals at
    several rates of queries over 1-4 columns with log-uniform selectivity,
    answered by the continuous-batching server; plus a burst of 256
    concurrent 4-column queries.  Latency is submit-to-done per request."""
    n = args.serve_rows
    cols = [gpu_column(torch, k, n, 5000 * (rank + 1) + i, dev) for i, k in enumerate(SERVE_KINDS)]
    ctx.attach_columns([c.data_ptr() for c in cols], n)
    samples = [host_sample(torch, c, seed=11 + i) for i, c in enumerate(cols)]
    out = {"table": f"{n} rows x {len(cols)} columns ({', '.join(SERVE_KINDS)})", "segment_rows": 1 << 23,
           "max_active": 1024, "rates": []}
    seconds = args.serve_seconds
    with R.Server(ctx, max_active=1024, segment_rows=1 << 23) as srv:
        # warm-up
        srv.replay(D.batch_queries(samples, 200, seed=1), np.linspace(0, 0.05, 200))
        for rate in args.serve_rates:
            rate = int(rate) if float(rate).is_integer() else rate
            nq = max(1, int(rate * seconds))
            qs = R.prepare(D.batch_queries(samples, nq, seed=int(rate)))
            arr = np.cumsum(np.random.default_rng(int(rate)).exponential(1.0 / rate, size=nq))
            st0 = srv.stats()
            t0 = time.perf_counter()
            lat = srv.replay(qs, arr)
            wall = time.perf_counter() - t0
            st1 = srv.stats()
            ok = lat[lat >= 0]
            steps, plans = st1["steps"] - st0["steps"], st1["plans"] - st0["plans"]
            out["rates"].append({"offered_qps": rate, "queries": nq, "achieved_qps": round(len(ok) / wall, 1),
                                 "rejected": int((lat < 0).sum()),
                                 "p50_ms": round(float(np.percentile(ok, 50)), 3),
                                 "p99_ms": round(float(np.percentile(ok, 99)), 3),
                                 "p999_ms": round(float(np.percentile(ok, 99.9)), 3),
                                 # the worker's steps (one segment each) and plans in the replay, and the
                                 # host time of a plan: planning slower than a step bounds the server
                                 "steps": steps, "plans": plans,
                                 "plan_ms_mean": round((st1["plan_ms_total"] - st0["plan_ms_total"]) / max(plans, 1), 3),
                                 "ms_per_step": round(wall * 1e3 / max(steps, 1), 3)})
        # the highest offered rate the server kept up with: every request
        # admitted (none rejected) and completions within 2 % of the offer
        kept = [r for r in out["rates"] if r["rejected"] == 0 and r["achieved_qps"] >= 0.98 * r["offered_qps"]]
        if kept:
            top = max(kept, key=lambda r: r["offered_qps"])
            out["max_sustained"] = {k: top[k] for k in ("offered_qps", "achieved_qps", "p50_ms", "p99_ms", "p999_ms")}
        over = [r for r in out["rates"] if r not in kept]
        if over:
            out["first_overloaded"] = min(over, key=lambda r: r["offered_qps"])["offered_qps"]
        q4 = R.prepare(D.batch_queries(samples, 256, seed=4, min_cols=4, max_cols=4))
        t0 = time.perf_counter()
        lat = srv.replay(q4, np.zeros(256))
        wall = time.perf_counter() - t0
        out["burst_256x4col"] = {"p50_ms": round(float(np.percentile(lat, 50)), 3),
                                 "p99_ms": round(float(np.percentile(lat, 99)), 3),
                                 "qps": round(256 / wall, 1)}
    del cols
    return out


def workload_config(wl, n, nq, kinds):
    """The `config` object of both arms' lines: the workload a step stands
    for (the reference arm times bounded samples of it, described in its
    cpu_baseline.sample)."""
    name = {"batched": f"batched scan {n:.3g} rows x 4 skewed columns, {nq} queries",
            "single": f"single-column {n:.3g}-row scan, 10% selectivity",
            "multi": f"4-column {n:.3g}-row conjunctive scan",
            "q6": f"fused scan-and-aggregate, {n:.3g} rows x 4 columns (TPC-H Q6 shape)"}[wl]
    return {"workload": name, "nrows_per_gpu": n, "ncols": len(kinds), "queries_per_step": nq,
            "column_kinds": kinds, "l2": f"inputs larger than L2 ({n * 4 / 1e6:.0f} MB per column)"}


def reference_columns(kinds, n):
    """The workload's columns on the host: generated exactly as the GPU arm
    generates them (same device generator and seeds, rank 0), so both arms
    answer the same queries on the same rows; the numpy generators of the
    same distributions stand in where no GPU is visible."""
    try:
        import torch
        if torch.cuda.is_available():
            dev = torch.device("cuda", 0)
            out = []
            for i, k in enumerate(kinds):
                col = gpu_column(torch, k, n, 1000 + i, dev)
                smp = host_sample(torch, col, seed=7 + i)
                out.append((col.cpu().numpy().view(np.uint32).copy(), smp))
                del col
            torch.cuda.empty_cache()
            return [c for c, _ in out], [m for _, m in out], "device generator of the GPU arm (same rows)"
    except Exception:  # fall back to the host generators below
        pass
    cols = cpu_sample_columns(kinds, n)
    smp = [np.sort(c[np.random.default_rng(7).integers(0, n, size=1 << 18)]) for c in cols]
    return cols, smp, "numpy generators of the same distributions"


def run_reference(args):
    """--impl reference: the reference's own CPU path (its bindex.cpp
    compiled unmodified, oracle/_ref) on this host, rank 0 only, on the
    workload's own row count: the BinDex of every column is built once
    (reported, not timed), then every step times `per_step` of the
    workload's queries through the reference's query loop (sieve + refine
    + AND merge per query, its timer-11 region), a disjoint seeded subset
    per step.  Without a harness binary for the workload's row count the
    2^24-row binary runs a prefix sample, and the line says so."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from rtscan_b200 import datagen as D
    wl = args.workload
    if wl == "q6":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no aggregate step (it stops at "
                          "the bitmap); the q6 line's cpu_baseline times a numpy port"}), flush=True)
        return
    kinds = {"single": ["uniform"], "multi": ["uniform"] * 4}.get(wl, BATCH_KINDS)
    n_full = args.nrows
    n = n_full if reference_binary(n_full) else REF_N
    binary = reference_binary(n)
    t_start = time.time()
    cols, smp, source = reference_columns(kinds, n_full if n == n_full else n)
    queries = make_queries(D, wl, smp, args.queries)
    bprq = row_query_bytes(n_full, queries)
    nq = len(queries)
    per_step = min(nq, args.ref_queries_per_step)
    order = np.random.default_rng(2024).permutation(nq)
    steps = args.warmup + args.steps
    picks = [[int(order[(st * per_step + i) % nq]) for i in range(per_step)] for st in range(steps)]
    if binary:
        flat = [queries[i] for p in picks for i in p]
        build_ms, ms, eq = run_reference_harness(binary, cols, flat, checked=1)
        kind, cores = "reference", REF_THREADS
        detail = {"reference_bindex_equals_scalar_checked": all(eq), "checked_queries": len(eq),
                  "index_build_ms": round(build_ms)}
    else:  # the oracle's restatement, one thread
        from oracle import oracle as O
        ms = []
        for p in picks:
            for i in p:
                q = queries[i]
                t0 = time.perf_counter()
                O.range_scan([cols[c] for c, _, _ in q], [t[1] for t in q], [t[2] for t in q])
                ms.append((time.perf_counter() - t0) * 1e3)
        kind, cores, detail = "port", 1, {}
    del cols
    step_ms = [sum(ms[st * per_step:(st + 1) * per_step]) for st in range(steps)][args.warmup:]
    vals = [per_step * n * bprq / (t * 1e-3) / 1e9 for t in step_ms]
    v = statistics.median(vals)
    t_med = statistics.median(step_ms)
    qps = per_step / (t_med * 1e-3) * n / n_full
    sample = (f"{n} rows x {len(kinds)} columns ({source}); each step {per_step} of the workload's {nq} queries "
              f"(seeded disjoint subsets, {len(picks) * per_step} queries over {steps} steps) through the "
              f"reference BinDex query loop, {cores} threads, index build excluded; credited {bprq:.4f} B per row "
              "and query, the workload's bytes share")
    if n != n_full:
        sample += f"; a prefix sample of the workload's {n_full} rows, queries_per_s scaled to them"
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "GB/s", "n_gpus": world,
            "steps": len(step_ms), "warmup": args.warmup, "ms_per_step": round(t_med, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded)",
            "config": workload_config(wl, n_full, nq, kinds),
            "rows_run": n, "queries_timed_per_step": per_step,
            "queries_per_s": round(qps, 3),
            "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "kind": kind, "cores": cores,
                             "sample": sample, **host_info(), **detail,
                             "wall_s": round(time.time() - t_start, 1)},
            "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1, help="ranks, one per GPU (started under torchrun if needed)")
    ap.add_argument("--dry-run", action="store_true", help="print each rank's world and exit (no GPU work)")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "single", "multi", "q6"])
    ap.add_argument("--nrows", type=int, default=100_000_000)
    ap.add_argument("--queries", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-queries-per-step", type=int, default=32,
                    help="--impl reference: queries of the workload timed per step")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-compare", action="store_true", help="skip the one-query-per-launch comparison")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-scan leg")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default batch launch shape")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the single-column, multi-column and selectivity-sweep legs (profiling runs)")
    ap.add_argument("--bindex-io", type=int, default=0, metavar="ROWS",
                    help="also time BinDex build vs save and load for a ROWS-row column (off by default)")
    ap.add_argument("--bindex-query", type=int, default=0, metavar="ROWS",
                    help="run the selectivity sweep (fused scan and BinDex) on ROWS-row columns alone")
    ap.add_argument("--pass-sweep", type=int, default=0, metavar="ROWS",
                    help="also time one pass of 1..512 queries over a ROWS-row table (off by default)")
    ap.add_argument("--serve-rows", type=int, default=1 << 28)
    ap.add_argument("--serve-rates", type=float, nargs="+",
                    default=[1000, 5000, 10000, 20000, 30000, 40000, 50000])
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    cmd = check_world(args.gpus)
    if cmd is not None:  # start the ranks and report their exit status
        raise SystemExit(subprocess.run(cmd).returncode)
    if args.dry_run:  # the resolved world, without touching a GPU
        world, rank, local = dist_env()
        print(json.dumps({"rank": rank, "local_rank": local, "world": world, "gpus": args.gpus}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
