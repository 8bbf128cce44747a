"""Repeated use does not leak device memory: after a warm-up cycle, more
cycles of every resource-owning call on one context (table loads, indexes,
batched scans, prepared graphs, a server, encoding, aggregates, compaction)
leave the device's free memory where it was, and so do contexts opened and
closed in a loop."""
import numpy as np
import pytest

import rtscan_b200 as R
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def free_bytes():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def one_cycle(ctx, cols, out, cnt, s2, rows, stride):
    n = len(cols[0])
    ctx.load_columns(cols)
    ctx.build_bindex(0, 32)
    qs = D.batch_queries(cols, 300, seed=1) + D.batch_queries(cols, 5, seed=2)
    s = torch.cuda.current_stream().cuda_stream
    ctx.scan_batch_async(qs, out.data_ptr(), stride, cnt.data_ptr(), s)
    pb = ctx.prepare_batch(qs[:40], out.data_ptr(), stride, cnt.data_ptr())
    pb.launch(s)
    pb.release()
    ctx.bindex_scan_async([(0, 10, 1 << 30)], out.data_ptr(), cnt.data_ptr(), s)
    ctx.bitmap_rows_async(out.data_ptr(), n, rows.data_ptr(), n, cnt.data_ptr(), s)
    ctx.scan_aggregate_async([(1, 0, 1 << 31)], 0, 1, cnt.data_ptr(), s2.data_ptr(), s)
    with R.Server(ctx, max_active=16, segment_rows=1 << 16) as srv:
        t = srv.submit([(0, 0, 1 << 30)])
        srv.wait(t, 10000)
        srv.fetch(t, want_bitmap=False)
    ctx.encode_table()
    ctx.encode_terms([(0, 5, 10)])
    torch.cuda.synchronize()


def test_no_growth_over_cycles():
    n = 300_001
    cols = [D.zipf(n, 1, 1.3), D.uniform(n, 2)]
    stride = (R.bitmap_words(n) + 31) // 32 * 32
    out = torch.empty(305 * stride, dtype=torch.int32, device="cuda")
    cnt = torch.empty(305, dtype=torch.int64, device="cuda")
    s2 = torch.empty(2, dtype=torch.int64, device="cuda")
    rows = torch.empty(n, dtype=torch.int32, device="cuda")
    with R.Context(0) as ctx:
        one_cycle(ctx, cols, out, cnt, s2, rows, stride)  # warm-up: scratch and caches
        before = free_bytes()
        for _ in range(4):
            one_cycle(ctx, cols, out, cnt, s2, rows, stride)
        after = free_bytes()
    assert before - after < 32 << 20, (before - after) / 2 ** 20


def test_contexts_open_and_close():
    n = 200_003
    cols = [D.uniform(n, 3), D.uniform(n, 4, 1000)]
    with R.Context(0) as ctx:  # first context: module load, library state
        ctx.load_columns(cols)
    before = free_bytes()
    for _ in range(5):
        with R.Context(0) as ctx:
            ctx.load_columns(cols)
            ctx.build_bindex(1, 16)
            ctx.scan([(1, 5, 50)])
    after = free_bytes()
    assert before - after < 16 << 20, (before - after) / 2 ** 20
