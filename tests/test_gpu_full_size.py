"""Parity at the workloads' full sizes.

* 1e8-row scans checked bit-exactly against the oracle over every row: one
  uniform column at five selectivities, two duplicate-heavy cardinalities,
  and 2-4 uniform columns through the fused, separate and BinDex paths.
* The 1024-query batch over four skewed 1e8-row columns: every query's
  bitmap and count equal one query per launch, the CUDA-graph replay equals
  the plain batch, and a seeded random 64 of its queries (plus the pass
  edges 0, 511, 512 and 1023) equal the oracle.
* The served 2^28-row table: every served result equals the direct scan of
  the same query, and 12 of those direct scans equal the oracle.
* Properties that hold at any size: a range split in two gives the OR of the
  halves' bitmaps and the sum of their counts, and the ranges below, inside
  and above a predicate partition the rows.

Columns are generated on the device by the benchmark's own seeded generator,
so these are the benchmark's inputs."""
from concurrent.futures import ThreadPoolExecutor
import os

import numpy as np
import pytest

import bench
import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = 100_000_000
N_SERVED = 1 << 28
MAXV = 0xFFFFFFFF


def stride_of(n):
    return (R.bitmap_words(n) + 31) // 32 * 32


def host(col):
    return col.cpu().numpy().view(np.uint32)


class Table:
    """Device columns of one workload attached to the shared context."""

    def __init__(self, ctx, kinds, n, seed):
        dev = torch.device("cuda:0")
        self.n = n
        self.cols = [bench.gpu_column(torch, k, n, seed + i, dev) for i, k in enumerate(kinds)]
        self.samples = [bench.host_sample(torch, c) for c in self.cols]
        self._host = {}
        ctx.attach_columns([c.data_ptr() for c in self.cols], n)

    def host_col(self, c):
        if c not in self._host:
            self._host[c] = host(self.cols[c])
        return self._host[c]

    def oracle(self, q):
        return O.range_scan([self.host_col(c) for c, _, _ in q], [t[1] for t in q], [t[2] for t in q])

    def oracle_many(self, qs):
        """The oracle of several queries on host threads (its C scan runs
        without the interpreter lock)."""
        for c in {c for q in qs for c, _, _ in q}:
            self.host_col(c)
        with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
            return list(ex.map(self.oracle, qs))


@pytest.fixture()
def table_scope(ctx):
    """Drop every big buffer and detach the columns after the test."""
    held = []
    yield held
    ctx.load_columns([np.zeros(64, np.uint32)])
    held.clear()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def run(fn, q, n):
    bm = torch.full((R.bitmap_words(n),), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    fn(q, bm.data_ptr(), cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return bm, int(cnt.item())


def assert_oracle(t, fn, q, what):
    bm, cnt = run(fn, q, t.n)
    want, wcnt = t.oracle(q)
    assert cnt == wcnt, (what, q, cnt, wcnt)
    assert np.array_equal(host(bm), want), (what, q)


def test_single_column_selectivities_1e8(ctx, table_scope):
    t = Table(ctx, ["uniform"], N, 31)
    table_scope.append(t)
    for sel in (0.001, 0.01, 0.10, 0.50, 0.90):
        q = [(0, *D.range_for_selectivity(t.samples[0], sel))]
        assert_oracle(t, ctx.scan_async, q, f"fused sel={sel}")
    q = [(0, *D.range_for_selectivity(t.samples[0], 0.10))]
    ctx.build_bindex(0, 128)
    assert_oracle(t, ctx.bindex_scan_async, q, "bindex")
    for q in ([(0, 0, MAXV)], [(0, MAXV, MAXV)], [(0, 0, 0)]):
        assert_oracle(t, ctx.scan_async, q, "edge")


@pytest.mark.parametrize("card", [1 << 6, 1 << 8])
def test_duplicate_heavy_1e8(ctx, table_scope, card):
    t = Table(ctx, [f"range:0:{card}"], N, 41 + card)
    table_scope.append(t)
    ctx.build_bindex(0, 128)
    for q in ([(0, 3, 3)], [(0, 0, card // 10)], [(0, card // 4, 3 * card // 4)], [(0, card - 1, MAXV)],
              [(0, card, MAXV)]):
        assert_oracle(t, ctx.scan_async, q, "fused")
        assert_oracle(t, ctx.bindex_scan_async, q, "bindex")


def test_multi_column_paths_1e8(ctx, table_scope):
    t = Table(ctx, ["uniform"] * 4, N, 51)
    table_scope.append(t)
    for c in range(4):
        ctx.build_bindex(c, 128)
    rng = np.random.default_rng(52)
    for ncols in (2, 3, 4):
        q = []
        for c in rng.choice(4, size=ncols, replace=False):
            sel = float(rng.uniform(0.05, 0.5))
            q.append((int(c), *D.range_for_selectivity(t.samples[c], sel, float(rng.uniform(sel / 2, 1 - sel / 2)))))
        want, wcnt = t.oracle(q)
        for name, fn in (("fused", ctx.scan_async), ("separate", ctx.scan_separate_async),
                         ("bindex", ctx.bindex_scan_async)):
            bm, cnt = run(fn, q, t.n)
            assert cnt == wcnt, (name, q, cnt, wcnt)
            assert np.array_equal(host(bm), want), (name, q)


def test_range_split_and_partition_1e8(ctx, table_scope):
    t = Table(ctx, ["uniform"], N, 61)
    table_scope.append(t)
    lo, hi = D.range_for_selectivity(t.samples[0], 0.3)
    mid = (lo + hi) // 2
    whole, cw = run(ctx.scan_async, [(0, lo, hi)], t.n)
    left, cl = run(ctx.scan_async, [(0, lo, mid)], t.n)
    right, cr = run(ctx.scan_async, [(0, mid + 1, hi)], t.n)
    assert cl + cr == cw
    assert torch.equal(left | right, whole)
    assert not bool((left & right).any())
    below, cb = run(ctx.scan_async, [(0, 0, lo - 1)], t.n)
    above, ca = run(ctx.scan_async, [(0, hi + 1, MAXV)], t.n)
    assert cb + cw + ca == t.n
    assert bool(((below | whole | above) == -1).all())  # 1e8 is a multiple of 32: no tail word
    assert not bool((below & whole).any()) and not bool((whole & above).any())


def test_batched_1024_skewed_1e8(ctx, table_scope):
    t = Table(ctx, bench.BATCH_KINDS, N, 71)
    table_scope.append(t)
    qs = D.batch_queries(t.samples, 1024, seed=72)
    nq, words, stride = len(qs), R.bitmap_words(N), stride_of(N)
    s = torch.cuda.current_stream().cuda_stream
    out_b = torch.full((nq, stride), -1, dtype=torch.int32, device="cuda")
    cnt_b = torch.full((nq,), -1, dtype=torch.int64, device="cuda")
    table_scope.append(out_b)
    ctx.scan_batch_async(qs, out_b.data_ptr(), stride, cnt_b.data_ptr(), s)
    torch.cuda.synchronize()
    # the sample against the oracle first, while only one result set is held:
    # a seeded random 64 of the queries and the edges of the two passes
    pick = sorted(set(np.random.default_rng(73).choice(nq, 64, replace=False).tolist()) | {0, 511, 512, 1023})
    for i, (want, wcnt) in zip(pick, t.oracle_many([qs[i] for i in pick])):
        assert int(cnt_b[i].item()) == wcnt, (i, qs[i])
        assert np.array_equal(host(out_b[i, :words]), want), (i, qs[i])
    out_e = torch.full((nq, stride), -1, dtype=torch.int32, device="cuda")
    cnt_e = torch.full((nq,), -1, dtype=torch.int64, device="cuda")
    table_scope.append(out_e)
    ctx.scan_each_async(qs, out_e.data_ptr(), stride, cnt_e.data_ptr(), s)
    torch.cuda.synchronize()
    assert torch.equal(cnt_b, cnt_e)
    bad = [i for i in range(nq) if not torch.equal(out_b[i, :words], out_e[i, :words])]
    assert not bad, bad[:10]
    # the CUDA-graph replay of the same batch writes the same results
    out_e.fill_(-1)
    cnt_e.fill_(-1)
    pb = ctx.prepare_batch(qs, out_e.data_ptr(), stride, cnt_e.data_ptr())
    try:
        for _ in range(2):
            pb.launch(s)
        torch.cuda.synchronize()
    finally:
        pb.release()
    assert torch.equal(cnt_b, cnt_e)
    bad = [i for i in range(nq) if not torch.equal(out_b[i, :words], out_e[i, :words])]
    assert not bad, bad[:10]


def test_served_table_2e28(ctx, table_scope):
    t = Table(ctx, bench.SERVE_KINDS, N_SERVED, 81)
    table_scope.append(t)
    qs = D.batch_queries(t.samples, 40, seed=82)
    lo, hi = D.range_for_selectivity(t.samples[0], 0.2)
    qs += [[(0, lo, hi)], [(0, 0, lo - 1)], [(0, hi + 1, MAXV)], [], [(2, 5, 4)]]
    want = []
    for q in qs:
        bm, cnt = ctx.scan(q)
        want.append((bm, cnt))
    checked = list(range(9)) + list(range(len(qs) - 5, len(qs) - 2))  # 9 mixed queries and the 3 edge ranges
    for i, (ref, rcnt) in zip(checked, t.oracle_many([qs[i] for i in checked])):
        assert want[i][1] == rcnt and np.array_equal(want[i][0], ref), (i, qs[i])
    k = len(qs) - 5
    assert want[k][1] + want[k + 1][1] + want[k + 2][1] == N_SERVED
    assert want[k + 3][1] == N_SERVED and want[k + 4][1] == 0
    with R.Server(ctx, max_active=16) as srv:
        tickets = [srv.submit(q) for q in qs]
        for i, tk in enumerate(tickets):
            srv.wait(tk, 120_000)
            bm, cnt = srv.fetch(tk)
            assert cnt == want[i][1], (i, qs[i], cnt, want[i][1])
            assert np.array_equal(bm, want[i][0]), (i, qs[i])
