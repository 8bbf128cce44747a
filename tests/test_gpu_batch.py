"""Batched scan (one pass answering many queries) against the oracle: every
query's bitmap and count must equal the scalar filter's, whatever the batch
size, the mix of column counts, or the pass split."""
import numpy as np
import pytest

import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def expect(cols, terms):
    n = len(cols[0])
    if any(lo > hi for _, lo, hi in terms):
        return np.zeros(O.words(n), np.uint32), 0
    if not terms:
        return O.mask_tail(np.full(O.words(n), 0xFFFFFFFF, np.uint32), n), n
    return O.range_scan([cols[c] for c, _, _ in terms], [t[1] for t in terms], [t[2] for t in terms])


def run_batch(ctx, queries, fn="batch"):
    n = ctx.nrows
    words = R.bitmap_words(n)
    stride = words + 5  # deliberately not a multiple of anything
    out = torch.full((max(1, len(queries)) * stride,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((max(1, len(queries)),), -1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    if fn == "graph":  # prepared once, replayed as a CUDA graph
        pb = ctx.prepare_batch(queries, out.data_ptr(), stride, cnt.data_ptr())
        try:
            pb.launch(s)
            torch.cuda.synchronize()
        finally:
            pb.release()
    else:
        runner = ctx.scan_batch_async if fn == "batch" else ctx.scan_each_async
        runner(queries, out.data_ptr(), stride, cnt.data_ptr(), s)
        torch.cuda.synchronize()
    o = out.cpu().numpy().view(np.uint32)
    return [(o[i * stride:i * stride + words], int(cnt[i].item()), o[i * stride + words:(i + 1) * stride])
            for i in range(len(queries))]


def check_batch(ctx, cols, queries):
    res = run_batch(ctx, queries)
    for i, q in enumerate(queries):
        want, wcnt = expect(cols, q)
        got, cnt, pad = res[i]
        assert cnt == wcnt, (i, q, cnt, wcnt)
        assert np.array_equal(got, want), (i, q)
        assert (pad == 0xFFFFFFFF).all(), "wrote past the bitmap"


@pytest.mark.parametrize("nq", [1, 2, 5, 20, 21, 31, 32, 33, 255, 256, 257, 700])
def test_batch_sizes(ctx, nq):
    n = 300_000 + 123
    cols = [D.uniform(n, 1), D.zipf(n, 2, 1.3), D.uniform(n, 3, 256), D.normal(n, 4)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, nq, seed=nq)
    check_batch(ctx, cols, qs)


@pytest.mark.parametrize("n", [1, 31, 32, 255, 256, 257, 1000, 8191, 65537])
def test_batch_row_counts(ctx, n):
    cols = [D.uniform(n, 10 + n), D.uniform(n, 20 + n, 64)]
    ctx.load_columns(cols)
    s0 = np.sort(cols[0])
    qs = [[(0, int(s0[0]), int(s0[-1]))], [(1, 3, 40)], [(0, 0, 1 << 31), (1, 10, 63)], [(1, 0, 0)],
          [(0, int(s0[len(s0) // 2]), 0xFFFFFFFF)]]
    check_batch(ctx, cols, qs)


def test_batch_special_queries(ctx):
    n = 100_003
    cols = [D.uniform(n, c + 50, [1 << 32, 256, 64, 1 << 20, 7, 1 << 32, 1000, 1 << 16, 300, 99][c]) for c in range(10)]
    ctx.load_columns(cols)
    qs = [
        [],                                        # no terms: all rows
        [(0, 0, 0xFFFFFFFF)],                      # always true
        [(1, 10, 5)],                              # empty term
        [(0, 5, 10), (0, 20, 30)],                 # disjoint ranges on one column: empty
        [(1, 10, 200), (1, 100, 255)],             # overlapping ranges merged
        [(c, 1, [1 << 31, 200, 60, 1 << 19, 6, 1 << 31, 900, 1 << 15, 250, 90][c]) for c in range(10)],  # 10 columns
        [(c, 0, [1 << 31, 200, 60, 1 << 19, 6, 1 << 31, 900, 1 << 15, 250, 90][c]) for c in range(9)],
        [(4, 3, 3)],
        [(2, 63, 63), (3, 0, 0)],
    ] + D.batch_queries(cols[:4], 40, seed=9)
    check_batch(ctx, cols, qs)


@pytest.mark.parametrize("nq", [90, 200, 300])
def test_batch_many_columns_per_pass(ctx, nq):
    """Queries over 6 different columns force passes with more than 4 table
    columns, in each pass shape (128, 256 and 512 query slots)."""
    n = 50_000 + 4096 * 3 + 17
    cols = [D.uniform(n, 70 + c, 1 << (8 + 4 * c)) for c in range(6)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, nq, seed=11, min_cols=1, max_cols=6)
    check_batch(ctx, cols, qs)


def test_batch_few_pass_after_table_pass(ctx):
    """520 queries over 7 columns: a 512-slot table pass, then an 8-query pass
    tested term by term, both with more than 4 columns."""
    n = 70_001
    cols = [D.uniform(n, 600 + c, 1 << (6 + 4 * c)) for c in range(7)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 520, seed=13, min_cols=1, max_cols=7)
    ctx.set_batch_config(4, 16, 512, 136 * 1024)
    check_batch(ctx, cols, qs)


@pytest.mark.parametrize("nq", [3, 128, 129, 256, 257])
def test_batch_pass_shapes_at_block_edges(ctx, nq):
    """Row counts one short of and one past the 1024-, 2048- and 4096-row
    blocks of the three pass shapes."""
    for n in (4095, 4097, 2 * 4096 + 2047, 3 * 4096 + 1025):
        cols = [D.zipf(n, 400 + n, 1.2), D.normal(n, 401)]
        ctx.load_columns(cols)
        check_batch(ctx, cols, D.batch_queries(cols, nq, seed=n + nq))


@pytest.mark.parametrize("nq", [100, 200, 500])
def test_batch_skewed_boundaries(ctx, nq):
    """Bounds packed into small values plus powers of two up to 2^32 - 1 (the
    shape for which the planner indexes boundaries by log-linear buckets),
    with rows sitting on and next to every bound; crowded buckets send many
    rows to the full search in every pass shape (128, 256 and 512 slots)."""
    n = 120_000
    rng = np.random.default_rng(5)
    edges = [0, 1, 2] + [v for k in range(2, 33) for v in ((1 << k) - 2, (1 << k) - 1, 1 << k)
                         if v <= 0xFFFFFFFF]
    edges = np.array(sorted(set(e for e in edges if e <= 0xFFFFFFFF)), dtype=np.uint64)
    near = rng.choice(edges, size=n // 2)
    small = rng.integers(0, 400, size=n // 4)
    wide = rng.integers(0, 1 << 32, size=n - n // 2 - n // 4)
    col = np.concatenate([near, small, wide]).astype(np.uint32)
    rng.shuffle(col)
    cols = [col, D.zipf(n, 7, 1.5)]
    ctx.load_columns(cols)
    pool = [int(e) for e in edges] + list(range(0, 400, 3))
    qs = []
    for i in range(nq):
        a, b = sorted(int(x) for x in rng.choice(pool, size=2))
        q = [(0, a, b)]
        if i % 3 == 0:
            q.append((1, int(rng.integers(0, 20)), int(rng.integers(20, 3000))))
        qs.append(q)
    check_batch(ctx, cols, qs)


def test_batch_duplicate_heavy(ctx):
    n = 200_000
    cols = [D.uniform(n, 80, 2), D.uniform(n, 81, 64), D.zipf(n, 82, 1.5)]
    ctx.load_columns(cols)
    qs = []
    for a in range(0, 64, 3):
        qs.append([(1, a, a)])
        qs.append([(1, a, 63), (0, 1, 1)])
        qs.append([(2, a, a + 5), (0, 0, 0)])
    check_batch(ctx, cols, qs)


def test_batch_equals_each(ctx):
    n = 1 << 20
    cols = [D.zipf(n, 90, 1.1), D.zipf(n, 91, 1.3), D.zipf(n, 92, 1.5), D.normal(n, 93)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 1024, seed=3)
    a = run_batch(ctx, qs, "batch")
    b = run_batch(ctx, qs, "each")
    for i in range(len(qs)):
        assert a[i][1] == b[i][1], i
        assert np.array_equal(a[i][0], b[i][0]), i


def test_batch_alone_and_in_the_mix(ctx):
    """A query's result does not depend on the other queries of its batch."""
    n = 400_000
    cols = [D.uniform(n, 95), D.normal(n, 96)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 600, seed=12)
    mixed = run_batch(ctx, qs)
    for i in (0, 17, 255, 256, 599):
        alone = run_batch(ctx, [qs[i]])[0]
        assert alone[1] == mixed[i][1]
        assert np.array_equal(alone[0], mixed[i][0])


@pytest.mark.parametrize("cfg", [(4, 16, 512, 136 * 1024), (4, 16, 256, 136 * 1024), (4, 16, 100, 136 * 1024),
                                 (4, 16, 512, 8 * 1024),
                                 (4, 8, 512, 136 * 1024), (4, 8, 512, 56 * 1024), (4, 8, 256, 56 * 1024),
                                 (4, 8, 128, 56 * 1024), (4, 8, 100, 136 * 1024),
                                 (3, 16, 256, 88 * 1024), (3, 16, 64, 16 * 1024), (3, 8, 256, 40 * 1024),
                                 (3, 8, 128, 140 * 1024), (3, 8, 1, 4096), (4, 16, 1, 4096)])
def test_batch_every_launch_shape(ctx, cfg):
    n = 150_011
    cols = [D.uniform(n, 200), D.zipf(n, 201, 1.1), D.uniform(n, 202, 1000), D.normal(n, 203)]
    ctx.load_columns(cols)
    old = ctx.batch_config()
    ctx.set_batch_config(*cfg)
    try:
        check_batch(ctx, cols, D.batch_queries(cols, 600, seed=cfg[2]) + [[], [(1, 3, 2)]])
    finally:
        ctx.set_batch_config(old["variant"], old["warps_per_cta"], old["max_queries_per_pass"],
                             old["table_budget_bytes"])


def test_autotune_picks_a_valid_shape_and_caches_it(ctx, tmp_path):
    n = 1 << 20
    cols = [D.zipf(n, 210, 1.3), D.normal(n, 211)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 200, seed=4)
    cache = str(tmp_path / "tune.txt")
    best = ctx.autotune_batch(qs, cache)
    assert best["variant"] in (3, 4) and best["warps_per_cta"] in (8, 16)
    assert 1 <= best["max_queries_per_pass"] <= 512
    assert open(cache).read().strip()
    again = ctx.autotune_batch(qs, cache)  # served from the cache
    assert again == best
    check_batch(ctx, cols, qs)
    with pytest.raises(R.RtsError):
        ctx.set_batch_config(3, 12, 256, 88 * 1024)
    with pytest.raises(R.RtsError):
        ctx.set_batch_config(4, 16, 513, 88 * 1024)


def test_autotuned_shape_is_not_slower_than_the_default(ctx):
    """The tuner searches pass sizes, table budgets, variants and warps per
    CTA on a sample of the real table, reports every candidate, and its
    choice, timed again on the whole table after tuning, is no slower than
    the default shape beyond timing noise (5 %)."""
    n = 1 << 25
    cols = [D.zipf(n, 220, 1.1), D.zipf(n, 221, 1.5), D.normal(n, 222), D.zipf(n, 223, 1.3)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 1024, seed=8)
    old = ctx.batch_config()
    try:
        ctx.set_batch_config(4, 16, 512, 136 * 1024)
        best = ctx.autotune_batch(qs)
        rep = ctx.autotune_report()
        assert rep["sample_rows"] == n and rep["queries"] == len(qs)
        shapes = {(c["variant"], c["warps_per_cta"], c["max_queries_per_pass"], c["table_budget_bytes"])
                  for c in rep["candidates"]}
        assert len(shapes) == len(rep["candidates"]) >= 18
        assert {v for v, _, _, _ in shapes} == {3, 4} and {w for _, w, _, _ in shapes} == {8, 16}
        assert rep["best_ms"] <= rep["default_ms"]
        words = R.bitmap_words(n)
        stride = (words + 31) // 32 * 32
        out = torch.empty(len(qs) * stride, dtype=torch.int32, device="cuda")
        cnt = torch.empty(len(qs), dtype=torch.int64, device="cuda")
        s = torch.cuda.current_stream()

        def med(reps=5):
            pq = R.prepare(qs)
            ctx.scan_batch_async(pq, out.data_ptr(), stride, cnt.data_ptr(), s.cuda_stream)
            ts = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                ctx.scan_batch_async(pq, out.data_ptr(), stride, cnt.data_ptr(), s.cuda_stream)
                e1.record(s)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            return sorted(ts)[reps // 2]

        tuned = med()
        ctx.set_batch_config(4, 16, 512, 136 * 1024)
        default = med()
        assert tuned <= default * 1.05, (best, tuned, default)
    finally:
        ctx.set_batch_config(old["variant"], old["warps_per_cta"], old["max_queries_per_pass"],
                             old["table_budget_bytes"])


@pytest.mark.parametrize("n,nq", [(70_001, 300), (9_000_011, 300), (9_000_011, 20), (9_000_011, 2),
                                  (9_000_011, 1)])
def test_batch_host_buffers(ctx, n, nq):
    """Host columns in, host bitmaps out: the upload, scan and download run as
    a row-chunked pipeline (two chunks at 9e6 rows), with queries outside the
    batch kernels (no term, an empty term, nine columns) among them; one
    kernel query runs as a fused scan per chunk, two term by term.  The
    context's own table is untouched."""
    ctx.load_columns([D.uniform(1000, 1)])
    cols = [D.uniform(n, 500 + c, [1 << 32, 1 << 20, 4096, 256, 64, 1 << 16, 1 << 32, 1000, 77][c])
            for c in range(9)]
    cols[2] = D.zipf(n, 502, 1.3)
    qs = D.batch_queries(cols[:4], nq, seed=17) + [
        [], [(3, 9, 2)], [(c, 1, [1 << 31, 1 << 19, 4000, 200, 60, 1 << 15, 1 << 31, 900, 70][c]) for c in range(9)]]
    stride = R.bitmap_words(n) + 3
    bms, counts = ctx.scan_batch_host(cols, qs, stride_words=stride)
    for i, q in enumerate(qs):
        want, wcnt = expect(cols, q)
        assert int(counts[i]) == wcnt, (i, q)
        assert np.array_equal(bms[i, :R.bitmap_words(n)], want), (i, q)
    assert ctx.nrows == 1000


def test_batch_host_buffers_many_chunks_and_a_refused_query(ctx):
    """A table of four row chunks: every upload is queued before the batch is
    planned, and a batch the planner refuses (a term on a column the call
    does not pass) fails with RTS_ERR_ARG after those uploads have finished,
    leaving the context usable for the next call."""
    n = (1 << 24) + 12_345
    ctx.load_columns([D.uniform(1000, 1)])
    cols = [D.uniform(n, 600), D.zipf(n, 601, 1.1), D.normal(n, 602)]
    qs = D.batch_queries(cols, 300, seed=18)
    with pytest.raises(R.RtsError) as e:
        ctx.scan_batch_host(cols, qs + [[(5, 0, 9)]])
    assert e.value.code == -1
    bms, counts = ctx.scan_batch_host(cols, qs)
    for i in (0, 1, 150, 299):
        want, wcnt = expect(cols, qs[i])
        assert int(counts[i]) == wcnt and np.array_equal(bms[i, :R.bitmap_words(n)], want), i
    assert ctx.nrows == 1000


def test_four_passes_share_positions(ctx):
    """1600 queries over four columns make four 512-slot passes (the table
    budget holds about 400 queries each) that share one position search per
    row, two map words per union position; every bitmap and count equals
    one query per launch, and a sample the scalar filter."""
    n = (1 << 21) + 77
    cols = [D.zipf(n, 240, 1.1), D.uniform(n, 241), D.normal(n, 242), D.zipf(n, 243, 1.5)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 1600, seed=33, min_cols=2, max_cols=4)
    want = run_batch(ctx, qs, "each")
    got = run_batch(ctx, qs, "batch")
    for i in range(len(qs)):
        assert got[i][1] == want[i][1] and np.array_equal(got[i][0], want[i][0]), i
    for i in (0, 700, 1599):
        ref, rcnt = expect(cols, qs[i])
        assert want[i][1] == rcnt and np.array_equal(want[i][0], ref), i


def test_batch_host_sparse_chunks_are_expanded(ctx):
    """Row chunks whose bitmap words are mostly zero leave the device as a
    nonzero-word mask and the nonzero words, which host threads expand: into buffers filled with
    ones beforehand, every bitmap (very selective, dense and outside-kernel
    queries mixed, four chunks) equals the device path's, the padding after
    each bitmap is untouched, and fewer bytes crossed than whole bitmaps."""
    n = (1 << 24) + 12_345
    cols = [D.uniform(n, 700), D.zipf(n, 701, 1.3), D.uniform(n, 702, 1 << 20)]
    s0 = np.sort(cols[0])
    qs = D.batch_queries(cols, 200, seed=19)
    rng = np.random.default_rng(20)
    for k in (3, 40, 500, 4000, 30_000):  # 3 .. 30000 matching rows of column 0
        i = int(rng.integers(0, n - k))
        qs.append([(0, int(s0[i]), int(s0[i + k - 1]))])
        qs.append([(0, int(s0[i]), int(s0[i + k - 1])), (2, 0, 1 << 19)])
    qs.append([(1, 0, 0xFFFFFFFF)])  # every row
    qs.append([(0, 5, 4)])           # empty
    words = R.bitmap_words(n)
    stride = words + 7
    host = np.full((len(qs), stride), 0xFFFFFFFF, dtype=np.uint32)
    bms, counts = ctx.scan_batch_host(cols, qs, host_bitmaps=host, stride_words=stride)
    h2d, d2h = ctx.host_transfer_bytes()
    ctx.load_columns(cols)
    want = run_batch(ctx, qs, "batch")
    for i in range(len(qs)):
        assert int(counts[i]) == want[i][1], (i, qs[i])
        assert np.array_equal(bms[i, :words], want[i][0]), (i, qs[i])
        assert (bms[i, words:] == 0xFFFFFFFF).all(), i
    for i in range(len(qs) - 12, len(qs)):
        ref, rcnt = expect(cols, qs[i])
        assert want[i][1] == rcnt and np.array_equal(want[i][0], ref), i
    assert h2d >= 4 * n * len(cols)
    assert d2h < len(qs) * words * 4, (d2h, len(qs) * words * 4)


@pytest.mark.parametrize("nq", [1, 7, 100, 200, 400])
def test_prepared_batch_graph_replays_match(ctx, nq):
    """Graph replays of each pass shape: a fused scan (1 query), term by term
    (7), 128 slots (100), 256 slots (200) and 512 slots (400), with queries
    outside the kernels."""
    n = 333_333
    cols = [D.uniform(n, 300), D.zipf(n, 301, 1.5), D.uniform(n, 302, 64)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, nq, seed=21) + [[], [(2, 9, 3)], [(c, 1, 0xFFFFFF00) for c in range(3)]]
    words = R.bitmap_words(n)
    stride = (words + 31) // 32 * 32
    out = torch.full((len(qs) * stride,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((len(qs),), -1, dtype=torch.int64, device="cuda")
    pb = ctx.prepare_batch(qs, out.data_ptr(), stride, cnt.data_ptr())
    s = torch.cuda.current_stream().cuda_stream
    for rep in range(2):
        out.fill_(-1)
        cnt.fill_(-1)
        pb.launch(s)
        torch.cuda.synchronize()
        o = out.cpu().numpy().view(np.uint32)
        for i, q in enumerate(qs):
            want, wcnt = expect(cols, q)
            assert int(cnt[i].item()) == wcnt, (rep, i)
            assert np.array_equal(o[i * stride:i * stride + words], want), (rep, i)
    pb.release()


def test_shared_positions_in_every_path(ctx):
    """A batch of 1100 queries over four columns plans two 512-slot passes
    that share one position search per row (and a third, smaller pass that
    searches on its own).  The plain batch, its CUDA-graph replay, the
    host-buffer path and the server all give every query's bitmap and count
    of one query per launch; a sample matches the scalar filter."""
    n = (1 << 22) + 123
    cols = [D.zipf(n, 230, 1.1), D.uniform(n, 231), D.normal(n, 232), D.uniform(n, 233, 4096)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 1100, seed=31)
    want = run_batch(ctx, qs, "each")
    for runner in ("batch", "graph"):
        got = run_batch(ctx, qs, runner)
        for i in range(len(qs)):
            assert got[i][1] == want[i][1] and np.array_equal(got[i][0], want[i][0]), (runner, i)
    bms, counts = ctx.scan_batch_host(cols, qs)
    ctx.load_columns(cols)
    for i in range(len(qs)):
        assert int(counts[i]) == want[i][1] and np.array_equal(bms[i, :R.bitmap_words(n)], want[i][0]), ("host", i)
    with R.Server(ctx, max_active=1100, segment_rows=1 << 20) as srv:
        tks = [srv.submit(q) for q in qs]
        for i, tk in enumerate(tks):
            srv.wait(tk, 120000)
            bm, cnt = srv.fetch(tk)
            assert cnt == want[i][1] and np.array_equal(bm, want[i][0]), ("served", i)
    for i in (0, 511, 512, 1023, 1099):
        ref, rcnt = expect(cols, qs[i])
        assert want[i][1] == rcnt and np.array_equal(want[i][0], ref), i
    # columns attached 4 bytes past an 8-byte boundary: the position search
    # loads one row at a time
    held = []
    for c in cols:
        t = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        t[1:] = torch.from_numpy(c.view(np.int32)).cuda()
        held.append(t)
    ctx.attach_columns([t.data_ptr() + 4 for t in held], n)
    got = run_batch(ctx, qs, "batch")
    for i in range(len(qs)):
        assert got[i][1] == want[i][1] and np.array_equal(got[i][0], want[i][0]), ("unaligned", i)
    ctx.load_columns(cols)
    del held
