"""The allocation-free scan entry point (rts_scan_separate_noalloc_async).

It serves callers that cannot let a library allocate device memory (an
engine whose pool allocator owns all of HBM, or a latency-critical path
where cudaMalloc's device-wide synchronisation is not acceptable).  Called
through the C-ABI with ctypes, it must produce the same bitmap and count as
the context-based rts_scan_separate_async -- bit-exact, the tolerance every
scan test here uses -- on two calls in a row that share its static scratch
array, whether this file runs alone in a fresh process or after the other
tests.  Kept in a file of its own that pytest collects last."""
import ctypes

import numpy as np
import pytest

import rtscan_b200 as R
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def noalloc_scan(dev_cols, n, terms, bm, cnt, stream):
    arr, nt = R.make_terms(terms)
    ptrs = (ctypes.c_void_p * len(dev_cols))(*[c.data_ptr() for c in dev_cols])
    rc = R.lib().rts_scan_separate_noalloc_async(ptrs, len(dev_cols), n, arr, nt, bm.data_ptr(), cnt.data_ptr(),
                                                  stream)
    if rc != 0:
        raise R.RtsError(rc, R.lib().rts_last_error(None).decode())


def test_noalloc_matches_separate_scan_on_consecutive_calls():
    n = 3_000_017  # not a multiple of 32 or 1024
    cols_np = [D.uniform(n, 1), D.zipf(n, 2, 1.3), D.uniform(n, 3, 256)]
    dev_cols = [torch.from_numpy(c.view(np.int32)).cuda() for c in cols_np]
    words = R.bitmap_words(n)
    s = torch.cuda.current_stream().cuda_stream
    queries = [
        [(0, 1 << 30, 3 << 30), (1, 0, 40), (2, 10, 200)],   # three passes through the scratch array
        [(2, 0, 127), (0, 0, 1 << 31)],                       # second call: different query, same array
    ]
    with R.Context(0) as ctx:
        ctx.attach_columns([c.data_ptr() for c in dev_cols], n)
        for terms in queries:
            want = torch.full((words,), -1, dtype=torch.int32, device="cuda")
            wcnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            ctx.scan_separate_async(terms, want.data_ptr(), wcnt.data_ptr(), s)
            got = torch.full((words,), -1, dtype=torch.int32, device="cuda")
            gcnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            noalloc_scan(dev_cols, n, terms, got, gcnt, s)
            torch.cuda.synchronize()
            assert int(gcnt.item()) == int(wcnt.item())
            assert torch.equal(got, want)


def test_noalloc_rejects_rows_beyond_its_limit():
    limit = 1 << 27
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    bm = torch.zeros(4, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(R.RtsError) as e:
        noalloc_scan([dummy], limit + 1, [(0, 1, 2)], bm, cnt, 0)
    assert e.value.code == -1
    assert "limit" in str(e.value)


def separate_scan(ctx, terms, words):
    s = torch.cuda.current_stream().cuda_stream
    want = torch.full((words,), -1, dtype=torch.int32, device="cuda")
    wcnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    ctx.scan_separate_async(terms, want.data_ptr(), wcnt.data_ptr(), s)
    torch.cuda.synchronize()
    return want, int(wcnt.item())


@pytest.mark.parametrize("terms", [
    [(0, 5, 4)],                              # lo > hi: no row (the fill path)
    [],                                       # no term: every row (the fill path)
    [(0, 0, 0xFFFFFFFF), (1, 0, 0xFFFFFFFF)],  # only full ranges: every row
    [(1, 3, 900)],                            # one live term: no scratch pass
    [(0, 1 << 31, 0xFFFFFFFF), (0, 0, 3 << 30), (2, 0, 200)],  # two terms merged on one column
], ids=["empty", "no_terms", "full_ranges", "one_term", "merged"])
def test_noalloc_edge_queries_match_separate_scan(terms):
    n = 100_003
    cols_np = [D.uniform(n, 11), D.zipf(n, 12, 1.1), D.uniform(n, 13, 256)]
    dev_cols = [torch.from_numpy(c.view(np.int32)).cuda() for c in cols_np]
    words = R.bitmap_words(n)
    with R.Context(0) as ctx:
        ctx.attach_columns([c.data_ptr() for c in dev_cols], n)
        want, wcnt = separate_scan(ctx, terms, words)
    for _ in range(2):
        got = torch.full((words,), -1, dtype=torch.int32, device="cuda")
        gcnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
        noalloc_scan(dev_cols, n, terms, got, gcnt, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert int(gcnt.item()) == wcnt and torch.equal(got, want)


def test_noalloc_at_its_row_limit():
    """Exactly RTS_NOALLOC_MAX_ROWS rows: the scratch passes use the array's
    last word."""
    n = 1 << 27
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    dev_cols = [torch.randint(-(1 << 31), 1 << 31, (n,), generator=g, device="cuda", dtype=torch.int32)
                for _ in range(2)]
    words = R.bitmap_words(n)
    terms = [(0, 1 << 30, 3 << 30), (1, 0, 1 << 31)]
    with R.Context(0) as ctx:
        ctx.attach_columns([c.data_ptr() for c in dev_cols], n)
        want, wcnt = separate_scan(ctx, terms, words)
    got = torch.full((words,), -1, dtype=torch.int32, device="cuda")
    gcnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    noalloc_scan(dev_cols, n, terms, got, gcnt, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(gcnt.item()) == wcnt and torch.equal(got, want)


def test_noalloc_requires_a_count():
    """dev_count is required here (rts_scan_separate_async accepts null)."""
    col = torch.zeros(64, dtype=torch.int32, device="cuda")
    bm = torch.zeros(2, dtype=torch.int32, device="cuda")
    arr, nt = R.make_terms([(0, 1, 2)])
    ptrs = (ctypes.c_void_p * 1)(col.data_ptr())
    rc = R.lib().rts_scan_separate_noalloc_async(ptrs, 1, 64, arr, nt, bm.data_ptr(), None, None)
    assert rc == -1


def test_noalloc_calls_after_the_device_is_full():
    """A caller's pool takes the rest of the device after one warm-up call:
    later calls still run, since the set-up placed the scratch array and the
    kernels on the device and the calls allocate nothing."""
    n = 2_000_033
    cols_np = [D.uniform(n, 21), D.uniform(n, 22, 1 << 12), D.zipf(n, 23, 1.5)]
    dev_cols = [torch.from_numpy(c.view(np.int32)).cuda() for c in cols_np]
    words = R.bitmap_words(n)
    s = torch.cuda.current_stream().cuda_stream
    queries = [[(0, 1 << 29, 1 << 31), (1, 100, 3000), (2, 0, 9)], [(2, 1, 50), (1, 0, 2000)], [(1, 7, 6)], []]
    with R.Context(0) as ctx:
        ctx.attach_columns([c.data_ptr() for c in dev_cols], n)
        wants = [separate_scan(ctx, q, words) for q in queries]
    outs = [(torch.full((words,), -1, dtype=torch.int32, device="cuda"),
             torch.full((1,), -1, dtype=torch.int64, device="cuda")) for _ in queries]
    noalloc_scan(dev_cols, n, queries[0], outs[0][0], outs[0][1], s)  # the warm-up call
    torch.cuda.synchronize()
    hog = None
    free, _ = torch.cuda.mem_get_info()
    for leave in (4 << 20, 8 << 20, 32 << 20):  # less than the 16 MiB scratch array
        try:
            hog = torch.empty(free - leave, dtype=torch.uint8, device="cuda")
            break
        except RuntimeError:
            continue
    assert hog is not None
    try:
        for _ in range(2):
            for q, (bm, cnt) in zip(queries, outs):
                noalloc_scan(dev_cols, n, q, bm, cnt, s)
        torch.cuda.synchronize()
    finally:
        del hog
        torch.cuda.empty_cache()
    for (bm, cnt), (want, wcnt) in zip(outs, wants):
        assert int(cnt.item()) == wcnt and torch.equal(bm, want)
