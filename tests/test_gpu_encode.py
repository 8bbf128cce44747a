"""Rank encoding (remap.cpp's normalEncode, made deterministic): the codes
are an order-preserving, tie-by-row-id permutation of the code range, and a
scan of the encoded table with rewritten terms selects exactly the rows the
original terms select on the original table."""
import numpy as np
import pytest

import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def scan(ctx, terms):
    n = ctx.nrows
    bm = torch.zeros(R.bitmap_words(n), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.scan_async(terms, bm.data_ptr(), cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return bm.cpu().numpy().view(np.uint32), int(cnt.item())


@pytest.mark.parametrize("kind", ["uniform", "uniform2p6", "zipf1.5", "normal"])
def test_encoded_scans_equal_original_scans(ctx, kind):
    n = 500_003
    cols = [D.column(kind, n, 5), D.zipf(n, 6, 1.1)]
    ctx.load_columns(cols)
    rng = np.random.default_rng(8)
    qs = D.batch_queries(cols, 40, seed=9)
    s0 = np.sort(cols[0])
    qs += [[(0, 0, 0)], [(0, 0xFFFFFFFF, 0xFFFFFFFF)], [(0, int(s0[0]), int(s0[0]))], [(0, int(s0[-1]), 0xFFFFFFFF)],
           [(0, 0, int(s0[0]) - 1 if s0[0] else 0)], [(0, int(s0[-1]) + 1 if s0[-1] < 0xFFFFFFFF else 0, 0xFFFFFFFF)],
           [(1, 3, 2)], [(0, int(s0[n // 2]), int(s0[n // 2])), (1, 0, 5)]]
    for _ in range(20):  # bounds on and around stored values
        v = int(s0[rng.integers(0, n)])
        qs.append([(0, max(0, v - int(rng.integers(0, 2))), min(0xFFFFFFFF, v + int(rng.integers(0, 2))))])
    want = [scan(ctx, q) for q in qs]
    ctx.encode_table()
    for q, (wb, wc) in zip(qs, want):
        eq = ctx.encode_terms(q)
        gb, gc = scan(ctx, eq)
        assert gc == wc and np.array_equal(gb, wb), (q, eq)


def test_codes_are_an_order_preserving_permutation(ctx):
    n = 100_000
    col = D.uniform(n, 7, 300)  # many duplicates
    ctx.load_columns([col, np.arange(n, dtype=np.uint32)])
    ctx.encode_table(1000, 1000 + 3 * n + 2)   # step 3
    # read the codes back by scanning each code range [code, code]: instead,
    # check order and ties through rewritten single-value terms
    order = np.lexsort((np.arange(n), col))      # stable sort by value, ties by row
    first = {}
    for r, row in enumerate(order):
        first.setdefault(int(col[row]), r)
    for v in (0, 1, 150, 299):
        (c, lo, hi), = ctx.encode_terms([(0, v, v)])
        cnt = int((col == v).sum())
        assert lo == 1000 + 3 * first[v] and hi == 1000 + 3 * (first[v] + cnt - 1)
    bm, cnt = scan(ctx, [(0, 1000, 1000 + 3 * 9)])   # the ten smallest codes: ten rows
    assert cnt == 10
    rows = np.nonzero(np.unpackbits(bm.astype(">u4").view(np.uint8))[:n])[0]
    assert np.array_equal(rows, np.sort(order[:10]))


def test_encoding_errors(ctx):
    ctx.load_columns([np.arange(1000, dtype=np.uint32)])
    with pytest.raises(R.RtsError):
        ctx.encode_terms([(0, 1, 2)])          # not encoded yet
    with pytest.raises(R.RtsError):
        ctx.encode_table(0, 999)               # fewer codes than rows
    ctx.encode_table()
    with pytest.raises(R.RtsError):
        ctx.encode_table()                     # already encoded
    with pytest.raises(R.RtsError):
        ctx.encode_terms([(3, 1, 2)])          # column out of range
    ctx.load_columns([np.arange(10, dtype=np.uint32)])   # a new table is not encoded
    with pytest.raises(R.RtsError):
        ctx.encode_terms([(0, 1, 2)])
