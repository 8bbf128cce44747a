"""After the scan: bitmap -> ascending row ids, masked sums and the fused
scan-and-aggregate, checked against numpy restatements (exact integers)."""
import numpy as np
import pytest

import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev_words(words):
    return torch.from_numpy(words.view(np.int32).copy()).cuda()


def rows_of(bitmap, n):
    """Set rows of an MSB-first bitmap, ascending (restatement)."""
    bits = np.unpackbits(bitmap.astype(">u4").view(np.uint8))[:n]
    return np.nonzero(bits)[0].astype(np.uint32)


def sum128(dev):
    lo, hi = (int(x) & (2 ** 64 - 1) for x in dev.cpu().tolist())
    return lo | (hi << 64)


@pytest.mark.parametrize("n", [1, 31, 33, 4096 * 32, 4096 * 32 + 5, 1_000_003])
@pytest.mark.parametrize("density", [0.0, 0.01, 0.5, 1.0])
def test_bitmap_rows(ctx, n, density):
    rng = np.random.default_rng(n + int(density * 100))
    words = R.bitmap_words(n)
    bm = (rng.random(words * 32) < density).astype(np.uint8)
    bm = np.packbits(bm).view(">u4").astype(np.uint32)
    bm[-1] |= 0xFFFFFFFF >> (n & 31) if n & 31 else 0  # garbage past nrows must be ignored
    want = rows_of(bm, n)
    ctx.load_columns([np.zeros(max(n, 1), np.uint32)])
    out = torch.full((max(1, len(want)) + 7,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    d = dev_words(bm)
    ctx.bitmap_rows_async(d.data_ptr(), n, out.data_ptr(), len(want), cnt.data_ptr())
    torch.cuda.synchronize()
    assert int(cnt.item()) == len(want)
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got[:len(want)], want)
    assert (got[len(want):] == 0xFFFFFFFF).all(), "wrote past capacity"


def test_bitmap_rows_capacity_truncates(ctx):
    n = 300_000
    rng = np.random.default_rng(3)
    bm = np.packbits((rng.random(R.bitmap_words(n) * 32) < 0.3).astype(np.uint8)).view(">u4").astype(np.uint32)
    bm[-1] &= ~(0xFFFFFFFF >> (n & 31)) & 0xFFFFFFFF
    want = rows_of(bm, n)
    ctx.load_columns([np.zeros(n, np.uint32)])
    cap = 1000
    out = torch.full((cap + 4,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.bitmap_rows_async(dev_words(bm).data_ptr(), n, out.data_ptr(), cap, cnt.data_ptr())
    torch.cuda.synchronize()
    assert int(cnt.item()) == len(want)
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got[:cap], want[:cap])
    assert (got[cap:] == 0xFFFFFFFF).all()


@pytest.mark.parametrize("n", [1, 1000, 1024 * 37 + 9, 2_000_000])
def test_bitmap_sum(ctx, n):
    cols = [D.uniform(n, 11), D.uniform(n, 12), D.zipf(n, 13, 1.2)]
    ctx.load_columns(cols)
    want_bm, _ = O.range_scan([cols[2]], [0], [40])
    sel = rows_of(want_bm, n)
    bm = dev_words(want_bm)
    s = torch.zeros(2, dtype=torch.int64, device="cuda")
    for a, b in [(0, -1), (1, -1), (0, 1), (2, 2)]:
        ctx.bitmap_sum_async(bm.data_ptr(), a, b, s.data_ptr())
        torch.cuda.synchronize()
        va = [int(x) for x in cols[a][sel]]
        want = sum(va) if b < 0 else sum(x * int(y) for x, y in zip(va, cols[b][sel]))
        assert sum128(s) == want, (a, b)


def test_bitmap_sum_overflows_64_bits(ctx):
    n = 1 << 20
    a = np.full(n, 0xFFFFFFFF, np.uint32)
    ctx.load_columns([a, a])
    bm = dev_words(O.mask_tail(np.full(R.bitmap_words(n), 0xFFFFFFFF, np.uint32), n))
    s = torch.zeros(2, dtype=torch.int64, device="cuda")
    ctx.bitmap_sum_async(bm.data_ptr(), 0, 1, s.data_ptr())
    torch.cuda.synchronize()
    assert sum128(s) == n * 0xFFFFFFFF * 0xFFFFFFFF  # > 2^64


def scan_agg(ctx, terms, a, b):
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.zeros(2, dtype=torch.int64, device="cuda")
    ctx.scan_aggregate_async(terms, a, b, cnt.data_ptr(), s.data_ptr())
    torch.cuda.synchronize()
    return int(cnt.item()), sum128(s)


def expect_agg(cols, terms, a, b):
    n = len(cols[0])
    hit = np.ones(n, bool)
    for c, lo, hi in terms:
        hit &= (cols[c] >= lo) & (cols[c] <= hi)
    if a < 0:
        return int(hit.sum()), 0
    va = cols[a][hit].astype(object)
    vb = cols[b][hit].astype(object) if b >= 0 else 1
    return int(hit.sum()), int(np.sum(va * vb)) if hit.any() else 0


@pytest.mark.parametrize("n", [1, 7, 1027, 1_000_001])
def test_scan_aggregate(ctx, n):
    cols = [D.uniform(n, 21), D.uniform(n, 22, 1000), D.zipf(n, 23, 1.3), D.normal(n, 24), D.uniform(n, 25, 64)]
    ctx.load_columns(cols)
    cases = [
        ([(1, 100, 600)], -1, -1),
        ([(1, 100, 600)], 0, -1),
        ([(1, 100, 600), (2, 0, 50)], 0, 3),
        ([(1, 100, 600), (1, 300, 999), (4, 3, 40)], 1, 1),   # merged terms; a x a with a constrained
        ([(3, 1 << 30, 3 << 30)], 3, -1),                      # aggregate column also in the predicate
        ([], 4, -1),                                           # no predicate: every row
        ([], -1, -1),
        ([(4, 50, 10)], 0, 1),                                 # empty range
        ([(1, 900, 999), (1, 0, 100)], 0, -1),                 # disjoint on one column
        ([(c, 0, 0xFFFFFFFF) for c in range(5)], 2, 4),        # 5 columns, always true
    ]
    for terms, a, b in cases:
        assert scan_agg(ctx, terms, a, b) == expect_agg(cols, terms, a, b), (terms, a, b)


def test_scan_aggregate_q6_shape(ctx):
    """TPC-H Q6 shape on synthetic integer-coded columns: shipdate in
    [19940101, 19950101), discount in [5, 7], quantity < 24, summing
    extendedprice x discount."""
    n = 3_000_000
    rng = np.random.default_rng(6)
    shipdate = (19920101 + rng.integers(0, 70000, n)).astype(np.uint32)
    discount = rng.integers(0, 11, n).astype(np.uint32)
    quantity = rng.integers(1, 51, n).astype(np.uint32)
    price = rng.integers(90000, 10_500_000, n).astype(np.uint32)
    cols = [shipdate, discount, quantity, price]
    ctx.load_columns(cols)
    terms = [(0, 19940101, 19950100), (1, 5, 7), (2, 0, 23)]
    assert scan_agg(ctx, terms, 3, 1) == expect_agg(cols, terms, 3, 1)


def test_aggregate_argument_errors(ctx):
    ctx.load_columns([np.arange(100, dtype=np.uint32)])
    s = torch.zeros(2, dtype=torch.int64, device="cuda")
    with pytest.raises(R.RtsError):
        ctx.scan_aggregate_async([(0, 1, 2)], 3, -1, 0, s.data_ptr())   # column out of range
    with pytest.raises(R.RtsError):
        ctx.scan_aggregate_async([(0, 1, 2)], -1, 0, 0, s.data_ptr())   # col_b without col_a
    with pytest.raises(R.RtsError):
        ctx.bitmap_sum_async(0, 0, -1, s.data_ptr())                    # null bitmap
