"""The oracle itself: its scalar filter against plain numpy, and its BinDex
restatement against its scalar filter (the two witnesses must agree except
at the reference's documented overflow edges)."""
import numpy as np
import pytest

from oracle import oracle as O
from rtscan_b200 import datagen as D


def np_bitmap(mask):
    n = len(mask)
    w = O.words(n)
    padded = np.zeros(w * 32, dtype=bool)
    padded[:n] = mask
    bits = padded.reshape(w, 32)
    weights = (1 << (31 - np.arange(32, dtype=np.uint64))).astype(np.uint64)
    return (bits.astype(np.uint64) * weights).sum(axis=1).astype(np.uint32)


@pytest.mark.parametrize("n", [1, 31, 33, 1000, 65537])
def test_raw_scan_matches_numpy(n):
    col = D.uniform(n, n, 1000)
    for op, t1, t2 in [("lt", 500, 0), ("le", 500, 0), ("gt", 10, 0), ("ge", 999, 0), ("eq", 7, 0),
                       ("bt", 100, 900)]:
        got = O.raw_scan(col, op, t1, t2)
        ref = {"lt": col < t1, "le": col <= t1, "gt": col > t1, "ge": col >= t1, "eq": col == t1,
               "bt": (col > t1) & (col < t2)}[op]
        assert np.array_equal(got, np_bitmap(ref))
        assert O.popcount(got, n) == int(ref.sum())


def test_range_scan_conjunction():
    n = 5000
    cols = [D.uniform(n, 1, 100), D.uniform(n, 2, 100)]
    bm, cnt = O.range_scan(cols, [10, 20], [60, 90])
    ref = (cols[0] >= 10) & (cols[0] <= 60) & (cols[1] >= 20) & (cols[1] <= 90)
    assert np.array_equal(bm, np_bitmap(ref)) and cnt == int(ref.sum())


def test_raw_scan_entry_and_merge():
    n = 4000
    cols = [D.uniform(n, 3, 50), D.uniform(n, 4, 50)]
    got = O.raw_scan_entry(cols, [("lt", [25], []), ("bt", [40], [5])])
    ref = (cols[0] < 25) & (cols[1] > 5) & (cols[1] < 40)
    assert np.array_equal(got, np_bitmap(ref))


# BinDex restatement vs scalar filter over many distributions and bounds.
KINDS = ["uniform", "uniform2p6", "uniform2p8", "zipf1.1", "zipf1.5", "normal"]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("K", [8, 128])
def test_bindex_restatement_agrees_with_scalar(kind, K):
    n = 450_000 if K == 128 else 60_001
    col = D.column(kind, n, 17)
    b = O.BinDex(col, K=K)
    s = np.sort(col)
    rng = np.random.default_rng(5)
    picks = [int(s[i]) for i in rng.integers(0, n, size=12)] + [int(s[0]), int(s[-1])]
    for t in picks:
        for op in ("lt", "le", "gt", "ge"):
            if (op == "le" and t == 0xFFFFFFFF) or (op == "gt" and t == 0xFFFFFFFF) or (op == "ge" and t == 0):
                continue  # reference overflow edges (bindex.cpp:1420,1425,1479)
            assert np.array_equal(O.mask_tail(b.scan(op, t), n), O.raw_scan(col, op, t)), (op, t)
        # eq on a value present in the column.  The reference asserts below
        # the minimum and when the value's run reaches the last area
        # (copy_filter_vector_xor, bindex.cpp:1092-1096); those are skipped.
        try:
            r = b.scan("eq", t)
        except RuntimeError:
            continue
        assert np.array_equal(O.mask_tail(r, n), O.raw_scan(col, "eq", t)), ("eq", t)
    for _ in range(10):
        a, c = sorted(int(x) for x in rng.choice(picks, 2))
        if c <= a or a + 1 < int(s[0]):
            continue
        assert np.array_equal(O.mask_tail(b.scan("bt", a, c), n), O.raw_scan(col, "bt", a, c)), (a, c)


def test_bindex_overflow_edges_are_the_references():
    """le 2^32-1 wraps to lt 0 inside the reference BinDex (bindex.cpp:1419-1421):
    the restatement reproduces that, the scalar filter does not."""
    n = 70_000
    col = D.uniform(n, 8)
    b = O.BinDex(col, K=8)
    assert O.popcount(b.scan("le", 0xFFFFFFFF), n) == 0
    assert O.popcount(O.raw_scan(col, "le", 0xFFFFFFFF), n) == n


def test_bindex_area_rule():
    """Area starts follow the duplicate rule of init_bindex (bindex.cpp:613-631):
    start values are the equal-count quantiles, start indexes the first row
    of that value unless it equals the previous area's start value."""
    n = 80_000
    col = D.uniform(n, 4, 16)  # heavy duplicates: runs span several areas
    K = 32
    b = O.BinDex(col, K=K)
    s = np.sort(col)
    sv, si = b.area_start_values(), b.area_start_indices()
    avg = n // K
    for i in range(1, K):
        assert sv[i] == s[i * avg]
        if sv[i] == sv[i - 1]:
            assert si[i] == i * avg
        else:
            assert si[i] == np.searchsorted(s, sv[i], side="left")
