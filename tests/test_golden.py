"""The oracle pinned against the reference's own outputs.

tests/golden/golden.json was written by tests/golden/make_golden.py from the
reference's bindex.cpp (compiled unmodified, driven by oracle/ref_harness.cpp).
Here the oracle's restatement must reproduce every recorded hit count and
bitmap hash: the scalar filter for the authority, the restated BinDex for the
reference's BinDex (including its documented overflow edges)."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from rtscan_b200 import datagen as D

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")


def load():
    with open(GOLDEN) as f:
        return json.load(f)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def column(kind, n, seed):
    if kind == "uniform1000":
        return D.uniform(n, seed, 1000)
    return D.column(kind, n, seed)


_cols_cache = {}


def case_columns(case):
    key = case["name"]
    if key not in _cols_cache:
        cols = [column(c["kind"], case["n"], c["seed"]) for c in case["columns"]]
        for c, spec in zip(cols, case["columns"]):
            assert sha(c) == spec["sha"], f"generator drift for {spec}"
        _cols_cache.clear()
        _cols_cache[key] = cols
    return _cols_cache[key]


CASES = load()["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_scalar_filter_matches_reference(case):
    cols = case_columns(case)
    n = case["n"]
    ncols = len(cols)
    for q in case["queries"]:
        text = "\n".join(q["lines"]) + "\nexit\n"
        parsed = O.ref_parse_scan_cmd(text, ncols)[0]
        bm = O.mask_tail(O.raw_scan_entry(cols, parsed), n)
        assert O.popcount(bm, n) == q["raw_hits"], q["lines"]
        assert sha(bm) == q["raw_sha"], q["lines"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_restated_bindex_matches_reference(case):
    cols = case_columns(case)
    n = case["n"]
    idx = [O.BinDex(c, K=128) for c in cols]
    for q in case["queries"]:
        text = "\n".join(q["lines"]) + "\nexit\n"
        parsed = O.ref_parse_scan_cmd(text, len(cols))[0]
        merged = None
        for c, (cmd, tl, tr) in enumerate(parsed):
            bm = np.full(O.words(n), 0xFFFFFFFF, np.uint32)
            for pi, t1 in enumerate(tl):
                t2 = tr[pi] if tr else 0
                bm = idx[c].scan(cmd, t1, t2)
            merged = bm if merged is None else merged & bm
        merged = O.mask_tail(merged, n)
        assert O.popcount(merged, n) == q["bindex_hits"], q["lines"]
        assert sha(merged) == q["bindex_sha"], q["lines"]
        assert (q["bindex_sha"] == q["raw_sha"]) == q["bindex_equal"]


def test_golden_covers_the_reference_edges():
    """The fixture records where the reference's BinDex overflows (le/gt at
    2^32-1, bindex.cpp:1419-1427); nothing else may differ."""
    bad = [(c["name"], q["lines"]) for c in CASES for q in c["queries"] if not q["bindex_equal"]]
    assert sorted(l[0] for _, l in bad) == ["gt 4294967295", "le 4294967295"]


def test_c1_is_pinned_at_its_own_size():
    """The plain single-column scan's own configuration (2^24 uniform rows
    from default_rng(42), `bt 1932185501 2361592940`) is a golden case with
    the count the reference reports for it."""
    c1 = [c for c in CASES if c["name"] == "c1_uniform32_2p24_1c"]
    assert len(c1) == 1 and c1[0]["n"] == 1 << 24
    assert c1[0]["columns"] == [{"kind": "uniform", "seed": 42, "sha": c1[0]["columns"][0]["sha"]}]
    q = c1[0]["queries"][0]
    assert q["lines"] == ["bt 1932185501 2361592940"]
    assert q["raw_hits"] == q["bindex_hits"] == 1_677_722
