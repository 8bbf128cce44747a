"""Property tests of the scan_cmd path (CPU: parsing and lowering are host
code).  Random operator lines (all six operators, bounds at and next to the
domain edges, reversed `bt` bounds) rendered as scan_cmd text, parsed and
lowered by the library, must select exactly the rows that the reference's
own checker selects on the same columns (raw_scan per column and the AND
merge, bindex.cpp:1851-1957, in its C restatement); and any text at all
must parse or fail with RTS_ERR_PARSE."""
import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402

import rtscan_b200 as R  # noqa: E402
from oracle import oracle as O  # noqa: E402

MAXV = 0xFFFFFFFF
EDGES = [0, 1, 2, 3, 1000, 1 << 31, MAXV - 2, MAXV - 1, MAXV]
values = st.one_of(st.sampled_from(EDGES), st.integers(0, MAXV))
line = st.tuples(st.sampled_from(["lt", "le", "gt", "ge", "eq", "bt"]), values, values)


@settings(max_examples=150, deadline=None)
@given(ncols=st.integers(1, 4), data=st.data())
def test_parsed_queries_select_what_the_reference_checker_selects(ncols, data):
    nq = data.draw(st.integers(1, 4))
    queries = [[data.draw(line) for _ in range(ncols)] for _ in range(nq)]
    text = "".join(f"{op} {t1} {t2}\n" if op == "bt" else f"{op} {t1}\n"
                   for q in queries for op, t1, t2 in q) + "exit\n"
    qs = R.parse_scan_cmd(text, ncols)
    assert len(qs) == nq

    # columns made of the bounds themselves, their neighbours and the edges
    rng = np.random.default_rng(data.draw(st.integers(0, 2**32 - 1)))
    pool = sorted({min(MAXV, max(0, v + d)) for q in queries for _, a, b in q for v in (a, b)
                   for d in (-1, 0, 1)} | set(EDGES))
    n = 257
    cols = [rng.choice(np.array(pool, dtype=np.uint64), size=n).astype(np.uint32) for _ in range(ncols)]

    for i, q in enumerate(queries):
        want = O.raw_scan_entry(cols, [(op, [t1], [t2] if op == "bt" else []) for op, t1, t2 in q])
        terms, empty = qs.query(i)
        if empty:
            got = np.zeros(O.words(n), np.uint32)
        else:
            got, _ = O.range_scan([cols[c] for c, _, _ in terms], [t[1] for t in terms], [t[2] for t in terms])
        assert np.array_equal(got, want), (i, q, terms, empty)


# Arbitrary text, and text close to valid (operator words, numbers in every
# form, separators, stray characters), must parse or fail with
# RTS_ERR_PARSE: never another status, never a crash.
near_valid = st.lists(
    st.one_of(st.sampled_from(["lt", "le", "gt", "ge", "eq", "bt", "exit", "ltx", "", "zipf"]),
              st.integers(-(1 << 40), 1 << 40).map(str),
              st.sampled_from(["1e3", "0x1F", "2.5", "-1", "+7", "1,2,3", ",", "1,,2", "nan", "inf", "4294967296",
                               "99999999999999999999", ".", "e", "\t", " ", "\r", "\n", "\n\n", "#", "\x00"])),
    max_size=40).map(lambda toks: " ".join(toks))


@settings(max_examples=300, deadline=None)
@given(text=st.one_of(st.text(max_size=200), near_valid), ncols=st.integers(1, 5))
def test_any_text_parses_or_is_a_parse_error(text, ncols):
    try:
        qs = R.parse_scan_cmd(text, ncols)
    except R.RtsError as e:
        assert e.code == -5, (e.code, text)
        return
    for i in range(len(qs)):
        terms, empty = qs.query(i)
        assert len(terms) == ncols
        for c, lo, hi in terms:
            assert 0 <= c < ncols and 0 <= lo <= 0xFFFFFFFF and 0 <= hi <= 0xFFFFFFFF
            if not empty:
                assert lo <= hi
