"""Property test of the scan_cmd path: random operator lines (all six
operators, bounds at and next to the domain edges, reversed `bt` bounds)
rendered as scan_cmd text, parsed and lowered by the library, must select
exactly the rows that the reference's own checker selects on the same
columns (raw_scan per column and the AND merge, bindex.cpp:1851-1957, in its
C restatement).  Runs on the CPU: parsing and lowering are host code."""
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
