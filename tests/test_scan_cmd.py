"""The product scan_cmd parser against the oracle's restatement of the
reference parsing (stringSplit, get_target_numbers and the query loop,
bindex.cpp:238-245, 1840-1849, 2165-2189)."""
import pytest

import rtscan_b200 as R
from oracle import oracle as O


def lowered(ref_query):
    """Reference lines of one query -> inclusive terms (+ empty flag)."""
    terms, empty = [], False
    for c, (cmd, tl, tr) in enumerate(ref_query):
        t1 = tl[0]
        t2 = tr[0] if tr else 0
        r = O.lower_op(cmd, t1, t2)
        if r is None:
            empty = True
            r = (1, 0)
        terms.append((c, r[0], r[1]))
    return terms, empty


def sweep_text(ncols, thresholds, notes="width 32\n\nlt 1\nlt 2\n"):
    lines = []
    for t in thresholds:
        lines += [f"lt {t}"] * ncols
    return "\n".join(lines) + "\nexit\n" + notes


@pytest.mark.parametrize("ncols", [1, 2, 3, 4])
def test_sweep_files(ncols):
    # the shape of the reference's uniform sweeps: lt at 10% steps of 2^32
    ths = [1] + [int(i * 0xFFFFFFFF / 10) for i in range(1, 10)] + [0xFFFFFFFF]
    text = sweep_text(ncols, ths)
    qs = R.parse_scan_cmd(text, ncols)
    ref = O.ref_parse_scan_cmd(text, ncols)
    assert len(qs) == len(ref) == len(ths)
    for i in range(len(qs)):
        assert qs.query(i) == lowered(ref[i])


def test_all_operators_and_number_forms():
    text = ("lt 5\nle 1e3\ngt 4294967295\nge 0\neq 12.9\nbt 100 7\n"
            "lt 4294967296\nle -1\nbt 3 4\neq 0x10\nge +7\nlt 2.5e2\n"
            "exit\n")
    ref = O.ref_parse_scan_cmd(text.replace("0x10", "16"), 6)
    qs = R.parse_scan_cmd(text, 6)
    assert len(qs) == 2
    for i in range(2):
        assert qs.query(i) == lowered(ref[i])
    # conversions match (CODE)stod: 4294967296 -> 0, -1 -> 4294967295, 12.9 -> 12
    assert qs.line(1, 0) == (R.OP_LT, 0, 0)
    assert qs.line(1, 1) == (R.OP_LE, 0xFFFFFFFF, 0)
    assert qs.line(0, 4) == (R.OP_EQ, 12, 0)
    assert qs.line(0, 5) == (R.OP_BT, 100, 7)


def test_exit_and_trailing_notes():
    text = "lt 5\nlt 6\nexit\nzipf 1.5 304045\n\nlt 1\nlt 1\n"
    assert len(R.parse_scan_cmd(text, 2)) == 1
    assert len(R.parse_scan_cmd("exit\nlt 3\n", 1)) == 0
    # end of text without exit; partial last query dropped
    assert len(R.parse_scan_cmd("lt 5\nlt 6\nlt 7\n", 2)) == 1
    # CRLF line ends
    qs = R.parse_scan_cmd("lt 5\r\nge 2\r\nexit\r\n", 2)
    assert qs.query(0)[0] == [(0, 0, 4), (1, 2, 0xFFFFFFFF)]


def test_comma_lists_expand():
    qs = R.parse_scan_cmd("lt 10,20,30\nge 7\nexit\n", 2)
    assert len(qs) == 3
    assert [qs.query(i)[0][0] for i in range(3)] == [(0, 0, 9), (0, 0, 19), (0, 0, 29)]
    assert all(qs.query(i)[0][1] == (1, 7, 0xFFFFFFFF) for i in range(3))
    qs = R.parse_scan_cmd("bt 1,5 9,2\nexit\n", 1)
    assert [qs.query(i)[0] for i in range(2)] == [[(0, 2, 8)], [(0, 3, 4)]]


def test_empty_queries_flagged():
    qs = R.parse_scan_cmd("lt 0\nge 1\nbt 5 6\nge 1\nexit\n", 2)
    assert qs.query(0)[1] is True
    assert qs.query(1)[1] is True


@pytest.mark.parametrize("text,ncols", [
    ("foo 5\nexit\n", 1),
    ("lt\nexit\n", 1),
    ("lt abc\nexit\n", 1),
    ("bt 5\nexit\n", 1),
    ("lt 5 6\nexit\n", 1),
    ("lt 5\n\nlt 6\nexit\n", 2),
    ("bt 1,2 3\nexit\n", 1),
    ("lt 1,2\nlt 1,2,3\nexit\n", 2),
    ("lt nan\nexit\n", 1),
    ("lt 1e300\nexit\n", 1),
])
def test_malformed_is_parse_error(text, ncols):
    with pytest.raises(R.RtsError) as e:
        R.parse_scan_cmd(text, ncols)
    assert e.value.code == -5
    assert "line" in str(e.value)


def test_bad_arguments():
    with pytest.raises(R.RtsError):
        R.parse_scan_cmd("lt 1\n", 0)
