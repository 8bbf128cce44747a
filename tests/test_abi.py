"""The C-ABI library loads on a CPU-only host and exports every entry point
include/rtscan_b200.h declares; context-free calls behave as documented."""
import ctypes
import os
import re

import pytest

import rtscan_b200 as R
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"RTS_API\s+[^;(]*?\b(rts_\w+)\s*\(", text)
    return names


def test_header_declares_entry_points():
    names = declared_entry_points()
    assert len(names) >= 30
    assert len(set(names)) == len(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(R.LIB_PATH)
    missing = [n for n in declared_entry_points() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_header():
    assert set(declared_entry_points()) == set(R.exported_names())


def test_version_and_words():
    assert "sm_100a" in R.version()
    for n, w in [(0, 0), (1, 1), (31, 1), (32, 1), (33, 2), (10**8, 3125000), (1 << 28, 1 << 23)]:
        assert R.bitmap_words(n) == w


@pytest.mark.parametrize("op", list(O.OPS))
def test_lower_op_matches_oracle(op):
    vals = [0, 1, 2, 5, 1 << 31, 0xFFFFFFFE, 0xFFFFFFFF]
    for t1 in vals:
        for t2 in vals:
            assert R.lower_op(op, t1, t2) == O.lower_op(op, t1, t2), (op, t1, t2)


def test_lower_op_exhaustive_small_domain():
    """Lowered range selects exactly the rows raw_scan selects, on every
    value of a small domain around both edges."""
    import numpy as np
    xs = np.array(list(range(0, 8)) + list(range(0xFFFFFFF8, 0x100000000)), dtype=np.uint64).astype(np.uint32)
    targets = [0, 1, 3, 7, 0xFFFFFFF8, 0xFFFFFFFE, 0xFFFFFFFF]
    for op in O.OPS:
        for t1 in targets:
            for t2 in (targets if op == "bt" else [0]):
                want = O.raw_scan(xs, op, *((min(t1, t2), max(t1, t2)) if op == "bt" else (t1, t2)))
                r = R.lower_op(op, t1, t2)
                got = np.zeros_like(want)
                if r is not None:
                    got = O.range_scan([xs], [r[0]], [r[1]])[0]
                assert np.array_equal(got, want), (op, t1, t2)


def test_bad_operator_is_an_error():
    with pytest.raises(R.RtsError) as e:
        R.lower_op(9, 1, 2)
    assert e.value.code == -1


def test_open_without_gpu_fails_loudly():
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(R.RtsError) as e:
        R.Context(0)
    assert e.value.code == -9
