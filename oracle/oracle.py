"""THE ORACLE (test infrastructure only) -- Python front end.

Loads ``oracle/liborc.so`` (the plain-C restatement in ``scan_oracle.c``) and
offers numpy-friendly calls.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` may import this module; the product
(``rtscan_b200``) never does.

Reference anchors (AntaresAlice/RTScan):
  * scalar filter ``raw_scan``            bindex.cpp:1851-1892
  * checker ``raw_scan_entry``            bindex.cpp:1894-1957
  * AND merge ``refine_result_bitmap``    bindex.cpp:1259-1281
  * hit count of ``compare_bitmap``       bindex.cpp:1959-1978
  * BinDex build/query                    bindex.cpp:599-671, 1365-1691
  * scan_cmd parsing                      bindex.cpp:238-245, 1840-1849, 2165-2189
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OPS = {"eq": 0, "lt": 1, "gt": 2, "le": 3, "ge": 4, "bt": 5}
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
P32 = ctypes.POINTER(ctypes.c_uint32)


def build() -> str:
    """Compile liborc.so (plain C, seconds)."""
    subprocess.run(["make", "-s", "-C", HERE, "liborc.so"], check=True)
    return os.path.join(HERE, "liborc.so")


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_words.restype = U64
        L.orc_words.argtypes = [U64]
        L.orc_raw_scan.argtypes = [P32, U64, ctypes.c_int, U32, U32, P32]
        L.orc_and_bitmap.argtypes = [P32, P32, U64]
        L.orc_popcount.restype = U64
        L.orc_popcount.argtypes = [P32, U64]
        L.orc_lower_op.restype = ctypes.c_int
        L.orc_lower_op.argtypes = [ctypes.c_int, U32, U32, P32, P32]
        L.orc_range_scan.restype = U64
        L.orc_range_scan.argtypes = [ctypes.POINTER(P32), ctypes.c_int, P32, P32, U64, P32]
        L.orc_bindex_build.restype = ctypes.c_void_p
        L.orc_bindex_build.argtypes = [P32, U32, ctypes.c_int, ctypes.c_int]
        L.orc_bindex_free.argtypes = [ctypes.c_void_p]
        L.orc_bindex_scan_op.restype = ctypes.c_int
        L.orc_bindex_scan_op.argtypes = [ctypes.c_void_p, P32, ctypes.c_int, U32, U32]
        L.orc_bindex_area_start_value.restype = U32
        L.orc_bindex_area_start_value.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_bindex_area_start_index.restype = U32
        L.orc_bindex_area_start_index.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _LIB = L
    return _LIB


def _p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(P32)


def words(n: int) -> int:
    return (n + 31) // 32


def raw_scan(col: np.ndarray, op: str, t1: int, t2: int = 0, bitmap: Optional[np.ndarray] = None) -> np.ndarray:
    """raw_scan (bindex.cpp:1851): XOR-sets matching rows into ``bitmap``."""
    col = np.ascontiguousarray(col, dtype=np.uint32)
    if bitmap is None:
        bitmap = np.zeros(words(len(col)), dtype=np.uint32)
    lib().orc_raw_scan(_p(col), len(col), OPS[op], t1 & 0xFFFFFFFF, t2 & 0xFFFFFFFF, _p(bitmap))
    return bitmap


def raw_scan_entry(cols: Sequence[np.ndarray], lines: Sequence[Tuple[str, List[int], List[int]]]) -> np.ndarray:
    """The reference checker for one query: per column, raw_scan of every
    target (bt swapped when t1>t2) XORed into a zeroed bitmap, then the AND
    merge into column 0's bitmap (bindex.cpp:1894-1957, 2276-2286)."""
    n = len(cols[0])
    merged = None
    for c, (cmd, tl, tr) in enumerate(lines):
        bm = np.zeros(words(n), dtype=np.uint32)
        for pi, t1 in enumerate(tl):
            t2 = tr[pi] if tr else 0
            if cmd == "bt" and t1 > t2:
                t1, t2 = t2, t1
            if cmd in OPS:
                raw_scan(cols[c], cmd, t1, t2, bm)
        if merged is None:
            merged = bm
        else:
            lib().orc_and_bitmap(_p(merged), _p(bm), len(bm))
    return merged


def popcount(bm: np.ndarray, n: int) -> int:
    return int(lib().orc_popcount(_p(np.ascontiguousarray(bm, dtype=np.uint32)), n))


def lower_op(op: str, t1: int, t2: int = 0) -> Optional[Tuple[int, int]]:
    """Canonical inclusive range for one op, or None when nothing matches."""
    lo, hi = U32(0), U32(0)
    r = lib().orc_lower_op(OPS[op], t1 & 0xFFFFFFFF, t2 & 0xFFFFFFFF, ctypes.byref(lo), ctypes.byref(hi))
    if r < 0:
        raise ValueError(op)
    return (lo.value, hi.value) if r == 1 else None


def range_scan(cols: Sequence[np.ndarray], lo: Sequence[int], hi: Sequence[int]) -> Tuple[np.ndarray, int]:
    """Conjunctive scalar filter: AND over terms of lo[t] <= cols[t] <= hi[t]."""
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    n = len(cols[0]) if cols else 0
    arr = (P32 * max(1, len(cols)))(*[_p(c) for c in cols])
    lo_a = np.ascontiguousarray(lo, dtype=np.uint32)
    hi_a = np.ascontiguousarray(hi, dtype=np.uint32)
    bm = np.zeros(max(1, words(n)), dtype=np.uint32)
    cnt = lib().orc_range_scan(arr, len(cols), _p(lo_a), _p(hi_a), n, _p(bm))
    return bm[: words(n)], int(cnt)


class BinDex:
    """Restated BinDex of one column (init_bindex, bindex.cpp:599-671)."""

    def __init__(self, col: np.ndarray, K: int = 128, block_init: int = 3276):
        self.col = np.ascontiguousarray(col, dtype=np.uint32)
        self.n = len(self.col)
        self.h = lib().orc_bindex_build(_p(self.col), self.n, K, block_init)
        if not self.h:
            raise ValueError("bad BinDex arguments")
        self.K = K

    def scan(self, op: str, t1: int, t2: int = 0) -> np.ndarray:
        r = np.zeros(words(self.n), dtype=np.uint32)
        rc = lib().orc_bindex_scan_op(self.h, _p(r), OPS[op], t1 & 0xFFFFFFFF, t2 & 0xFFFFFFFF)
        if rc != 0:
            raise RuntimeError("reference asserts on this query")
        return r

    def filter_vector(self, k: int) -> np.ndarray:
        L = lib()
        L.orc_bindex_fv.restype = P32
        L.orc_bindex_fv.argtypes = [ctypes.c_void_p, ctypes.c_int]
        p = L.orc_bindex_fv(self.h, k)
        return np.ctypeslib.as_array(p, shape=(words(self.n),)).copy()

    def area_start_values(self) -> np.ndarray:
        return np.array([lib().orc_bindex_area_start_value(self.h, a) for a in range(self.K)], dtype=np.uint32)

    def area_start_indices(self) -> np.ndarray:
        return np.array([lib().orc_bindex_area_start_index(self.h, a) for a in range(self.K)], dtype=np.uint32)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_bindex_free(h)
            self.h = None


def mask_tail(bm: np.ndarray, n: int) -> np.ndarray:
    """Zero the bits past row n-1 (the reference leaves them undefined)."""
    bm = bm.copy()
    rem = n & 31
    if rem:
        bm[n >> 5] &= np.uint32((0xFFFFFFFF << (32 - rem)) & 0xFFFFFFFF)
    return bm


# --------------------------------------------------------------------------
# scan_cmd restatement (bindex.cpp:238-245 stringSplit, 1840-1849
# get_target_numbers, query loop 2165-2189).  Test-side only; the product
# parser lives in rtscan_b200/csrc/scan_cmd.cpp.
# --------------------------------------------------------------------------

def cast_code(v: float) -> int:
    """(CODE)stod(value): truncation toward zero, then the low 32 bits, which
    is what x86-64 g++ emits for a double -> uint32 conversion."""
    i = int(v)  # truncates toward zero
    return i & 0xFFFFFFFF


def ref_parse_scan_cmd(text: str, ncols: int):
    """Split a scan_cmd text into queries of ``ncols`` lines each.  Returns a
    list of queries, each a list of (cmd, target_l, target_r)."""
    queries = []
    lines = text.split("\n")
    i = 0
    while True:
        q = []
        for _ in range(ncols):
            if i >= len(lines):
                return queries
            raw = lines[i]
            i += 1
            parts = raw.split(" ")
            if parts[0] == "exit":
                return queries
            tl = [cast_code(float(x)) for x in parts[1].split(",") if x != ""] if len(parts) > 1 else []
            tr = [cast_code(float(x)) for x in parts[2].split(",") if x != ""] if len(parts) > 2 else []
            q.append((parts[0], tl, tr))
        queries.append(q)
