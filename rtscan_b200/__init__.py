"""rtscan_b200 -- B200-native multi-column range-predicate scan.

Python front end over the C-ABI in ``include/rtscan_b200.h`` (the library
``librtscan_b200.so`` built by ``rtscan_b200.build``).  Scripting, tests and
the benchmark use it; the compute path is the CUDA library, and every call
raises ``RtsError`` if that library is missing or a call fails -- there is no
CPU fallback.

Names follow the reference (AntaresAlice/RTScan): a *column* is a uint32
array, a *query* is a conjunction of per-column range terms produced from a
``scan_cmd`` text, a *bitmap* is MSB-first packed 32-bit words
(bindex.cpp:1217), a *BinDex* is the per-column sieve index
(bindex.cpp:599-671).
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, List, Optional, Sequence, Tuple

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librtscan_b200.so")

OP_EQ, OP_LT, OP_GT, OP_LE, OP_GE, OP_BT = range(6)
OPS = {"eq": OP_EQ, "lt": OP_LT, "gt": OP_GT, "le": OP_LE, "ge": OP_GE, "bt": OP_BT}
BM_AND, BM_OR, BM_COPY, BM_NOT, BM_ANDNOT, BM_FILL = range(6)

STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_NOMEM", -4: "ERR_IO", -5: "ERR_PARSE",
          -6: "ERR_STATE", -7: "ERR_TIMEOUT", -8: "ERR_FULL", -9: "ERR_NODEV", -10: "ERR_CANCELLED"}


class RtsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Term(ctypes.Structure):
    """One conjunct lo <= column <= hi (rts_term)."""
    _fields_ = [("column", ctypes.c_int32), ("lo", ctypes.c_uint32), ("hi", ctypes.c_uint32)]

    def __repr__(self):
        return f"Term(col={self.column}, lo={self.lo}, hi={self.hi})"


class ServerConfig(ctypes.Structure):
    """rts_server_config (zero fields take the library defaults)."""
    _fields_ = [("max_active", ctypes.c_int32), ("max_queue", ctypes.c_int32), ("segment_rows", ctypes.c_uint64),
                ("max_inflight_steps", ctypes.c_int32)]


class BatchConfig(ctypes.Structure):
    """rts_batch_config: launch shape of the batched kernel."""
    _fields_ = [("variant", ctypes.c_int32), ("warps_per_cta", ctypes.c_int32),
                ("max_queries_per_pass", ctypes.c_int32), ("table_budget_bytes", ctypes.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("steps", ctypes.c_uint64), ("queued", ctypes.c_uint64),
                ("active", ctypes.c_uint32), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("p999_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("plans", ctypes.c_uint64), ("plan_ms_total", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.c_void_p
_U32P = ctypes.POINTER(ctypes.c_uint32)
_U64P = ctypes.POINTER(ctypes.c_uint64)
_TERMP = ctypes.POINTER(Term)
_lib = None

# (name, restype, argtypes) of every exported entry point.
_SIGS = [
    ("rts_last_error", ctypes.c_char_p, [_P]),
    ("rts_version", ctypes.c_char_p, []),
    ("rts_bitmap_words", ctypes.c_uint64, [ctypes.c_uint64]),
    ("rts_lower_op", ctypes.c_int32, [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, _U32P, _U32P,
                                      ctypes.POINTER(ctypes.c_int32)]),
    ("rts_parse_scan_cmd", ctypes.c_int32, [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(_P)]),
    ("rts_qset_size", ctypes.c_int32, [_P]),
    ("rts_qset_query", ctypes.c_int32, [_P, ctypes.c_int32, ctypes.POINTER(_TERMP), ctypes.POINTER(ctypes.c_int32),
                                        ctypes.POINTER(ctypes.c_int32)]),
    ("rts_qset_line", ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), _U32P,
                                       _U32P]),
    ("rts_qset_free", None, [_P]),
    ("rts_open", ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(_P)]),
    ("rts_close", None, [_P]),
    ("rts_load_columns", ctypes.c_int32, [_P, ctypes.POINTER(_P), ctypes.c_int32, ctypes.c_uint64]),
    ("rts_load_file", ctypes.c_int32, [_P, ctypes.c_char_p, ctypes.c_int32, ctypes.c_uint64]),
    ("rts_attach_columns", ctypes.c_int32, [_P, ctypes.POINTER(_P), ctypes.c_int32, ctypes.c_uint64]),
    ("rts_nrows", ctypes.c_uint64, [_P]),
    ("rts_ncols", ctypes.c_int32, [_P]),
    ("rts_device", ctypes.c_int32, [_P]),
    ("rts_sm_count", ctypes.c_int32, [_P]),
    ("rts_column_ptr", _P, [_P, ctypes.c_int32]),
    ("rts_kernel_launches", ctypes.c_uint64, [_P]),
    ("rts_scan_async", ctypes.c_int32, [_P, _TERMP, ctypes.c_int32, _P, _P, _P]),
    ("rts_scan_separate_async", ctypes.c_int32, [_P, _TERMP, ctypes.c_int32, _P, _P, _P]),
    ("rts_scan", ctypes.c_int32, [_P, _TERMP, ctypes.c_int32, _P, _U64P]),
    ("rts_bitmap_op_async", ctypes.c_int32, [_P, ctypes.c_int32, _P, _P, _P, ctypes.c_uint64, ctypes.c_uint32, _P]),
    ("rts_bitmap_count_async", ctypes.c_int32, [_P, _P, ctypes.c_uint64, _P, _P]),
    ("rts_build_bindex", ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int32]),
    ("rts_drop_bindex", ctypes.c_int32, [_P, ctypes.c_int32]),
    ("rts_bindex_areas", ctypes.c_int32, [_P, ctypes.c_int32, _U32P, _U64P, ctypes.c_int32]),
    ("rts_bindex_filter_vector", ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int32, _P]),
    ("rts_bindex_scan_async", ctypes.c_int32, [_P, _TERMP, ctypes.c_int32, _P, _P, _P]),
    ("rts_scan_batch_async", ctypes.c_int32, [_P, _TERMP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, _P,
                                              ctypes.c_uint64, _P, _P]),
    ("rts_scan_each_async", ctypes.c_int32, [_P, _TERMP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, _P,
                                             ctypes.c_uint64, _P, _P]),
    ("rts_scan_batch_host", ctypes.c_int32, [_P, ctypes.POINTER(_P), ctypes.c_int32, ctypes.c_uint64, _TERMP,
                                             ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, _P, ctypes.c_uint64,
                                             _P]),
    ("rts_host_transfer_bytes", ctypes.c_int32, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("rts_scan_separate_noalloc_async", ctypes.c_int32, [ctypes.POINTER(_P), ctypes.c_int32, ctypes.c_uint64,
                                                         _TERMP, ctypes.c_int32, _P, _P, _P]),
    ("rts_encode_table", ctypes.c_int32, [_P, ctypes.c_uint32, ctypes.c_uint32]),
    ("rts_encode_terms", ctypes.c_int32, [_P, _TERMP, ctypes.c_int32, _TERMP]),
    ("rts_save_bindex", ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_char_p]),
    ("rts_load_bindex", ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_char_p]),
    ("rts_bindex_file_info", ctypes.c_int32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_uint64)]),
    ("rts_bitmap_rows_async", ctypes.c_int32, [_P, _P, ctypes.c_uint64, _P, ctypes.c_uint64, _P, _P]),
    ("rts_bitmap_sum_async", ctypes.c_int32, [_P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P]),
    ("rts_scan_aggregate_async", ctypes.c_int32, [_P, _TERMP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P,
                                                  _P, _P]),
    ("rts_batch_prepare", ctypes.c_int32, [_P, _TERMP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, _P,
                                           ctypes.c_uint64, _P, ctypes.POINTER(_P)]),
    ("rts_batch_launch", ctypes.c_int32, [_P, _P]),
    ("rts_batch_release", None, [_P]),
    ("rts_set_batch_config", ctypes.c_int32, [_P, ctypes.POINTER(BatchConfig)]),
    ("rts_get_batch_config", ctypes.c_int32, [_P, ctypes.POINTER(BatchConfig)]),
    ("rts_autotune_batch", ctypes.c_int32, [_P, _TERMP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32,
                                            ctypes.c_char_p, ctypes.POINTER(BatchConfig)]),
    ("rts_autotune_report", ctypes.c_int32, [_P, ctypes.c_char_p, ctypes.c_uint64, _U64P]),
    ("rts_server_start", ctypes.c_int32, [_P, ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)]),
    ("rts_server_submit", ctypes.c_int32, [_P, _TERMP, ctypes.c_int32, _U64P]),
    ("rts_server_poll", ctypes.c_int32, [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32), _U64P]),
    ("rts_server_wait", ctypes.c_int32, [_P, ctypes.c_uint64, ctypes.c_int32, _U64P]),
    ("rts_server_fetch", ctypes.c_int32, [_P, ctypes.c_uint64, _P, _U64P]),
    ("rts_server_cancel", ctypes.c_int32, [_P, ctypes.c_uint64]),
    ("rts_server_get_stats", ctypes.c_int32, [_P, ctypes.POINTER(ServerStats)]),
    ("rts_server_stop", ctypes.c_int32, [_P]),
    ("rts_server_replay", ctypes.c_int32, [_P, _TERMP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
]


def lib() -> ctypes.CDLL:
    """Load the native library (raises RtsError when it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RtsError(-9, f"native library missing: {LIB_PATH} (run python -m rtscan_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_names() -> List[str]:
    return [s[0] for s in _SIGS]


def _check(rc: int, ctx=None):
    if rc != 0:
        msg = lib().rts_last_error(ctx)
        raise RtsError(rc, msg.decode() if msg else "")


def bindex_file_info(path: str):
    """(K, nrows) from a saved BinDex file's header; raises on a bad file."""
    k = ctypes.c_int32()
    n = ctypes.c_uint64()
    _check(lib().rts_bindex_file_info(path.encode(), ctypes.byref(k), ctypes.byref(n)))
    return k.value, n.value


def version() -> str:
    return lib().rts_version().decode()


def bitmap_words(nrows: int) -> int:
    return int(lib().rts_bitmap_words(nrows))


def lower_op(op, t1: int, t2: int = 0) -> Optional[Tuple[int, int]]:
    """Inclusive range of one reference operator, or None if it matches nothing."""
    code = OPS[op] if isinstance(op, str) else int(op)
    lo, hi, ne = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int32()
    _check(lib().rts_lower_op(code, t1 & 0xFFFFFFFF, t2 & 0xFFFFFFFF, ctypes.byref(lo), ctypes.byref(hi),
                              ctypes.byref(ne)))
    return (lo.value, hi.value) if ne.value else None


def make_terms(ranges: Sequence[Tuple[int, int, int]]):
    """ctypes array of Term from (column, lo, hi) triples."""
    arr = (Term * max(1, len(ranges)))()
    for i, (c, lo, hi) in enumerate(ranges):
        arr[i] = Term(c, lo & 0xFFFFFFFF, hi & 0xFFFFFFFF)
    return arr, len(ranges)


class QuerySet:
    """Parsed scan_cmd text (rts_parse_scan_cmd)."""

    def __init__(self, text: str, ncols: int):
        data = text.encode()
        h = _P()
        _check(lib().rts_parse_scan_cmd(data, len(data), ncols, ctypes.byref(h)))
        self._h = h
        self.ncols = ncols

    def __len__(self):
        return int(lib().rts_qset_size(self._h))

    def query(self, i: int) -> Tuple[List[Tuple[int, int, int]], bool]:
        tp, nt, em = _TERMP(), ctypes.c_int32(), ctypes.c_int32()
        _check(lib().rts_qset_query(self._h, i, ctypes.byref(tp), ctypes.byref(nt), ctypes.byref(em)))
        return [(tp[k].column, tp[k].lo, tp[k].hi) for k in range(nt.value)], bool(em.value)

    def line(self, i: int, c: int) -> Tuple[int, int, int]:
        op, t1, t2 = ctypes.c_int32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().rts_qset_line(self._h, i, c, ctypes.byref(op), ctypes.byref(t1), ctypes.byref(t2)))
        return op.value, t1.value, t2.value

    def queries(self) -> List[List[Tuple[int, int, int]]]:
        out = []
        for i in range(len(self)):
            terms, empty = self.query(i)
            out.append(terms)
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.rts_qset_free(h)
            self._h = None


def parse_scan_cmd(text: str, ncols: int) -> QuerySet:
    return QuerySet(text, ncols)


class PreparedQueries:
    """Queries packed once into the C-ABI's CSR arrays (terms + offsets), so
    repeated batch calls skip the Python-side packing."""

    def __init__(self, queries):
        flat = []
        offs = [0]
        for q in queries:
            flat.extend(q)
            offs.append(len(flat))
        self.terms, _ = make_terms(flat)
        self.offsets = (ctypes.c_int32 * len(offs))(*offs)
        self.n = len(queries)

    def csr(self):
        return self.terms, self.offsets

    def __len__(self):
        return self.n


def prepare(queries) -> PreparedQueries:
    return PreparedQueries(queries)


class PreparedBatch:
    """A batch replayed as one CUDA graph launch (rts_batch_prepare)."""

    def __init__(self, ctx, h):
        self.ctx = ctx
        self._h = h

    def launch(self, stream: int = 0):
        _check(lib().rts_batch_launch(self._h, stream), self.ctx._h)

    def release(self):
        if self._h:
            lib().rts_batch_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Server:
    """Continuous-batching scan server over a context's resident columns
    (rts_server_*).  The context must not be used for other calls while the
    server runs."""

    def __init__(self, ctx: "Context", max_active: int = 0, max_queue: int = 0, segment_rows: int = 0,
                 max_inflight_steps: int = 0):
        cfg = ServerConfig(max_active, max_queue, segment_rows, max_inflight_steps)
        h = _P()
        _check(lib().rts_server_start(ctx._h, ctypes.byref(cfg), ctypes.byref(h)), None)
        self._h = h
        self.ctx = ctx

    def _c(self, rc):
        _check(rc, None)

    def submit(self, terms) -> int:
        arr, n = make_terms(terms)
        t = ctypes.c_uint64()
        self._c(lib().rts_server_submit(self._h, arr, n, ctypes.byref(t)))
        return t.value

    def poll(self, ticket: int):
        done, cnt = ctypes.c_int32(), ctypes.c_uint64()
        self._c(lib().rts_server_poll(self._h, ticket, ctypes.byref(done), ctypes.byref(cnt)))
        return bool(done.value), (cnt.value if done.value else None)

    def wait(self, ticket: int, timeout_ms: int = 60000) -> int:
        cnt = ctypes.c_uint64()
        self._c(lib().rts_server_wait(self._h, ticket, timeout_ms, ctypes.byref(cnt)))
        return cnt.value

    def fetch(self, ticket: int, want_bitmap: bool = True):
        import numpy as np
        bm = np.zeros(bitmap_words(self.ctx.nrows), dtype=np.uint32) if want_bitmap else None
        cnt = ctypes.c_uint64()
        self._c(lib().rts_server_fetch(self._h, ticket, bm.ctypes.data if bm is not None else None,
                                       ctypes.byref(cnt)))
        return bm, cnt.value

    def cancel(self, ticket: int):
        self._c(lib().rts_server_cancel(self._h, ticket))

    def stats(self) -> dict:
        st = ServerStats()
        self._c(lib().rts_server_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def replay(self, queries, arrival_s):
        """Open-loop replay; returns per-query latency in ms (-1 = rejected)."""
        import numpy as np
        pq = queries if isinstance(queries, PreparedQueries) else PreparedQueries(queries)
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        lat = np.zeros(len(pq), dtype=np.float64)
        self._c(lib().rts_server_replay(self._h, pq.terms, pq.offsets, len(pq),
                                        arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return lat

    def stop(self):
        if self._h:
            h, self._h = self._h, None
            self._c(lib().rts_server_stop(h))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


class Context:
    """A device context with resident columns (rts_ctx)."""

    def __init__(self, device: int = 0):
        h = _P()
        _check(lib().rts_open(device, ctypes.byref(h)))
        self._h = h

    # -- lifetime
    def close(self):
        if self._h:
            lib().rts_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        _check(rc, self._h)

    # -- table
    def load_columns(self, cols) -> None:
        """Upload host uint32 arrays (numpy) as resident columns."""
        import numpy as np
        cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
        n = len(cols[0])
        if any(len(c) != n for c in cols):
            raise ValueError("columns differ in length")
        ptrs = (_P * len(cols))(*[c.ctypes.data for c in cols])
        self._c(lib().rts_load_columns(self._h, ptrs, len(cols), n))

    def load_file(self, path: str, ncols: int, nrows: int = 0) -> None:
        self._c(lib().rts_load_file(self._h, path.encode(), ncols, nrows))

    def attach_columns(self, dev_ptrs: Sequence[int], nrows: int) -> None:
        ptrs = (_P * len(dev_ptrs))(*dev_ptrs)
        self._c(lib().rts_attach_columns(self._h, ptrs, len(dev_ptrs), nrows))

    @property
    def nrows(self) -> int:
        return int(lib().rts_nrows(self._h))

    @property
    def ncols(self) -> int:
        return int(lib().rts_ncols(self._h))

    @property
    def sm_count(self) -> int:
        return int(lib().rts_sm_count(self._h))

    @property
    def launches(self) -> int:
        return int(lib().rts_kernel_launches(self._h))

    def column_ptr(self, c: int) -> int:
        return int(lib().rts_column_ptr(self._h, c) or 0)

    # -- scans (device pointers are plain ints, e.g. torch tensor data_ptr())
    def scan_async(self, terms, bitmap_ptr: int, count_ptr: int, stream: int = 0) -> None:
        arr, n = make_terms(terms)
        self._c(lib().rts_scan_async(self._h, arr, n, bitmap_ptr, count_ptr, stream))

    def encode_table(self, encode_min: int = 0, encode_max: int = 0) -> None:
        """Rank-encode the resident table (codes in [encode_min, encode_max),
        default [0, nrows))."""
        self._c(lib().rts_encode_table(self._h, encode_min, encode_max or self.nrows))

    def encode_terms(self, terms):
        """Terms on the original values -> terms on the codes."""
        arr, n = make_terms(terms)
        out = (Term * max(1, n))()
        self._c(lib().rts_encode_terms(self._h, arr, n, out))
        return [(t.column, t.lo, t.hi) for t in out[:n]]

    def save_bindex(self, column: int, path: str) -> None:
        self._c(lib().rts_save_bindex(self._h, column, path.encode()))

    def load_bindex(self, column: int, path: str) -> None:
        """Load a saved BinDex for `column` (checked against the resident column)."""
        self._c(lib().rts_load_bindex(self._h, column, path.encode()))

    def bitmap_rows_async(self, bitmap_ptr: int, nrows: int, rows_ptr: int, capacity: int, count_ptr: int,
                          stream: int = 0) -> None:
        """Ascending uint32 row ids of the set bits (at most `capacity`)."""
        self._c(lib().rts_bitmap_rows_async(self._h, bitmap_ptr, nrows, rows_ptr, capacity, count_ptr, stream))

    def bitmap_sum_async(self, bitmap_ptr: int, col_a: int, col_b: int, sum_ptr: int, stream: int = 0) -> None:
        """128-bit sum of column col_a (x col_b when col_b >= 0) over the set
        rows, as two uint64 words (low, high) at sum_ptr."""
        self._c(lib().rts_bitmap_sum_async(self._h, bitmap_ptr, col_a, col_b, sum_ptr, stream))

    def scan_aggregate_async(self, terms, col_a: int, col_b: int, count_ptr: int, sum_ptr: int,
                             stream: int = 0) -> None:
        """Query and aggregate in one pass, no bitmap."""
        arr, n = make_terms(terms)
        self._c(lib().rts_scan_aggregate_async(self._h, arr, n, col_a, col_b, count_ptr, sum_ptr, stream))

    def scan_separate_async(self, terms, bitmap_ptr: int, count_ptr: int, stream: int = 0) -> None:
        arr, n = make_terms(terms)
        self._c(lib().rts_scan_separate_async(self._h, arr, n, bitmap_ptr, count_ptr, stream))

    def bindex_scan_async(self, terms, bitmap_ptr: int, count_ptr: int, stream: int = 0) -> None:
        arr, n = make_terms(terms)
        self._c(lib().rts_bindex_scan_async(self._h, arr, n, bitmap_ptr, count_ptr, stream))

    def scan(self, terms, want_bitmap: bool = True):
        """Blocking scan to host memory: returns (bitmap numpy uint32 or None, count)."""
        import numpy as np
        arr, n = make_terms(terms)
        cnt = ctypes.c_uint64()
        bm = np.zeros(bitmap_words(self.nrows), dtype=np.uint32) if want_bitmap else None
        self._c(lib().rts_scan(self._h, arr, n, bm.ctypes.data if bm is not None else None, ctypes.byref(cnt)))
        return bm, int(cnt.value)

    @staticmethod
    def _csr(queries):
        if isinstance(queries, PreparedQueries):
            return queries.terms, queries.offsets
        return PreparedQueries(queries).csr()

    def scan_batch_async(self, queries, bitmaps_ptr: int, stride_words: int, counts_ptr: int, stream: int = 0):
        arr, off = self._csr(queries)
        self._c(lib().rts_scan_batch_async(self._h, arr, off, len(queries), bitmaps_ptr, stride_words, counts_ptr,
                                           stream))

    def scan_each_async(self, queries, bitmaps_ptr: int, stride_words: int, counts_ptr: int, stream: int = 0):
        arr, off = self._csr(queries)
        self._c(lib().rts_scan_each_async(self._h, arr, off, len(queries), bitmaps_ptr, stride_words, counts_ptr,
                                          stream))

    def scan_batch_host(self, host_cols, queries, host_bitmaps=None, stride_words: int = 0):
        """Host columns (numpy uint32, ideally pinned) in, host bitmaps out.
        Returns (bitmaps [nq, stride] uint32, counts [nq] uint64)."""
        import numpy as np
        n = len(host_cols[0])
        words = bitmap_words(n)
        stride = stride_words or words
        arr, off = self._csr(queries)
        if host_bitmaps is None:
            host_bitmaps = np.zeros((len(queries), stride), dtype=np.uint32)
        counts = np.zeros(len(queries), dtype=np.uint64)
        ptrs = (_P * len(host_cols))(*[c.ctypes.data for c in host_cols])
        self._c(lib().rts_scan_batch_host(self._h, ptrs, len(host_cols), n, arr, off, len(queries),
                                          host_bitmaps.ctypes.data, stride, counts.ctypes.data))
        return host_bitmaps, counts

    def host_transfer_bytes(self):
        """(host-to-device, device-to-host) bytes of the last scan_batch_host."""
        h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
        self._c(lib().rts_host_transfer_bytes(self._h, ctypes.byref(h2d), ctypes.byref(d2h)))
        return int(h2d.value), int(d2h.value)

    def prepare_batch(self, queries, bitmaps_ptr: int, stride_words: int, counts_ptr: int) -> "PreparedBatch":
        """Plan `queries` once and capture their launches in a CUDA graph."""
        arr, off = self._csr(queries)
        h = _P()
        self._c(lib().rts_batch_prepare(self._h, arr, off, len(queries), bitmaps_ptr, stride_words, counts_ptr,
                                        ctypes.byref(h)))
        return PreparedBatch(self, h)

    def batch_config(self) -> dict:
        c = BatchConfig()
        self._c(lib().rts_get_batch_config(self._h, ctypes.byref(c)))
        return c.as_dict()

    def set_batch_config(self, variant: int, warps_per_cta: int, max_queries_per_pass: int,
                         table_budget_bytes: int):
        c = BatchConfig(variant, warps_per_cta, max_queries_per_pass, table_budget_bytes)
        self._c(lib().rts_set_batch_config(self._h, ctypes.byref(c)))

    def autotune_batch(self, queries, cache_path: Optional[str] = None) -> dict:
        arr, off = self._csr(queries)
        c = BatchConfig()
        self._c(lib().rts_autotune_batch(self._h, arr, off, len(queries),
                                         cache_path.encode() if cache_path else None, ctypes.byref(c)))
        return c.as_dict()

    def autotune_report(self) -> dict:
        """Every candidate of the last autotune_batch with its time per call
        on the sample, the best and the default shape's times."""
        import json
        need = ctypes.c_uint64(0)
        self._c(lib().rts_autotune_report(self._h, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(max(1, need.value))
        self._c(lib().rts_autotune_report(self._h, buf, need.value, None))
        return json.loads(buf.value.decode()) if buf.value else {}

    def bitmap_op_async(self, op: int, dst: int, a: int, b: int, words: int, value: int = 0, stream: int = 0):
        self._c(lib().rts_bitmap_op_async(self._h, op, dst, a, b, words, value, stream))

    def bitmap_count_async(self, bitmap: int, nbits: int, count_ptr: int, stream: int = 0):
        self._c(lib().rts_bitmap_count_async(self._h, bitmap, nbits, count_ptr, stream))

    # -- BinDex
    def build_bindex(self, column: int, K: int = 128) -> None:
        self._c(lib().rts_build_bindex(self._h, column, K))

    def drop_bindex(self, column: int) -> None:
        self._c(lib().rts_drop_bindex(self._h, column))

    def bindex_filter_vector(self, column: int, k: int):
        import numpy as np
        out = np.zeros(bitmap_words(self.nrows), dtype=np.uint32)
        self._c(lib().rts_bindex_filter_vector(self._h, column, k, out.ctypes.data))
        return out

    def bindex_areas(self, column: int, K: int):
        import numpy as np
        s = np.zeros(K, dtype=np.uint32)
        r = np.zeros(K, dtype=np.uint64)
        self._c(lib().rts_bindex_areas(self._h, column, s.ctypes.data_as(_U32P), r.ctypes.data_as(_U64P), K))
        return s, r
