"""The allocation-free scan entry point (rts_scan_separate_noalloc_async).

It serves callers that cannot let a library allocate device memory (an
engine whose pool allocator owns all of HBM, or a latency-critical path
where cudaMalloc's device-wide synchronisation is not acceptable).  Called
through the C-ABI with ctypes, it must produce the same bitmap and count as
the context-based rts_scan_separate_async -- bit-exact, the tolerance every
scan test here uses -- on two calls in a row that share its static scratch
array, whether this file runs alone in a fresh process or after the other
tests.  Kept in a file of its own that pytest collects last."""
import ctypes

import numpy as np
import pytest

import rtscan_b200 as R
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def noalloc_scan(dev_cols, n, terms, bm, cnt, stream):
    arr, nt = R.make_terms(terms)
    ptrs = (ctypes.c_void_p * len(dev_cols))(*[c.data_ptr() for c in dev_cols])
    rc = R.lib().rts_scan_separate_noalloc_async(ptrs, len(dev_cols), n, arr, nt, bm.data_ptr(), cnt.data_ptr(),
                                                  stream)
    if rc != 0:
        raise R.RtsError(rc, R.lib().rts_last_error(None).decode())


def test_noalloc_matches_separate_scan_on_consecutive_calls():
    n = 3_000_017  # not a multiple of 32 or 1024
    cols_np = [D.uniform(n, 1), D.zipf(n, 2, 1.3), D.uniform(n, 3, 256)]
    dev_cols = [torch.from_numpy(c.view(np.int32)).cuda() for c in cols_np]
    words = R.bitmap_words(n)
    s = torch.cuda.current_stream().cuda_stream
    queries = [
        [(0, 1 << 30, 3 << 30), (1, 0, 40), (2, 10, 200)],   # three passes through the scratch array
        [(2, 0, 127), (0, 0, 1 << 31)],                       # second call: different query, same array
    ]
    with R.Context(0) as ctx:
        ctx.attach_columns([c.data_ptr() for c in dev_cols], n)
        for terms in queries:
            want = torch.full((words,), -1, dtype=torch.int32, device="cuda")
            wcnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            ctx.scan_separate_async(terms, want.data_ptr(), wcnt.data_ptr(), s)
            got = torch.full((words,), -1, dtype=torch.int32, device="cuda")
            gcnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            noalloc_scan(dev_cols, n, terms, got, gcnt, s)
            torch.cuda.synchronize()
            assert int(gcnt.item()) == int(wcnt.item())
            assert torch.equal(got, want)


def test_noalloc_rejects_rows_beyond_its_limit():
    limit = 1 << 27
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    bm = torch.zeros(4, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(R.RtsError) as e:
        noalloc_scan([dummy], limit + 1, [(0, 1, 2)], bm, cnt, 0)
    assert e.value.code == -1
    assert "limit" in str(e.value)
