"""GPU paths against the golden fixtures recorded from the reference itself
(tests/golden/golden.json): the scan_cmd text goes through the product
parser, every device path must reproduce the reference scalar filter's hit
count and bitmap hash for every query: the fused, separate and BinDex scans,
the batched passes of every shape, the fused aggregate's count, and scans of
the rank-encoded table with rewritten terms."""
import hashlib
import json
import os

import numpy as np
import pytest

import rtscan_b200 as R
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")
with open(GOLDEN) as f:
    CASES = json.load(f)["cases"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def column(kind, n, seed):
    if kind == "uniform1000":
        return D.uniform(n, seed, 1000)
    return D.column(kind, n, seed)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_golden_case(ctx, case):
    n = case["n"]
    cols = [column(c["kind"], n, c["seed"]) for c in case["columns"]]
    ctx.load_columns(cols)
    for c in range(len(cols)):
        ctx.build_bindex(c, 128)
    words = R.bitmap_words(n)
    bm = torch.empty(words, dtype=torch.int32, device="cuda")
    cnt = torch.empty(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    queries = []
    for q in case["queries"]:
        qs = R.parse_scan_cmd("\n".join(q["lines"]) + "\nexit\n", len(cols))
        assert len(qs) == 1
        terms, _ = qs.query(0)
        queries.append(terms)
        for name, fn in (("fused", ctx.scan_async), ("separate", ctx.scan_separate_async),
                         ("bindex", ctx.bindex_scan_async)):
            bm.fill_(-1)
            fn(terms, bm.data_ptr(), cnt.data_ptr(), s)
            torch.cuda.synchronize()
            got = bm.cpu().numpy().view(np.uint32)
            assert int(cnt.item()) == q["raw_hits"], (name, q["lines"])
            assert sha(got) == q["raw_sha"], (name, q["lines"])
    # the whole case as one batch, and repeated past 32 and 256 queries so
    # that the table-driven pass shapes answer it too
    stride = (words + 31) // 32 * 32
    for reps in (1, 3, 20):
        batch = queries * reps
        out = torch.empty(len(batch) * stride, dtype=torch.int32, device="cuda")
        cnts = torch.empty(len(batch), dtype=torch.int64, device="cuda")
        for runner in ((ctx.scan_each_async, ctx.scan_batch_async) if reps == 1 else (ctx.scan_batch_async,)):
            out.fill_(-1)
            runner(batch, out.data_ptr(), stride, cnts.data_ptr(), s)
            torch.cuda.synchronize()
            o = out.cpu().numpy().view(np.uint32)
            for i in range(len(batch)):
                q = case["queries"][i % len(queries)]
                assert int(cnts[i].item()) == q["raw_hits"], (runner.__name__, reps, q["lines"])
                assert sha(o[i * stride:i * stride + words]) == q["raw_sha"], (runner.__name__, reps, q["lines"])
    # the fused scan-and-aggregate's count
    s2 = torch.zeros(2, dtype=torch.int64, device="cuda")
    for terms, q in zip(queries, case["queries"]):
        if len({t[0] for t in terms}) <= 8:
            ctx.scan_aggregate_async(terms, -1, -1, cnt.data_ptr(), s2.data_ptr(), s)
            torch.cuda.synchronize()
            assert int(cnt.item()) == q["raw_hits"], ("aggregate", q["lines"])
    # the rank-encoded table with rewritten terms
    ctx.encode_table()
    for terms, q in zip(queries, case["queries"]):
        bm.fill_(-1)
        ctx.scan_async(ctx.encode_terms(terms), bm.data_ptr(), cnt.data_ptr(), s)
        torch.cuda.synchronize()
        assert int(cnt.item()) == q["raw_hits"], ("encoded", q["lines"])
        assert sha(bm.cpu().numpy().view(np.uint32)) == q["raw_sha"], ("encoded", q["lines"])
