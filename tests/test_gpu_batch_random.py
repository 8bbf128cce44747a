"""Seeded random batches against the oracle.  Each trial draws a row count,
1-8 columns of mixed kinds and a query count biased to the edges of the
pass routing: one to three queries (fused scans per query when narrow), up
to 20 (term by term), 21-128, 129-256 and 257-512 (the 128-, 256- and
512-slot tables), more than 512 (several passes).  Queries over up to 8
columns, plus empty and unconstrained ones.  Odd trials run the table
passes on 8-warp CTAs (one or two per SM).  Every bitmap and count must
equal the scalar filter's."""
import numpy as np
import pytest

import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

EDGE_COUNTS = [1, 2, 3, 4, 19, 20, 21, 32, 33, 127, 128, 129, 255, 256, 257, 511, 512, 513]


def column(rng, n, kind, seed):
    if kind == 0:
        return D.uniform(n, seed)
    if kind == 1:
        return D.uniform(n, seed, int(rng.choice([2, 64, 256, 1 << 16])))
    if kind == 2:
        return D.zipf(n, seed, float(rng.choice([1.1, 1.3, 1.5])))
    return D.normal(n, seed)


def expect(cols, q, n):
    if any(lo > hi for _, lo, hi in q):
        return np.zeros(O.words(n), np.uint32), 0
    if not q:
        return O.mask_tail(np.full(O.words(n), 0xFFFFFFFF, np.uint32), n), n
    return O.range_scan([cols[c] for c, _, _ in q], [t[1] for t in q], [t[2] for t in q])


@pytest.mark.parametrize("trial", range(24))
def test_random_batch(ctx, trial):
    rng = np.random.default_rng(1000 + trial)
    n = int(rng.choice([int(rng.integers(1, 5000)), int(rng.integers(5000, 150_000))]))
    ncols = int(rng.integers(1, 9))
    cols = [column(rng, n, int(rng.integers(0, 4)), 7000 + 10 * trial + c) for c in range(ncols)]
    ctx.load_columns(cols)
    nq = int(rng.choice(EDGE_COUNTS)) if trial % 3 else int(rng.integers(1, 1100))
    max_cols = int(rng.integers(1, min(ncols, 8) + 1))
    qs = D.batch_queries(cols, nq, seed=trial, min_cols=1, max_cols=max_cols)
    if trial % 4 == 0:  # outside the kernels: no term, an empty term
        qs += [[], [(0, 9, 3)]]
    words = R.bitmap_words(n)
    stride = words + (trial % 5)
    out = torch.full((len(qs) * stride,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((len(qs),), -1, dtype=torch.int64, device="cuda")
    old = ctx.batch_config()
    if trial % 2:  # odd trials: 8-warp CTAs for the table passes
        ctx.set_batch_config(4, 8, 512, 136 * 1024 if trial % 4 == 1 else 56 * 1024)
    try:
        ctx.scan_batch_async(qs, out.data_ptr(), stride, cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
    finally:
        ctx.set_batch_config(old["variant"], old["warps_per_cta"], old["max_queries_per_pass"],
                             old["table_budget_bytes"])
    o = out.cpu().numpy().view(np.uint32)
    c = cnt.cpu().numpy()
    for i, q in enumerate(qs):
        want, wcnt = expect(cols, q, n)
        assert int(c[i]) == wcnt, (trial, n, ncols, nq, i, q)
        assert np.array_equal(o[i * stride:i * stride + words], want), (trial, n, ncols, nq, i, q)
        assert (o[i * stride + words:(i + 1) * stride] == 0xFFFFFFFF).all(), "wrote past the bitmap"
