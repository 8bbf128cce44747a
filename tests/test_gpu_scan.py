"""GPU parity of the fused and separate-pass scans against the oracle.

Every case compares the CUDA result bit-exactly (bitmap words and count)
with the oracle's conjunctive scalar filter (raw_scan + AND merge of the
reference, bindex.cpp:1851-1892, 1259-1281) on the same seeded inputs.
"""
import numpy as np
import pytest

import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev_cols(cols):
    return [torch.from_numpy(c.view(np.int32)).cuda() for c in cols]


def run_scan(ctx, terms, path="fused"):
    n = ctx.nrows
    bm = torch.full((max(1, R.bitmap_words(n)),), -1, dtype=torch.int32, device="cuda")  # poison
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    fn = {"fused": ctx.scan_async, "separate": ctx.scan_separate_async, "bindex": ctx.bindex_scan_async}[path]
    fn(terms, bm.data_ptr(), cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return bm.cpu().numpy().view(np.uint32)[: R.bitmap_words(n)], int(cnt.item())


def expect(cols, terms):
    n = len(cols[0])
    if any(lo > hi for _, lo, hi in terms):
        return np.zeros(O.words(n), np.uint32), 0
    if not terms:
        return O.mask_tail(np.full(O.words(n), 0xFFFFFFFF, np.uint32), n), n
    return O.range_scan([cols[c] for c, _, _ in terms], [t[1] for t in terms], [t[2] for t in terms])


def check(ctx, cols, terms, path="fused"):
    got, cnt = run_scan(ctx, terms, path)
    want, wcnt = expect(cols, terms)
    assert cnt == wcnt, (path, terms, cnt, wcnt)
    assert np.array_equal(got, want), (path, terms)


SIZES = [1, 31, 32, 33, 1023, 1024, 1025, 4097, 100003, 1 << 20]


@pytest.mark.parametrize("n", SIZES)
def test_single_column_sizes(ctx, n):
    col = D.uniform(n, seed=n)
    ctx.load_columns([col])
    s = np.sort(col)
    for lo, hi in [(0, 0xFFFFFFFE), (1, 0xFFFFFFFF), (int(s[n // 3]), int(s[(2 * n) // 3])), (5, 4),
                   (int(s[0]), int(s[0])), (0, 0)]:
        check(ctx, [col], [(0, lo, hi)])


@pytest.mark.parametrize("ncols", [2, 3, 4, 5, 17])
def test_multi_column(ctx, ncols):
    n = 200_000 + 77
    cols = [D.uniform(n, seed=100 + c, domain=(1 << 32) if c % 2 == 0 else 256) for c in range(ncols)]
    ctx.load_columns(cols)
    rng = np.random.default_rng(ncols)
    for _ in range(4):
        terms = []
        for c in range(ncols):
            a, b = sorted(rng.integers(0, (1 << 32) if c % 2 == 0 else 256, size=2).tolist())
            if c % 2 == 0:
                a, b = a // 2, b // 2 + (1 << 31)  # keep per-column selectivity high enough to leave hits
            terms.append((c, a, b))
        check(ctx, cols, terms)
        check(ctx, cols, terms, "separate")


def test_repeated_column_terms_and_always_true(ctx):
    n = 70_001
    cols = [D.uniform(n, 1), D.uniform(n, 2, 64)]
    ctx.load_columns(cols)
    check(ctx, cols, [(0, 100, 1 << 31), (0, 1 << 30, 0xFFFFFFFF), (1, 3, 40)])
    check(ctx, cols, [(0, 0, 0xFFFFFFFF)])                 # always true -> all rows
    check(ctx, cols, [(1, 0, 0xFFFFFFFF), (0, 0, 0xFFFFFFFF)])
    check(ctx, cols, [(0, 10, 20), (0, 30, 40)])          # disjoint -> empty
    check(ctx, cols, [])                                   # no terms -> all rows


def test_duplicate_heavy_domains(ctx):
    n = 300_000
    for dom in (2, 64, 256):
        col = D.uniform(n, dom, dom)
        ctx.load_columns([col])
        for lo in range(0, dom, max(1, dom // 8)):
            check(ctx, [col], [(0, lo, lo)])
            check(ctx, [col], [(0, lo, dom - 1)])


def test_unaligned_attached_columns(ctx):
    """Borrowed device columns that are not 16-byte aligned take the scalar
    path; results must not change."""
    n = 50_000
    base = D.uniform(n + 3, 9)
    t = torch.from_numpy(base.view(np.int32)).cuda()
    ptr = t.data_ptr() + 4  # 4-byte offset: not 16-byte aligned
    col = base[1:n + 1]
    ctx.attach_columns([ptr], n)
    check(ctx, [col], [(0, 1 << 30, 3 << 30)])
    check(ctx, [col], [(0, 1 << 30, 3 << 30)], "separate")
    del t


def test_attached_torch_columns(ctx):
    n = 1 << 18
    cols = [D.uniform(n, 11), D.zipf(n, 12, 1.3)]
    dc = dev_cols(cols)
    ctx.attach_columns([d.data_ptr() for d in dc], n)
    check(ctx, cols, [(0, 0, 1 << 31), (1, 0, 5)])


def test_blocking_scan_to_host(ctx):
    n = 123_457
    cols = [D.normal(n, 5)]
    ctx.load_columns(cols)
    bm, cnt = ctx.scan([(0, 1 << 31, (1 << 31) + (1 << 27))])
    want, wcnt = O.range_scan(cols, [1 << 31], [(1 << 31) + (1 << 27)])
    assert cnt == wcnt and np.array_equal(bm, want)


def test_bitmap_ops_and_count(ctx):
    n = 10_000_019
    words = R.bitmap_words(n)
    ctx.load_columns([D.uniform(n, 1)])
    rng = np.random.default_rng(3)
    a = rng.integers(0, 1 << 32, size=words, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 1 << 32, size=words, dtype=np.uint64).astype(np.uint32)
    ta = torch.from_numpy(a.view(np.int32)).cuda()
    tb = torch.from_numpy(b.view(np.int32)).cuda()
    out = torch.empty_like(ta)
    s = torch.cuda.current_stream().cuda_stream
    for op, f in [(R.BM_AND, lambda x, y: x & y), (R.BM_OR, lambda x, y: x | y), (R.BM_COPY, lambda x, y: x),
                  (R.BM_NOT, lambda x, y: ~x), (R.BM_ANDNOT, lambda x, y: y & ~x)]:
        ctx.bitmap_op_async(op, out.data_ptr(), ta.data_ptr(), tb.data_ptr(), words, 0, s)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), f(a, b)), op
    ctx.bitmap_op_async(R.BM_FILL, out.data_ptr(), 0, 0, words, 0xDEADBEEF, s)
    torch.cuda.synchronize()
    assert (out.cpu().numpy().view(np.uint32) == 0xDEADBEEF).all()
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.bitmap_count_async(ta.data_ptr(), n, cnt.data_ptr(), s)
    torch.cuda.synchronize()
    assert int(cnt.item()) == O.popcount(a, n)


def test_each_path(ctx):
    n = 250_000
    cols = [D.uniform(n, 21), D.uniform(n, 22, 256), D.zipf(n, 23, 1.1)]
    ctx.load_columns(cols)
    qs = D.batch_queries(cols, 12, seed=5, max_cols=3)
    words = R.bitmap_words(n)
    stride = (words + 31) // 32 * 32
    out = torch.empty(len(qs) * stride, dtype=torch.int32, device="cuda")
    cnt = torch.empty(len(qs), dtype=torch.int64, device="cuda")
    ctx.scan_each_async(qs, out.data_ptr(), stride, cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    o = out.cpu().numpy().view(np.uint32)
    for i, q in enumerate(qs):
        want, wcnt = expect(cols, q)
        assert int(cnt[i].item()) == wcnt
        assert np.array_equal(o[i * stride:i * stride + words], want)


def test_reference_operator_lines(ctx):
    """scan_cmd text -> parsed queries -> GPU, against the reference
    checker restated (raw_scan_entry, bindex.cpp:1894-1957)."""
    n = 99_999
    cols = [D.uniform(n, 31), D.uniform(n, 32, 64), D.uniform(n, 33, 256)]
    ctx.load_columns(cols)
    text = ("lt 2147483648\nge 10\nbt 7 200\n"
            "le 4294967295\nlt 1\ngt 0\n"
            "gt 4294967295\neq 5\neq 100\n"
            "ge 0\nbt 40 3\nle 77\n"
            "exit\nfree notes\n")
    qs = R.parse_scan_cmd(text, 3)
    ref = O.ref_parse_scan_cmd(text, 3)
    assert len(qs) == len(ref)
    for i in range(len(qs)):
        terms, empty = qs.query(i)
        got, cnt = run_scan(ctx, terms)
        want = O.raw_scan_entry(cols, ref[i])
        assert cnt == O.popcount(want, n)
        assert np.array_equal(got, O.mask_tail(want, n))


def test_all_equal_column(ctx):
    n = 70_000
    col = np.full(n, 123456, np.uint32)
    ctx.load_columns([col])
    for lo, hi in [(123456, 123456), (0, 123455), (123457, 0xFFFFFFFF), (0, 0xFFFFFFFF), (123456, 0xFFFFFFFF)]:
        check(ctx, [col], [(0, lo, hi)])


def test_load_file_and_its_failures(ctx, tmp_path):
    n = 10_007
    cols = [D.uniform(n, 61), D.uniform(n, 62, 100)]
    f = tmp_path / "t.bin"
    D.write_columns(str(f), cols)
    ctx.load_file(str(f), 2)
    assert ctx.nrows == n
    check(ctx, cols, [(1, 10, 20), (0, 0, 1 << 31)])
    short = tmp_path / "short.bin"
    short.write_bytes(f.read_bytes()[:-4])
    with pytest.raises(R.RtsError) as e:
        ctx.load_file(str(short), 2, n)               # fewer bytes than 2 x n values
    assert e.value.code == -4
    with pytest.raises(R.RtsError) as e:
        ctx.load_file(str(tmp_path / "none.bin"), 2)
    assert e.value.code == -4
    with pytest.raises(R.RtsError):
        ctx.load_file(str(f), 0)


def test_server_result_pool_too_large_is_refused(ctx):
    n = 1 << 20
    col = D.uniform(n, 63)
    ctx.load_columns([col])
    with pytest.raises(R.RtsError) as e:            # 2^24 slots x 128 KiB bitmaps: no such device memory
        R.Server(ctx, max_active=1 << 24, segment_rows=1 << 16)
    assert e.value.code == -3
    with R.Server(ctx, max_active=4, segment_rows=1 << 16) as srv:   # the context still works
        t = srv.submit([(0, 0, 1 << 31)])
        assert srv.wait(t, 5000) == int((col <= (1 << 31)).sum())
