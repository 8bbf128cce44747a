"""GPU BinDex: index contents against the oracle's restated BinDex, and
query results (sieve mode and candidate mode) against the scalar filter."""
import struct

import numpy as np
import pytest

import rtscan_b200 as R
from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

KINDS = ["uniform", "uniform2p6", "uniform2p8", "zipf1.1", "zipf1.5", "normal"]


def bindex_scan(ctx, terms):
    n = ctx.nrows
    bm = torch.full((R.bitmap_words(n),), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    ctx.bindex_scan_async(terms, bm.data_ptr(), cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return bm.cpu().numpy().view(np.uint32), int(cnt.item())


def expect(cols, terms):
    n = len(cols[0])
    if any(lo > hi for _, lo, hi in terms):
        return np.zeros(O.words(n), np.uint32), 0
    if not terms:
        return O.mask_tail(np.full(O.words(n), 0xFFFFFFFF, np.uint32), n), n
    return O.range_scan([cols[c] for c, _, _ in terms], [t[1] for t in terms], [t[2] for t in terms])


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("K", [8, 128])
def test_index_matches_restated_bindex(ctx, kind, K):
    n = 300_007
    col = D.column(kind, n, 3)
    ctx.load_columns([col])
    ctx.build_bindex(0, K)
    ob = O.BinDex(col, K=K)
    starts, ranks = ctx.bindex_areas(0, K)
    assert np.array_equal(starts, ob.area_start_values())
    s = np.sort(col)
    assert np.array_equal(ranks, np.searchsorted(s, starts, side="left").astype(np.uint64))
    for k in sorted({0, 1, K // 2, K - 2}):
        assert np.array_equal(ctx.bindex_filter_vector(0, k), ob.filter_vector(k)), k


@pytest.mark.parametrize("kind", KINDS)
def test_single_column_queries(ctx, kind):
    n = (1 << 20) + 13
    col = D.column(kind, n, 11)
    ctx.load_columns([col])
    ctx.build_bindex(0, 128)
    s = np.sort(col)
    rng = np.random.default_rng(2)
    cases = [(0, 0), (0, 0xFFFFFFFE), (1, 0xFFFFFFFF), (int(s[0]), int(s[0])), (int(s[-1]), 0xFFFFFFFF),
             (int(s[n // 2]), int(s[n // 2])), (5, 4)]
    for _ in range(25):
        i, j = sorted(rng.integers(0, n, size=2).tolist())
        cases.append((int(s[i]), int(s[j])))
        cases.append((int(s[i]), int(s[i]) + int(rng.integers(0, 3))))  # tight: candidate mode
    for lo, hi in cases:
        got, cnt = bindex_scan(ctx, [(0, lo, hi)])
        want, wcnt = expect([col], [(0, lo, hi)])
        assert cnt == wcnt, (kind, lo, hi, cnt, wcnt)
        assert np.array_equal(got, want), (kind, lo, hi)


@pytest.mark.parametrize("ncols", [2, 3, 4])
def test_conjunctive_queries(ctx, ncols):
    n = 500_003
    kinds = ["uniform", "zipf1.3", "uniform2p8", "normal"][:ncols]
    cols = [D.column(k, n, 40 + i) for i, k in enumerate(kinds)]
    ctx.load_columns(cols)
    for c in range(ncols):
        ctx.build_bindex(c, 128)
    qs = D.batch_queries(cols, 40, seed=ncols, min_sel=1e-4, max_sel=0.9, min_cols=1, max_cols=ncols)
    for q in qs:
        got, cnt = bindex_scan(ctx, q)
        want, wcnt = expect(cols, q)
        assert cnt == wcnt, (q, cnt, wcnt)
        assert np.array_equal(got, want), q


def test_rows_in_two_refine_ranges(ctx):
    """Rows that lie in the refine windows of two terms (identical columns
    with equal or overlapping bounds, both bounds of a term inside one area)
    are corrected and counted once; refine sets of thousands of rows take
    the refine launch, small ones the sieve's last block."""
    n = (1 << 21) + 7
    a = D.uniform(n, 91)
    b = a.copy()
    c = (a ^ np.uint32(0x5A5A)).astype(np.uint32)
    cols = [a, b, c]
    ctx.load_columns(cols)
    for i in range(3):
        ctx.build_bindex(i, 128)
    s = np.sort(a)
    rng = np.random.default_rng(5)
    qs = []
    for _ in range(12):
        i, j = sorted(rng.integers(0, n, size=2).tolist())
        lo, hi = int(s[i]), int(s[j])
        qs.append([(0, lo, hi), (1, lo, hi)])
        k = int(rng.integers(0, n - 20000))
        qs.append([(0, int(s[k]), int(s[k + 9000])), (1, int(s[k + 3000]), int(s[k + 15000]))])
        qs.append([(0, int(s[k]), int(s[k + 500])), (1, int(s[k + 100]), int(s[k + 700])), (2, 0, 0xFFFF0000)])
    for q in qs:
        got, cnt = bindex_scan(ctx, q)
        want, wcnt = expect(cols, q)
        assert cnt == wcnt, (q, cnt, wcnt)
        assert np.array_equal(got, want), q


def test_missing_index_is_an_error(ctx):
    n = 10_000
    ctx.load_columns([D.uniform(n, 1), D.uniform(n, 2)])
    ctx.build_bindex(0, 16)
    with pytest.raises(R.RtsError) as e:
        bindex_scan(ctx, [(0, 1, 2), (1, 3, 4)])
    assert e.value.code == -6
    with pytest.raises(R.RtsError):
        ctx.build_bindex(1, 1)


def test_blocking_scan_uses_index(ctx):
    n = 200_000
    cols = [D.uniform(n, 5), D.zipf(n, 6, 1.1)]
    ctx.load_columns(cols)
    ctx.build_bindex(0, 64)
    ctx.build_bindex(1, 64)
    q = [(0, 1 << 30, 1 << 31), (1, 0, 3)]
    bm, cnt = ctx.scan(q)
    want, wcnt = expect(cols, q)
    assert cnt == wcnt and np.array_equal(bm, want)


@pytest.mark.parametrize("K", [4, 128])
def test_saved_index_loads_and_answers_the_same(ctx, tmp_path, K):
    n = 700_001
    cols = [D.zipf(n, 31, 1.3), D.uniform(n, 32), D.normal(n, 33)]
    ctx.load_columns(cols)
    for c in range(3):
        ctx.build_bindex(c, K)
        ctx.save_bindex(c, str(tmp_path / f"c{c}.bdx"))
    assert R.bindex_file_info(str(tmp_path / "c0.bdx")) == (K, n)
    rng = np.random.default_rng(4)
    qs = D.batch_queries(cols, 30, seed=5) + [[(0, 0, 3)], [(2, 1 << 31, 0xFFFFFFFF), (1, 7, 1 << 30)]]
    before = [bindex_scan(ctx, q) for q in qs]
    fvs = [ctx.bindex_filter_vector(0, k) for k in (0, K // 2, K - 2)]
    areas = ctx.bindex_areas(1, K)
    # a fresh table from the same columns, indexes from the files
    ctx.load_columns(cols)
    for c in range(3):
        ctx.load_bindex(c, str(tmp_path / f"c{c}.bdx"))
    for q, (bm, cnt) in zip(qs, before):
        got, gcnt = bindex_scan(ctx, q)
        want, wcnt = expect(cols, q)
        assert gcnt == cnt == wcnt and np.array_equal(got, bm) and np.array_equal(got, want), q
    for k, fv in zip((0, K // 2, K - 2), fvs):
        assert np.array_equal(ctx.bindex_filter_vector(0, k), fv)
    s2, r2 = ctx.bindex_areas(1, K)
    assert np.array_equal(s2, areas[0]) and np.array_equal(r2, areas[1])


def test_loading_rejects_other_columns_and_damage(ctx, tmp_path):
    n = 200_003
    a, b = D.uniform(n, 41), D.uniform(n, 42)
    ctx.load_columns([a, b])
    ctx.build_bindex(0, 16)
    f = tmp_path / "a.bdx"
    ctx.save_bindex(0, str(f))
    with pytest.raises(R.RtsError) as e:        # the index of column 0 against column 1
        ctx.load_bindex(1, str(f))
    assert e.value.code == -5
    raw = bytearray(f.read_bytes())
    raw[len(raw) // 2] ^= 0x10                   # one bit in the payload
    bad = tmp_path / "bad.bdx"
    bad.write_bytes(bytes(raw))
    with pytest.raises(R.RtsError) as e:
        ctx.load_bindex(0, str(bad))
    assert e.value.code == -5
    short = tmp_path / "short.bdx"
    short.write_bytes(f.read_bytes()[:-4096])
    with pytest.raises(R.RtsError) as e:
        ctx.load_bindex(0, str(short))
    assert e.value.code == -5
    ctx.load_columns([a[:-5]])                   # a table of another size
    with pytest.raises(R.RtsError):
        ctx.load_bindex(0, str(f))


C1, C2, C3 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)


def np_checksum(words):
    """The file format's checksum (order-dependent sum of a 64-bit mix of
    (index, word) over 32-bit words), restated with wrapping numpy uint64."""
    w = np.asarray(words).view(np.uint32).astype(np.uint64)
    i = np.arange(len(w), dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = w + (i + np.uint64(1)) * C1
        z = (z ^ (z >> np.uint64(30))) * C2
        z = (z ^ (z >> np.uint64(27))) * C3
        z = z ^ (z >> np.uint64(31))
    return int(np.sum(z, dtype=np.uint64))


def split_index_file(raw):
    """Header fields and the six payload arrays of a BinDex file."""
    K, n, stride, ns = struct.unpack_from("<IQQQ", raw, 12)
    lo, hi = struct.unpack_from("<II", raw, 40)
    off = 112
    arrays = []
    for dtype, count in (("<u4", K), ("<u8", K), ("<u4", ns), ("<u4", n), ("<u4", n), ("<u4", (K - 1) * stride)):
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off).copy()
        off += a.nbytes
        arrays.append(a)
    return {"K": K, "n": n, "stride": stride, "min": lo, "max": hi}, arrays


def join_index_file(raw, fields, arrays):
    """The file with the given arrays and min/max and every checksum
    recomputed, so that only the loader's consistency checks can refuse it."""
    head = bytearray(raw[:112])
    struct.pack_into("<II", head, 40, fields["min"], fields["max"])
    for k, a in enumerate(arrays):
        struct.pack_into("<Q", head, 56 + 8 * k, np_checksum(a))
    struct.pack_into("<Q", head, 104, np_checksum(np.frombuffer(bytes(head[:104]), dtype="<u4")))
    return bytes(head) + b"".join(a.tobytes() for a in arrays)


@pytest.mark.parametrize("damage", ["rank", "rank_past_n", "start", "sample", "fv_bit", "fv_padding", "min"])
def test_loading_refuses_consistent_checksums_over_wrong_tables(ctx, tmp_path, damage):
    """A file whose checksums all agree but whose area table, sample, filter
    vectors or min/max disagree with its sorted values (a faulty writer or a
    crafted file) is refused with RTS_ERR_PARSE, and the untouched file still
    loads and answers exactly."""
    n, K = 200_003, 16
    col = D.zipf(n, 51, 1.3)
    ctx.load_columns([col])
    ctx.build_bindex(0, K)
    f = tmp_path / "a.bdx"
    ctx.save_bindex(0, str(f))
    raw = f.read_bytes()
    fields, arrays = split_index_file(raw)
    assert join_index_file(raw, fields, arrays) == raw  # the restated checksums are the file's
    start, rank, sample, sval, spos, fv = arrays
    if damage == "rank":
        rank[5] += 1
    elif damage == "rank_past_n":
        rank[K - 1] = n + 1000
    elif damage == "start":
        start[7] += 1
    elif damage == "sample":
        sample[3] ^= 1
    elif damage == "fv_bit":
        fv[3 * fields["stride"] + 100] ^= 1 << 9
    elif damage == "fv_padding":
        words = (n + 31) // 32
        assert fields["stride"] > words
        fv[2 * fields["stride"] + words] = 1
    else:
        fields["min"] += 1
    bad = tmp_path / "bad.bdx"
    bad.write_bytes(join_index_file(raw, fields, arrays))
    with pytest.raises(R.RtsError) as e:
        ctx.load_bindex(0, str(bad))
    assert e.value.code == -5
    ctx.load_bindex(0, str(f))
    q = [(0, 3, 900)]
    got, cnt = bindex_scan(ctx, q)
    want, wcnt = expect([col], q)
    assert cnt == wcnt and np.array_equal(got, want)
