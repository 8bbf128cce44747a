"""BinDex file header, checked on the CPU against a Python restatement of
the format (rts_bindex_file_info reads only the header)."""
import struct

import pytest

import rtscan_b200 as R

M64 = (1 << 64) - 1


def mix(i, w):
    z = (w + (i + 1) * 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def checksum(b: bytes) -> int:
    words = struct.unpack(f"<{len(b) // 4}I", b)
    return sum(mix(i, w) for i, w in enumerate(words)) & M64


def header(K=128, n=1_000_000, fv_stride=None, nsample=None, payload=None, magic=b"RTSBDX1\0", version=1):
    fv_stride = fv_stride if fv_stride is not None else ((n + 31) // 32 + 3) // 4 * 4
    nsample = nsample if nsample is not None else (n + 1023) // 1024
    if payload is None:
        payload = K * 12 + nsample * 4 + n * 8 + (K - 1) * fv_stride * 4
    body = magic + struct.pack("<IIQQQIIQ6Q", version, K, n, fv_stride, nsample, 7, 9, payload, *range(6))
    return body + struct.pack("<Q", checksum(body))


def test_header_is_112_bytes():
    assert len(header()) == 112


def test_file_info_reads_the_header(tmp_path):
    p = tmp_path / "a.bdx"
    p.write_bytes(header(K=64, n=123_457))
    assert R.bindex_file_info(str(p)) == (64, 123_457)


@pytest.mark.parametrize("bad", ["magic", "version", "flip", "payload", "stride", "k"])
def test_file_info_rejects_bad_headers(tmp_path, bad):
    h = {
        "magic": lambda: header(magic=b"RTSBDX2\0"),
        "version": lambda: header(version=2),
        "flip": lambda: header()[:20] + bytes([header()[20] ^ 1]) + header()[21:],
        "payload": lambda: header(payload=12345),
        "stride": lambda: header(fv_stride=10),
        "k": lambda: header(K=1),
    }[bad]()
    p = tmp_path / "b.bdx"
    p.write_bytes(h)
    with pytest.raises(R.RtsError) as e:
        R.bindex_file_info(str(p))
    assert e.value.code == -5  # RTS_ERR_PARSE


def test_file_info_missing_and_truncated(tmp_path):
    with pytest.raises(R.RtsError) as e:
        R.bindex_file_info(str(tmp_path / "none.bdx"))
    assert e.value.code == -4  # RTS_ERR_IO
    p = tmp_path / "t.bdx"
    p.write_bytes(header()[:50])
    with pytest.raises(R.RtsError) as e:
        R.bindex_file_info(str(p))
    assert e.value.code == -5


def test_every_single_bit_flip_is_refused(tmp_path):
    """The header checksum covers every byte: flipping any one bit of a valid
    header (fields, magic or the checksum itself) is a parse error."""
    good = header(K=64, n=77_777)
    p = tmp_path / "f.bdx"
    for i in range(len(good)):
        for bit in (0, 3, 7):
            p.write_bytes(good[:i] + bytes([good[i] ^ (1 << bit)]) + good[i + 1:])
            with pytest.raises(R.RtsError) as e:
                R.bindex_file_info(str(p))
            assert e.value.code == -5, (i, bit)


hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402


@settings(max_examples=200, deadline=None)
@given(data=st.one_of(
    st.binary(max_size=300),
    # well-formed headers (valid checksum) with arbitrary field values
    st.builds(lambda K, n, s, ns, pl: header(K=K, n=n, fv_stride=s, nsample=ns, payload=pl),
              st.integers(0, 1 << 20), st.integers(0, 1 << 40), st.integers(0, 1 << 40),
              st.integers(0, 1 << 32), st.integers(0, (1 << 64) - 1))))
def test_any_header_is_read_or_refused(tmp_path_factory, data):
    p = tmp_path_factory.mktemp("fz") / "x.bdx"
    p.write_bytes(data)
    try:
        K, n = R.bindex_file_info(str(p))
    except R.RtsError as e:
        assert e.code in (-4, -5), (e.code, data[:32])
        return
    # accepted: the fields it reports are the header's
    k2, n2 = struct.unpack("<IQ", data[12:16] + data[16:24])
    assert (K, n) == (k2, n2)
