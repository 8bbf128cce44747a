"""Bit layout of the pass kernel's wide lanes, on the CPU.

batch4_kernel (rtscan_b200/csrc/batch4.cuh) runs step 2 of its 16-warp
passes over up to four columns with wide lanes: lane (16-row tile k, group
pair gp) ANDs the table words of 16 rows for groups 2gp and 2gp + 1,
transposes each 16 x 32 mask as two 16 x 16 blocks in the 16-bit halves of
16 registers (transpose16x2) and writes 16-bit halves of the stage words,
which step 3 reads as 32-bit words of (query, 32-row tile) at
q * kTiles + (T ^ swizzle(q / 32)).  This test restates that index and bit
arithmetic with numpy, for every shape (GV = 16, 8, 4 groups), on random
masks, and checks every stage word against the words computed directly
(bit 31 - r of query q's word for tile T = the mask bit of row 32T + r),
including blocks whose last rows lie past the table (zeroed).
"""
import numpy as np
import pytest

W = 16  # warps per CTA of the wide shapes


def swap_bits(x, i, j, s, m):
    """Delta swap of x[..., i] bits under m << s with x[..., j] bits under m."""
    a, b = x[:, i], x[:, j]
    t = ((a >> s) ^ b) & m
    x[:, j] = b ^ t
    x[:, i] = (a ^ (t << s)) & 0xFFFFFFFF


def byte_perm_pairs(a, b):
    """__byte_perm(a, b, 0x6240) and __byte_perm(a, b, 0x7351)."""
    byte = lambda v, k: (v >> (8 * k)) & 0xFF
    lo = byte(a, 0) | byte(b, 0) << 8 | byte(a, 2) << 16 | byte(b, 2) << 24
    hi = byte(a, 1) | byte(b, 1) << 8 | byte(a, 3) << 16 | byte(b, 3) << 24
    return lo, hi


def transpose16x2(x):
    """The kernel's transpose16x2 on every row of x (lanes x 16 words)."""
    for i in range(0, 16, 2):
        swap_bits(x, i, i + 1, 1, 0x55555555)
    for base in range(0, 16, 4):
        for i in range(base, base + 2):
            swap_bits(x, i, i + 2, 2, 0x33333333)
    for base in range(0, 16, 8):
        for i in range(base, base + 4):
            swap_bits(x, i, i + 4, 4, 0x0F0F0F0F)
    for i in range(8):
        x[:, i], x[:, i + 8] = byte_perm_pairs(x[:, i].copy(), x[:, i + 8].copy())


def wide_stage(masks, gv, nvalid):
    """Stage words written by the wide lanes of one block: masks[row, group]
    are the ANDed table words of the block's rows."""
    tpw = 32 // gv
    tiles = W * tpw
    swz = lambda g: (tpw * g) & (tiles - 1)
    lane = np.arange(W * 32)
    warp, ln = lane // 32, lane % 32
    k, gp = ln // (gv // 2), ln % (gv // 2)
    T, hh = tpw * warp + k % tpw, k // tpw
    row0 = 32 * T + 16 * hh
    st16 = np.zeros(32 * gv * tiles * 2, dtype=np.uint64)
    valid = np.clip(nvalid - row0, 0, 16)
    v16 = np.where(valid >= 16, 0xFFFF, (0xFFFF << (16 - valid)) & 0xFFFF).astype(np.uint64)
    for e in (0, 1):
        x = np.zeros((lane.size, 16), dtype=np.uint64)
        for r in range(16):
            x[:, 15 - r] = masks[row0 + r, 2 * gp + e]
        transpose16x2(x)
        x &= (v16 | v16 << 16)[:, None]
        gq = 2 * gp + e
        col = T ^ swz(gq)
        half = np.where(hh == 1, 0, 1)
        for i in range(16):
            st16[((32 * gq + i) * tiles + col) * 2 + half] = x[:, i] & 0xFFFF
            st16[((32 * gq + 16 + i) * tiles + col) * 2 + half] = x[:, i] >> 16
    return st16, tiles, swz


@pytest.mark.parametrize("gv", [16, 8, 4])
def test_wide_lanes_write_every_stage_word(gv):
    rng = np.random.default_rng(gv)
    rows = W * (32 // gv) * 32
    for nvalid in (rows, rows - 24, 17):
        masks = rng.integers(0, 2**32, size=(rows, gv), dtype=np.uint64)
        st16, tiles, swz = wide_stage(masks, gv, nvalid)
        q = np.arange(32 * gv)
        g, j = q // 32, q % 32
        for T in range(tiles):
            phys = q * tiles + (T ^ swz(g))
            got = st16[2 * phys] | st16[2 * phys + 1] << 16
            want = np.zeros(q.size, dtype=np.uint64)
            for r in range(32):
                if 32 * T + r < nvalid:
                    want |= ((masks[32 * T + r, g] >> j.astype(np.uint64)) & 1) << np.uint64(31 - r)
            assert np.array_equal(got, want), (gv, nvalid, T)
