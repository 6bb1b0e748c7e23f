"""CPU: the selector arithmetic of the BC4/BC5 encode kernels, restated in numpy.

bc4_block_thread / bc5_block_thread (quicktex_b200/csrc/qt_kernels.cu) find each
texel's level as floor((14*(v - min) + 4 + delta) / (2*delta)) with a
multiply-high by a magic number, look the selector up in the Levels table
{1,7,6,5,4,3,2,0} (BC4Encoder.cpp:45-64) with one PTX prmt.b32 and no clamp
(levels 8 and 9 hit prmt's sign-replicate mode, which yields 0 = map[7]; CUDA's
__byte_perm masks selectors to 3 bits and has no such mode), and accumulate
the PRMT words with integer adds, subtracting the table's constant filler bytes
once at the end. Here that arithmetic is emulated bit for bit and compared with
the reference's own rule: the count of thresholds delta*(2c+1) - (4 - 14*min)
that 14*v reaches, mapped through the Levels table and packed 3 bits per texel.
BC4: every (min, max) pair and every value between them. BC5: random channel
pairs, solid channels and the low-half borrow included.
"""

import numpy as np

LEVELS = np.array([1, 7, 6, 5, 4, 3, 2, 0], np.int64)
MAP_LO = 1 | (7 << 8) | (6 << 16) | (5 << 24)
MAP_HI = 4 | (3 << 8) | (2 << 16) | (0 << 24)
MASK32 = 0xFFFFFFFF


def magic() -> np.ndarray:
    m = np.zeros(256, np.int64)
    for delta in range(1, 256):
        d = 2 * delta
        lg = (d - 1).bit_length()
        m[delta] = (((1 << (12 + lg)) // d + 1) << (20 - lg)) & MASK32
    return m


M = magic()


def umulhi(a, b):
    return ((a & MASK32) * (b & MASK32)) >> 32


def prmt(x: int, y: int, s):
    """PTX prmt.b32 (default mode: 4-bit selectors, bit 3 replicates the selected byte's sign)
    with constant x, y and selector array s."""
    src = np.array([(x >> (8 * i)) & 0xFF for i in range(4)] + [(y >> (8 * i)) & 0xFF for i in range(4)], np.int64)
    out = np.zeros_like(s)
    for i in range(4):
        n = (s >> (4 * i)) & 0xF
        b = src[n & 7]
        b = np.where(n & 8, np.where(b & 0x80, 0xFF, 0), b)
        out |= b << (8 * i)
    return out


def filler(word: int, n: int) -> int:
    return sum(word << (3 * j) for j in range(n)) & MASK32


def reference_selectors(v, mn, mx):
    """BC4Encoder::EncodeBlock's selector of each value (BC4Encoder.cpp:45-64)."""
    delta = mx - mn
    bias = 4 - 14 * mn
    count = np.zeros_like(v)
    for c in range(7):
        count += (14 * v >= delta * (2 * c + 1) - bias).astype(np.int64)
    return LEVELS[count]


def pack48(sel):
    """3 bits per texel -> (bits 0..31, bits 32..47)."""
    field = np.zeros(sel.shape[0], object)
    for i in range(16):
        field = field + (sel[:, i].astype(object) << (3 * i))
    lo = np.array([int(f) & MASK32 for f in field], np.int64)
    hi = np.array([int(f) >> 32 for f in field], np.int64)
    return lo, hi


def test_bc4_selectors_every_min_max_value():
    rows = []
    for mn in range(256):
        for mx in range(mn + 1, 256):
            vals = np.arange(mn, mx + 1)
            for start in range(0, len(vals), 14):
                v = vals[(start + np.arange(16)) % len(vals)]
                v[0], v[1] = mn, mx
                rows.append((mn, mx, v))
    mn = np.array([r[0] for r in rows], np.int64)[:, None]
    mx = np.array([r[1] for r in rows], np.int64)[:, None]
    v = np.stack([r[2] for r in rows]).astype(np.int64)
    delta = mx - mn
    k = (4 + delta - 14 * mn) & MASK32
    q = umulhi((14 * v + k) & MASK32, M[delta])
    assert q.max() <= 9
    word = prmt(MAP_LO, MAP_HI, q)
    a0 = np.zeros(len(rows), np.int64)
    a1 = np.zeros(len(rows), np.int64)
    for i in range(16):
        if i < 10:
            a0 = (a0 + (word[:, i] << (3 * i))) & MASK32
        else:
            a1 = (a1 + (word[:, i] << (3 * (i - 10)))) & MASK32
    a0 = (a0 - filler(0x01010100, 10)) & MASK32
    a1 = (a1 - filler(0x01010100, 6)) & MASK32
    lo, hi = (a0 | (a1 << 30)) & MASK32, a1 >> 2
    rlo, rhi = pack48(reference_selectors(v, mn, mx))
    assert np.array_equal(lo, rlo) and np.array_equal(hi, rhi)


def test_bc5_paired_selectors():
    rng = np.random.default_rng(5)
    n = 40000
    ends = rng.integers(0, 256, (n, 2, 2))
    mn, mx = ends.min(2), ends.max(2)
    mx[::7, 0] = mn[::7, 0]   # solid first channel
    mx[::11, 1] = mn[::11, 1]  # solid second channel
    v = [rng.integers(mn[:, c, None], mx[:, c, None] + 1, (n, 16)) for c in range(2)]
    for c in range(2):
        v[c][:, 2 * c], v[c][:, 2 * c + 1] = mn[:, c], mx[:, c]
    d0, d1 = mx[:, 0] - mn[:, 0], mx[:, 1] - mn[:, 1]
    k0, k1 = 4 + d0 - 14 * mn[:, 0], 4 + d1 - 14 * mn[:, 1]
    kp = ((k0 & 0xFFFF) + (((k1 - (k0 < 0)) & MASK32) << 16)) & MASK32
    g = np.zeros((n, 4), np.int64)
    for i in range(16):
        num = (14 * (v[0][:, i] | (v[1][:, i] << 16)) + kp) & MASK32
        q0, q1 = umulhi(num & 0xFFFF, M[d0]), umulhi(num >> 16, M[d1])
        assert q0.max() <= 9 and q1.max() <= 9
        word = prmt(MAP_LO, MAP_HI, q0 + (q1 << 8))
        g[:, i // 5] = (g[:, i // 5] + (word << (3 * (i % 5)))) & MASK32
    for j, cnt in enumerate((5, 5, 5, 1)):
        g[:, j] = (g[:, j] - filler(0x01000100, cnt)) & MASK32
    for c, d in ((0, d0), (1, d1)):
        f = (g & 0xFFFF) if c == 0 else (g >> 16)
        lo = (f[:, 0] | (f[:, 1] << 15) | (f[:, 2] << 30)) & MASK32
        hi = (f[:, 2] >> 2) | (f[:, 3] << 13)
        live = d > 0  # solid channels are written as BC4Block(min) instead
        rlo, rhi = pack48(reference_selectors(v[c][live], mn[live, c, None], mx[live, c, None]))
        assert np.array_equal(lo[live], rlo) and np.array_equal(hi[live], rhi)
