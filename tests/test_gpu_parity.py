"""GPU parity: the CUDA path, called through the C-ABI, against the oracle.

Bit-exact comparison (integer/byte output) on seeded inputs at sizes the
oracle finishes in seconds: every BC1 level 0-19 x colour mode x interpolator,
BC3/BC4/BC5, all decoders, and every texture size 1..17 x 1..17 (wrap-around
padding on encode, wrapped overwrite on decode).
"""

import numpy as np
import pytest

import workloads as syn
from oracle import BC1Params
from quicktex_b200 import capi

pytestmark = pytest.mark.gpu

MODES = [capi.FOUR_COLOR, capi.THREE_COLOR, capi.THREE_COLOR_BLACK]
IMG = syn.block_mix(64, 64, workload=2, stream=7)
IMGA = syn.alpha_mix(36, 28, workload=3, stream=3)
IMGN = syn.normal_map(40, 24)


def assert_same(got: bytes, exp: bytes, bsize: int, what: str = ""):
    if got == exp:
        return
    g = np.frombuffer(got, np.uint8).reshape(-1, bsize)
    e = np.frombuffer(exp, np.uint8).reshape(-1, bsize)
    bad = np.where((g != e).any(1))[0]
    raise AssertionError(f"{what}: {len(bad)}/{len(e)} units differ; first {bad[:4].tolist()}: "
                         f"got {g[bad[0]].tobytes().hex()} expected {e[bad[0]].tobytes().hex()}")


@pytest.mark.parametrize("interp", range(4))
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("level", range(20))
def test_bc1_encode_levels(oracle_lib, level, mode, interp):
    for img in (IMG, IMGA):
        h, w = img.shape[:2]
        exp = oracle_lib.bc1_encode(img, w, h, BC1Params(level=level, color_mode=mode, interpolator=interp))
        got = capi.bc1_encode(img, w, h, capi.params_for_level(level, mode, interp))
        assert_same(got, exp, 8, f"L{level} mode {mode} interp {interp} {w}x{h}")


@pytest.mark.parametrize(
    "over",
    [
        dict(error_mode=0), dict(error_mode=1, level=18), dict(error_mode=2, level=13), dict(endpoint_mode=0, level=10),
        dict(endpoint_mode=1, level=3), dict(endpoint_mode=2, level=12), dict(exhaustive=1, level=8),
        dict(search_rounds=7, level=9), dict(power_iterations=10, level=4), dict(orderings4=3, orderings3=5, level=11),
        dict(two_cf_passes=1, level=7), dict(two_ep_passes=1, level=2, error_mode=3),
    ],
)
@pytest.mark.parametrize("mode", MODES)
def test_bc1_encode_advanced(oracle_lib, over, mode):
    over = dict(over)
    level = over.pop("level", 5)
    for interp in (0, 2):
        exp = oracle_lib.bc1_encode(IMG, 64, 64, BC1Params(level=level, color_mode=mode, interpolator=interp, **over))
        got = capi.bc1_encode(IMG, 64, 64, capi.params_for_level(level, mode, interp, **over))
        assert_same(got, exp, 8, f"L{level} {over} mode {mode} interp {interp}")


@pytest.mark.parametrize("level", [0, 5, 10, 18])
@pytest.mark.parametrize("interp", range(4))
def test_bc3_encode(oracle_lib, level, interp):
    h, w = IMGA.shape[:2]
    exp = oracle_lib.bc3_encode(IMGA, w, h, BC1Params(level=level, interpolator=interp))
    got = capi.bc3_encode(IMGA, w, h, capi.params_for_level(level, capi.FOUR_COLOR, interp))
    assert_same(got, exp, 16, f"bc3 L{level} interp {interp}")


def test_bc4_bc5_encode(oracle_lib):
    for img in (IMGA, IMGN, IMG):
        h, w = img.shape[:2]
        for c in range(4):
            assert_same(capi.bc4_encode(img, w, h, c), oracle_lib.bc4_encode(img, w, h, c), 8, f"bc4 ch{c}")
        for c0, c1 in ((0, 1), (1, 0), (3, 2), (2, 2)):
            assert_same(capi.bc5_encode(img, w, h, c0, c1), oracle_lib.bc5_encode(img, w, h, c0, c1), 16, "bc5")


@pytest.mark.parametrize("interp", range(4))
def test_decoders(oracle_lib, interp):
    rng = np.random.default_rng(interp)
    for w, h in ((64, 64), (37, 13), (5, 5), (1, 1), (2, 7)):
        nb = ((w + 3) // 4) * ((h + 3) // 4)
        b8 = rng.integers(0, 256, nb * 8, dtype=np.uint8)
        b16 = rng.integers(0, 256, nb * 16, dtype=np.uint8)
        for wa in (False, True):
            assert_same(capi.bc1_decode(b8, w, h, interp, wa), oracle_lib.bc1_decode(b8, w, h, interp, wa), 4, "bc1 dec")
        assert_same(capi.bc3_decode(b16, w, h, interp), oracle_lib.bc3_decode(b16, w, h, interp), 4, "bc3 dec")
        for c in range(4):
            assert_same(capi.bc4_decode(b8, w, h, c), oracle_lib.bc4_decode(b8, w, h, c), 4, "bc4 dec")
        assert_same(capi.bc5_decode(b16, w, h, 0, 1), oracle_lib.bc5_decode(b16, w, h, 0, 1), 4, "bc5 dec")
        assert_same(capi.bc5_decode(b16, w, h, 2, 2), oracle_lib.bc5_decode(b16, w, h, 2, 2), 4, "bc5 dec same ch")


def test_all_small_sizes(oracle_lib):
    """Every size 1..17 x 1..17: encode padding wraps, decode overwrite wraps."""
    base = syn.alpha_mix(20, 20, workload=3, stream=11)
    p_oracle = BC1Params(level=10, color_mode=capi.THREE_COLOR_BLACK, interpolator=1)
    p = capi.params_for_level(10, capi.THREE_COLOR_BLACK, 1)
    for w in range(1, 18):
        for h in range(1, 18):
            img = np.ascontiguousarray(base[:h, :w])
            enc = capi.bc1_encode(img, w, h, p)
            assert_same(enc, oracle_lib.bc1_encode(img, w, h, p_oracle), 8, f"bc1 {w}x{h}")
            assert_same(capi.bc1_decode(enc, w, h, 1), oracle_lib.bc1_decode(enc, w, h, 1), 4, f"bc1 dec {w}x{h}")
            e5 = capi.bc5_encode(img, w, h, 0, 3)
            assert_same(e5, oracle_lib.bc5_encode(img, w, h, 0, 3), 16, f"bc5 {w}x{h}")
            assert_same(capi.bc5_decode(e5, w, h, 0, 3), oracle_lib.bc5_decode(e5, w, h, 0, 3), 4, f"bc5 dec {w}x{h}")
