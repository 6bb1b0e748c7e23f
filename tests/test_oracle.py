"""Pinning the oracle (CPU only).

The oracle (oracle/qt_oracle.c) is trusted as the GPU checker only because
  * it reproduces the reference's own known-answer vectors (tests/golden/kat.json,
    taken from the reference's tests/images and tests/test_bc{1,4}.py), and
  * it reproduces the reference's output hashes (tests/golden/ref_hashes.json,
    generated by running the unmodified reference), and
  * where the compiled reference is present, it agrees with it live.
"""

import hashlib
import json
import os

import numpy as np
import pytest

import workloads as syn
from oracle import BC1Params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KAT = json.load(open(os.path.join(GOLDEN, "kat.json")))
HASHES_PATH = os.path.join(GOLDEN, "ref_hashes.json")
MODES = {"four": 0x04, "three": 0x03, "three_black": 0x13}
INTERPS = {"ideal": 0, "round": 1, "nvidia": 2, "amd": 3}


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def kat_rgba(entry):
    return np.frombuffer(bytes.fromhex(entry["rgba"]), np.uint8), entry["w"], entry["h"]


@pytest.mark.parametrize("mode", [0x04, 0x03, 0x13])
def test_bc1_kat_encode(oracle_lib, mode):
    """tests/test_bc1.py:134-185 of the reference, at the default level 5 / Ideal."""
    def enc(name):
        rgba, w, h = kat_rgba(KAT["bc1"][name])
        return oracle_lib.bc1_encode(rgba, w, h, BC1Params(level=5, color_mode=mode))

    grey = enc("greyscale")
    assert grey.hex() == KAT["bc1"]["greyscale"]["block"]
    three = enc("three_color")
    c0, c1 = int.from_bytes(three[0:2], "little"), int.from_bytes(three[2:4], "little")
    if mode != 0x04:
        assert three.hex() == KAT["bc1"]["three_color"]["block"]
    else:
        assert c0 > c1
    tb = enc("three_color_black")
    c0, c1 = int.from_bytes(tb[0:2], "little"), int.from_bytes(tb[2:4], "little")
    sels = [(tb[4 + i // 4] >> (2 * (i % 4))) & 3 for i in range(16)]
    if mode == 0x13:
        assert tb.hex() == KAT["bc1"]["three_color_black"]["block"]
    elif mode == 0x03:
        assert not (3 in sels and c0 <= c1)
    else:
        assert c0 > c1


@pytest.mark.parametrize("name", ["greyscale", "three_color", "three_color_black"])
def test_bc1_kat_decode(oracle_lib, name):
    """tests/test_bc1.py:188-206: decoding the expected block gives the fixture image exactly (RGB)."""
    e = KAT["bc1"][name]
    rgba, w, h = kat_rgba(e)
    out = np.frombuffer(oracle_lib.bc1_decode(bytes.fromhex(e["block"]), 4, 4), np.uint8).reshape(16, 4)
    assert (out[:, :3] == rgba.reshape(16, 4)[:, :3]).all()


def test_bc4_kat(oracle_lib):
    """tests/test_bc4.py:145-179: BC4Encoder(0) on 8value.png; BC4Decoder(0) of both blocks."""
    e8 = KAT["bc4"]["eight_value"]
    rgba, w, h = kat_rgba(e8)
    assert oracle_lib.bc4_encode(rgba, w, h, 0).hex() == e8["block"]
    for name in ("eight_value", "six_value"):
        e = KAT["bc4"][name]
        rgba, _, _ = kat_rgba(e)
        out = np.frombuffer(oracle_lib.bc4_decode(bytes.fromhex(e["block"]), 4, 4, 0), np.uint8).reshape(16, 4)
        assert (out[:, 0] == rgba.reshape(16, 4)[:, 0]).all()
        assert (out[:, 1:3] == 0).all() and (out[:, 3] == 255).all()


@pytest.mark.skipif(not os.path.exists(HASHES_PATH), reason="ref_hashes.json not generated")
def test_oracle_matches_reference_hashes_512(oracle_lib):
    """A slice of the 512x512 sweep of every level (full sweep: tests/golden/make_golden.py)."""
    hashes = json.load(open(HASHES_PATH))
    g = hashes["gradient_512"]
    img = syn.gradient_noise(512, 512)
    assert sha(img) == g["input"]["sha256"]
    enc = oracle_lib.bc1_encode(img, 512, 512, BC1Params(level=5))
    assert sha(enc) == g["bc1_L5_four_ideal"]
    assert sha(oracle_lib.bc1_decode(enc, 512, 512)) == g["bc1_decode_ideal"]
    sweep = hashes["mix_512_sweep"]
    img = syn.block_mix(512, 512, workload=2, stream=1)
    assert sha(img) == sweep["input"]["sha256"]
    for key, h in sweep["bc1"].items():
        L, mode, interp = key.split("_", 2)[0], key.split("_")[1], key.rsplit("_", 1)[1]
        mode = key[len(L) + 1:-(len(interp) + 1)]
        level = int(L[1:])
        if level in (0, 2, 6, 9, 13, 17) or (level == 18 and interp == "ideal"):
            got = oracle_lib.bc1_encode(img, 512, 512, BC1Params(level=level, color_mode=MODES[mode], interpolator=INTERPS[interp]))
            assert sha(got) == h, key


def test_oracle_matches_reference_hashes_hazards(oracle_lib):
    """A slice of the adversarial hazard corpus (all settings: tests/golden/make_golden.py)."""
    entry = json.load(open(HASHES_PATH))["hazard_mix"]
    img = syn.hazard_mix()
    assert sha(img) == entry["input"]["sha256"]
    assert syn.hazard_counts(img) == entry["input"]["counts"]
    h, w = img.shape[:2]
    for key, digest in entry["bc1"].items():
        level, interp = int(key.split("_")[0][1:]), key.rsplit("_", 1)[1]
        mode = key[len(key.split("_")[0]) + 1:-(len(interp) + 1)]
        if level in (0, 2, 5, 9, 13) or (level == 18 and interp in ("ideal", "nvidia")):
            got = oracle_lib.bc1_encode(img, w, h, BC1Params(level=level, color_mode=MODES[mode], interpolator=INTERPS[interp]))
            assert sha(got) == digest, key
    for key in ("L0_ideal", "L5_amd", "L10_round", "L18_nvidia"):
        level, interp = int(key.split("_")[0][1:]), key.split("_")[1]
        got = oracle_lib.bc3_encode(img, w, h, BC1Params(level=level, interpolator=INTERPS[interp]))
        assert sha(got) == entry["bc3"][key], key


def test_oracle_matches_reference_live(oracle_lib, reference_lib):
    """Live comparison with the compiled reference on fresh seeded inputs (every level,
    mode and interpolator; LeastSquares x Nvidia excluded: the reference reads
    uninitialised memory there, BC1Encoder.cpp:510, and its output varies with the
    OpenMP thread count)."""
    img = syn.alpha_mix(44, 36, workload=9, stream=2)
    for level in range(20):
        for mode in (0x04, 0x03, 0x13):
            for interp in range(4):
                p = BC1Params(level=level, color_mode=mode, interpolator=interp)
                if interp == 2 and reference_lib.level_params(level, mode)[1] == 0:
                    continue
                assert oracle_lib.bc1_encode(img, 44, 36, p) == reference_lib.bc1_encode(img, 44, 36, p), (level, mode, interp)
    assert oracle_lib.bc3_encode(img, 44, 36, BC1Params(level=18)) == reference_lib.bc3_encode(img, 44, 36, BC1Params(level=18))
    for c in range(4):
        assert oracle_lib.bc4_encode(img, 44, 36, c) == reference_lib.bc4_encode(img, 44, 36, c)
    rng = np.random.default_rng(3)
    for w, h in ((44, 36), (5, 3), (1, 1), (17, 9)):
        nb = ((w + 3) // 4) * ((h + 3) // 4)
        b8, b16 = rng.integers(0, 256, nb * 8, dtype=np.uint8), rng.integers(0, 256, nb * 16, dtype=np.uint8)
        for it in range(4):
            assert oracle_lib.bc1_decode(b8, w, h, it, True) == reference_lib.bc1_decode(b8, w, h, it, True)
            assert oracle_lib.bc3_decode(b16, w, h, it) == reference_lib.bc3_decode(b16, w, h, it)
        assert oracle_lib.bc5_decode(b16, w, h, 1, 3) == reference_lib.bc5_decode(b16, w, h, 1, 3)


def test_oracle_rejects_like_reference(oracle_lib):
    with pytest.raises(RuntimeError, match="Level out of range"):
        oracle_lib.bc1_encode(np.zeros(64, np.uint8), 4, 4, BC1Params(level=20))
    with pytest.raises(RuntimeError, match="Channel out of range"):
        oracle_lib.bc4_encode(np.zeros(64, np.uint8), 4, 4, 5)
