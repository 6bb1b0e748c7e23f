"""GPU parity at full workload sizes against the reference's own outputs.

tests/golden/ref_hashes.json holds sha256 digests of the unmodified
reference encoder/decoder run on the seeded workloads (generated by
tests/golden/make_golden.py); here the CUDA path, called through the C-ABI,
must reproduce every digest: 512^2 BC1 L5 encode + decode, the 4096^2 BC1
sweep of levels {0,10,18} x 3 colour modes x 4 interpolators, 8192^2 BC3 L5,
BC4 channels {0,1,3} and BC5, and their decodes. The known-answer vectors of
the reference's tests run through the drop-in Python API.
"""

import hashlib
import json
import os

import numpy as np
import pytest

import quicktex_b200 as qt
import workloads as syn
from quicktex_b200 import capi

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
HASHES = json.load(open(os.path.join(GOLDEN, "ref_hashes.json")))
KAT = json.load(open(os.path.join(GOLDEN, "kat.json")))
MODES = {"four": 0x04, "three": 0x03, "three_black": 0x13}
INTERPS = {"ideal": 0, "round": 1, "nvidia": 2, "amd": 3}


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def parse(key):
    level, rest = key.split("_", 1)
    interp = rest.rsplit("_", 1)[1]
    mode = rest[: -(len(interp) + 1)]
    return int(level[1:]), MODES[mode], INTERPS[interp]


def test_gradient_512():
    g = HASHES["gradient_512"]
    img = syn.gradient_noise(512, 512)
    assert sha(img) == g["input"]["sha256"], "input generator drifted"
    enc = capi.bc1_encode(img, 512, 512, capi.params_for_level(5))
    assert sha(enc) == g["bc1_L5_four_ideal"]
    assert sha(capi.bc1_decode(enc, 512, 512)) == g["bc1_decode_ideal"]


def test_sweep_512_all_levels():
    s = HASHES["mix_512_sweep"]
    img = syn.block_mix(512, 512, workload=2, stream=1)
    assert sha(img) == s["input"]["sha256"]
    bad = [k for k, h in s["bc1"].items() if sha(capi.bc1_encode(img, 512, 512, capi.params_for_level(*parse(k)))) != h]
    assert not bad, bad


@pytest.mark.skipif("mix_4096" not in HASHES, reason="full-size hashes not generated")
def test_mix_4096_36_settings():
    s = HASHES["mix_4096"]
    img = syn.block_mix(4096, 4096)
    assert sha(img) == s["input"]["sha256"]
    bad = [k for k, h in s["bc1"].items() if sha(capi.bc1_encode(img, 4096, 4096, capi.params_for_level(*parse(k)))) != h]
    assert not bad, bad


@pytest.mark.skipif("alpha_8192" not in HASHES, reason="full-size hashes not generated")
def test_alpha_8192_bc3_bc4():
    s = HASHES["alpha_8192"]
    img = syn.alpha_mix(8192, 8192)
    assert sha(img) == s["input"]["sha256"]
    e3 = capi.bc3_encode(img, 8192, 8192, capi.params_for_level(5))
    assert sha(e3) == s["bc3_L5_ideal"]
    assert sha(capi.bc3_decode(e3, 8192, 8192)) == s["bc3_decode_ideal"]
    for c in (0, 1, 3):
        e4 = capi.bc4_encode(img, 8192, 8192, c)
        assert sha(e4) == s[f"bc4_ch{c}"]
        assert sha(capi.bc4_decode(e4, 8192, 8192, c)) == s[f"bc4_decode_ch{c}"]


@pytest.mark.skipif("normal_8192" not in HASHES, reason="full-size hashes not generated")
def test_normal_8192_bc5():
    s = HASHES["normal_8192"]
    img = syn.normal_map(8192, 8192)
    assert sha(img) == s["input"]["sha256"]
    e5 = capi.bc5_encode(img, 8192, 8192, 0, 1)
    assert sha(e5) == s["bc5_01"]
    assert sha(capi.bc5_decode(e5, 8192, 8192, 0, 1)) == s["bc5_decode_01"]


# ---- the reference's known-answer tests, through the drop-in API ----------------
from quicktex_b200.s3tc.bc1 import BC1Block, BC1Decoder, BC1Encoder, BC1Texture  # noqa: E402
from quicktex_b200.s3tc.bc4 import BC4Block, BC4Decoder, BC4Encoder, BC4Texture  # noqa: E402


def kat_tex(entry):
    return qt.RawTexture.frombytes(bytes.fromhex(entry["rgba"]), entry["w"], entry["h"])


@pytest.mark.parametrize("mode", ["FourColor", "ThreeColor", "ThreeColorBlack"])
def test_bc1_encoder_kat(mode):
    """tests/test_bc1.py:134-185 of the reference."""
    cm = getattr(BC1Encoder.ColorMode, mode)
    enc = BC1Encoder(color_mode=cm)
    grey = enc.encode(kat_tex(KAT["bc1"]["greyscale"]))
    assert grey.size_blocks == (1, 1)
    assert not grey[0, 0].is_3color and grey[0, 0] == BC1Block.frombytes(bytes.fromhex(KAT["bc1"]["greyscale"]["block"]))
    three = enc.encode(kat_tex(KAT["bc1"]["three_color"]))[0, 0]
    if mode != "FourColor":
        assert three.is_3color and three == BC1Block.frombytes(bytes.fromhex(KAT["bc1"]["three_color"]["block"]))
    else:
        assert not three.is_3color
    tb = enc.encode(kat_tex(KAT["bc1"]["three_color_black"]))[0, 0]
    has_black = 3 in [j for row in tb.selectors for j in row]
    if mode == "ThreeColorBlack":
        assert tb.is_3color and has_black and tb == BC1Block.frombytes(bytes.fromhex(KAT["bc1"]["three_color_black"]["block"]))
    elif mode == "ThreeColor":
        assert not (has_black and tb.is_3color)
    else:
        assert not tb.is_3color


@pytest.mark.parametrize("name", ["greyscale", "three_color", "three_color_black"])
def test_bc1_decoder_kat(name):
    """tests/test_bc1.py:188-206: exact match of the decoded block with the fixture image."""
    from PIL import Image, ImageChops

    e = KAT["bc1"][name]
    tex = BC1Texture(4, 4)
    tex[0, 0] = BC1Block.frombytes(bytes.fromhex(e["block"]))
    out = BC1Decoder().decode(tex)
    assert out.size == (4, 4)
    img = Image.frombytes("RGBA", (4, 4), bytes.fromhex(e["rgba"]))
    diff = ImageChops.difference(Image.frombytes("RGBA", (4, 4), out.tobytes()), img).convert("L")
    assert diff.histogram()[0] == 16


def test_bc4_kat():
    """tests/test_bc4.py:145-179."""
    from PIL import Image, ImageChops

    e8 = KAT["bc4"]["eight_value"]
    out = BC4Encoder(0).encode(kat_tex(e8))
    assert out.size_blocks == (1, 1) and not out[0, 0].is_6value
    assert out[0, 0] == BC4Block.frombytes(bytes.fromhex(e8["block"]))
    for name in ("eight_value", "six_value"):
        e = KAT["bc4"][name]
        tex = BC4Texture(4, 4)
        tex[0, 0] = BC4Block.frombytes(bytes.fromhex(e["block"]))
        dec = BC4Decoder(0).decode(tex)
        img = Image.frombytes("RGBA", (4, 4), bytes.fromhex(e["rgba"]))
        diff = ImageChops.difference(Image.frombytes("RGBA", (4, 4), dec.tobytes()), img).convert("L")
        assert diff.histogram()[0] == 16


def test_drop_in_api_matches_capi():
    img = syn.alpha_mix(100, 60, workload=9, stream=4)
    tex = qt.RawTexture.frombytes(img.tobytes(), 100, 60)
    from quicktex_b200.s3tc.bc3 import BC3Decoder, BC3Encoder
    from quicktex_b200.s3tc.bc5 import BC5Decoder, BC5Encoder
    from quicktex_b200.s3tc.interpolator import InterpolatorAMD

    e = BC3Encoder(13, InterpolatorAMD())
    b3 = e.encode(tex)
    assert b3.tobytes() == capi.bc3_encode(img, 100, 60, capi.params_for_level(13, 4, 3))
    assert BC3Decoder(InterpolatorAMD()).decode(b3).tobytes() == capi.bc3_decode(b3.tobytes(), 100, 60, 3)
    b5 = BC5Encoder(3, 1).encode(tex)
    assert b5.tobytes() == capi.bc5_encode(img, 100, 60, 3, 1)
    assert BC5Decoder(3, 1).decode(b5).tobytes() == capi.bc5_decode(b5.tobytes(), 100, 60, 3, 1)
    enc = BC1Encoder(7, BC1Encoder.ColorMode.ThreeColorBlack)
    enc.search_rounds = 40
    enc.orderings = (60, 20)
    assert enc.encode(tex).tobytes() == capi.bc1_encode(img, 100, 60, capi.params_for_level(7, 0x13, 0, search_rounds=40, orderings4=60, orderings3=20))
