"""GPU parity on the adversarial hazard corpus.

workloads.hazard_mix builds a 512x384 texture whose blocks aim at the
encoder branches that natural content almost never reaches:

  * FindEndpoints' greyscale branch, with max.r - min.r < 2 and >= 2
    (BC1Encoder.cpp:474-494), also inside the 3-colour+black trial, where the
    metrics ignore black texels but the branch reads pixel (0, 0);
  * WriteBlockSolid's all-black rule and its equal / swapped 565 endpoint
    rules (BC1Encoder.cpp:345-393);
  * the near-black rule (r|g|b) < 4 (Color.h:82) from both sides, and the
    3-colour+black trial it triggers (has_black && !max.IsBlack(),
    BC1Encoder.cpp:327-335);
  * blocks of one RGB colour with varying alpha, which are not solid because
    IsSingleColor compares RGBA (ColorBlock.h:80-86);
  * two-colour and solid blocks of extreme channel values.

Each branch is reached by at least 1,000 blocks (asserted below). The CUDA
path, through the C-ABI, must reproduce the unmodified reference's output
digests (tests/golden/ref_hashes.json, written by make_golden.py) for BC1 at
every level 0-19 x colour mode x interpolator and for BC3 at every level x
interpolator. The LeastSquares endpoint mode (level 1) reads an uninitialised
array in the reference (BC1Encoder.cpp:510), so those settings are compared
with the oracle, which zero-initialises it, instead.
"""

import hashlib
import json
import os

import pytest

import workloads as syn
from oracle import BC1Params
from quicktex_b200 import capi

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ENTRY = json.load(open(os.path.join(GOLDEN, "ref_hashes.json")))["hazard_mix"]
MODES = {"four": 0x04, "three": 0x03, "three_black": 0x13}
INTERPS = {"ideal": 0, "round": 1, "nvidia": 2, "amd": 3}


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


@pytest.fixture(scope="module")
def corpus():
    img = syn.hazard_mix()
    assert sha(img) == ENTRY["input"]["sha256"], "input generator drifted"
    return img


def test_every_hazard_is_reached_by_1000_blocks(corpus):
    counts = syn.hazard_counts(corpus)
    assert counts == ENTRY["input"]["counts"]
    low = {k: v for k, v in counts.items() if v < 1000}
    assert not low, low


@pytest.mark.parametrize("level", range(20))
def test_bc1_hazards_every_mode_and_interpolator(corpus, level, oracle_lib):
    h, w = corpus.shape[:2]
    bad = []
    for mn, m in MODES.items():
        for iname, it in INTERPS.items():
            key = f"L{level}_{mn}_{iname}"
            out = capi.bc1_encode(corpus, w, h, capi.params_for_level(level, m, it))
            if key in ENTRY["bc1"]:
                ok = sha(out) == ENTRY["bc1"][key]
            else:  # LeastSquares: the reference's output is undefined; the oracle is the checker
                ok = bytes(out) == oracle_lib.bc1_encode(corpus, w, h, BC1Params(level=level, color_mode=m, interpolator=it))
            if not ok:
                bad.append(key)
    assert not bad, bad


@pytest.mark.parametrize("level", range(20))
def test_bc3_hazards_every_interpolator(corpus, level, oracle_lib):
    h, w = corpus.shape[:2]
    bad = []
    for iname, it in INTERPS.items():
        key = f"L{level}_{iname}"
        out = capi.bc3_encode(corpus, w, h, capi.params_for_level(level, capi.FOUR_COLOR, it))
        if key in ENTRY["bc3"]:
            ok = sha(out) == ENTRY["bc3"][key]
        else:
            ok = bytes(out) == oracle_lib.bc3_encode(corpus, w, h, BC1Params(level=level, interpolator=it))
        if not ok:
            bad.append(key)
    assert not bad, bad
