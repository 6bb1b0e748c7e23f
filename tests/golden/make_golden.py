"""Generate the committed golden fixtures under tests/golden/.

Run where the reference source tree exists (it builds and runs the unmodified
reference, oracle/_ref/libqtref.so), with QT_REFERENCE_ROOT naming its root:

    QT_REFERENCE_ROOT=<reference root> python tests/golden/make_golden.py [--skip-full | --ce-only]

Writes
  kat.json         the reference's own known-answer vectors: the 4x4 PNG
                   fixtures of tests/images/{bc1,bc4} as raw RGBA8 bytes, with
                   the expected blocks of tests/images/__init__.py:18-32.
  ref_hashes.json  sha256 of the reference's output on the seeded workloads at
                   full size (512^2 BC1 L5 encode+decode; 4096^2 BC1 at levels
                   {0,10,18} x 3 colour modes x 4 interpolators; 8192^2 BC3 L5,
                   BC5, BC4 channels {0,1,3} and their decodes), plus a 512^2
                   sweep of every level 0-19, and the adversarial hazard
                   corpus (workloads.hazard_mix: greyscale, all-black solid,
                   near-black, 3-colour+black, RGB-uniform with varying alpha,
                   extreme two-colour and solid blocks) for BC1 at every level
                   x colour mode x interpolator and BC3 at every level x
                   interpolator (--hazard-only adds just these to the existing
                   file). Each entry also records the
                   sha256 of its input so a mismatch in the generator is caught
                   before the codec is blamed. Every hash is cross-checked
                   against the oracle restatement (qt_oracle.c) before writing.
  ce_counts.json   candidate evaluations per block (the algorithmic work unit
                   of the BC1 issue roofline) counted by the oracle on the
                   4096^2 workload for each of its 36 settings, and the part of
                   them in second cluster-fit passes that repeat the first
                   pass's trials (work an encoder may skip with identical
                   output). --ce-only writes only this file, from the oracle
                   alone.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import workloads as syn  # noqa: E402
from oracle import BC1Params  # noqa: E402

REF_ROOT = os.environ.get("QT_REFERENCE_ROOT")  # root of the reference source tree (required)
REF_IMAGES = os.path.join(REF_ROOT or "", "tests", "images")
MODES = {"four": 0x04, "three": 0x03, "three_black": 0x13}
INTERPS = {"ideal": 0, "round": 1, "nvidia": 2, "amd": 3}


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


def kat() -> dict:
    from PIL import Image

    def rgba(path):
        im = Image.open(path).convert("RGBA")
        return {"w": im.size[0], "h": im.size[1], "rgba": im.tobytes("raw", "RGBA").hex()}

    out = {"bc1": {}, "bc4": {}}
    # tests/images/__init__.py:18-20
    for name, fname, block in [("greyscale", "greyscale_unpacked.png", "ffff494a78787878"),
                               ("three_color", "3color_unpacked.png", "e00700f829292929"),
                               ("three_color_black", "3color_black_unpacked.png", "e00700f827272727")]:
        out["bc1"][name] = dict(rgba(os.path.join(REF_IMAGES, "bc1", fname)), block=block)
    # tests/images/__init__.py:31-32: BC4Block(8, 248, ...) and BC4Block(240, 16, ...), selectors [[0,1,2,3]]*2+[[4,5,6,7]]*2
    sel = 0
    for i, s in enumerate([0, 1, 2, 3] * 2 + [4, 5, 6, 7] * 2):
        sel |= s << (3 * i)
    selhex = sel.to_bytes(6, "little").hex()
    out["bc4"]["six_value"] = dict(rgba(os.path.join(REF_IMAGES, "bc4", "6value.png")), block="08f8" + selhex)
    out["bc4"]["eight_value"] = dict(rgba(os.path.join(REF_IMAGES, "bc4", "8value.png")), block="f010" + selhex)
    # block byte strings of tests/test_bc1.py:9-12 and tests/test_bc4.py:9-11
    out["bc1_block_bytes"] = "ffff284278787878"
    out["bc4_block_bytes"] = "f010888668accffa"
    return out


def checked(name, ref_out, orc_out):
    if ref_out != orc_out:
        raise SystemExit(f"oracle disagrees with the reference on {name}")
    return sha(ref_out)


def write_ce_counts(ce: dict, rep: dict) -> None:
    with open(os.path.join(HERE, "ce_counts.json"), "w") as f:
        json.dump({"unit": "candidate evaluations per 4x4 block, 4096^2 block_mix workload", "per_block": ce,
                   "per_block_repeated": rep,
                   "repeated": "of per_block, the evaluations in second four-colour cluster-fit passes whose "
                               "input gives the first pass's start hash and texel order (or zero error): "
                               "they repeat the first pass's trials and cannot change the result"},
                  f, indent=1)


def ce_only() -> None:
    """ce_counts.json from the oracle alone (the counts need no reference run)."""
    oracle.build()
    orc = oracle.Oracle()
    orc.set_threads(os.cpu_count())
    img = syn.block_mix(4096, 4096)
    ce, rep = {}, {}
    for L in (0, 10, 18):
        for mn, m in MODES.items():
            for iname, it in INTERPS.items():
                orc.ce_reset()
                orc.bc1_encode(img, 4096, 4096, BC1Params(level=L, color_mode=m, interpolator=it))
                ce[f"L{L}_{mn}_{iname}"] = orc.ce_count() / (1024 * 1024)
                rep[f"L{L}_{mn}_{iname}"] = orc.ce_repeated_count() / (1024 * 1024)
                print(f"  4096 L{L} {mn} {iname}", flush=True)
    write_ce_counts(ce, rep)


def hazard_entry(ref, orc) -> dict:
    """Reference hashes of the adversarial hazard corpus: BC1 at every level x colour mode x
    interpolator, BC3 at every level x interpolator. The LeastSquares endpoint mode (level 1) is
    left out for every interpolator: the reference reads an uninitialised array there
    (BC1Encoder.cpp:510), and on this corpus its output differs from a zero-initialised copy of
    itself on a few blocks for each interpolator, so no implementation can be pinned to it."""
    img = syn.hazard_mix()
    h, w = img.shape[:2]
    bc1, bc3 = {}, {}
    for L in range(20):
        if oracle.Reference().level_params(L, 0x04)[1] == 0:
            continue
        for iname, it in INTERPS.items():
            p = BC1Params(level=L, interpolator=it)
            bc3[f"L{L}_{iname}"] = checked(f"hazard bc3 L{L} {iname}", ref.bc3_encode(img, w, h, p),
                                           orc.bc3_encode(img, w, h, p))
            for mn, m in MODES.items():
                p = BC1Params(level=L, color_mode=m, interpolator=it)
                bc1[f"L{L}_{mn}_{iname}"] = checked(f"hazard L{L} {mn} {iname}", ref.bc1_encode(img, w, h, p),
                                                    orc.bc1_encode(img, w, h, p))
    return {"input": {"gen": "hazard_mix", "w": w, "h": h, "sha256": sha(img), "counts": syn.hazard_counts(img)},
            "bc1": bc1, "bc3": bc3}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-full", action="store_true", help="only the 512^2 cases")
    ap.add_argument("--ce-only", action="store_true", help="only ce_counts.json, from the oracle")
    ap.add_argument("--hazard-only", action="store_true", help="only the hazard corpus, added to ref_hashes.json")
    args = ap.parse_args()
    if args.ce_only:
        ce_only()
        return

    if not REF_ROOT:
        raise SystemExit("set QT_REFERENCE_ROOT to the root of the reference source tree")
    oracle.build(ref_root=REF_ROOT)
    ref, orc = oracle.Reference(), oracle.Oracle()
    ref.set_threads(os.cpu_count())
    orc.set_threads(os.cpu_count())

    if args.hazard_only:
        path = os.path.join(HERE, "ref_hashes.json")
        hashes = json.load(open(path))
        hashes["hazard_mix"] = hazard_entry(ref, orc)
        with open(path, "w") as f:
            json.dump(hashes, f, indent=1)
        return

    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat(), f, indent=1)

    hashes: dict = {}
    t0 = time.time()

    # workload 1: 512x512 gradient + noise, BC1 L5 four-colour Ideal, encode + decode
    img = syn.gradient_noise(512, 512)
    enc = ref.bc1_encode(img, 512, 512, BC1Params(level=5))
    hashes["gradient_512"] = {
        "input": {"gen": "gradient_noise", "w": 512, "h": 512, "sha256": sha(img)},
        "bc1_L5_four_ideal": checked("g512 enc", enc, orc.bc1_encode(img, 512, 512, BC1Params(level=5))),
        "bc1_decode_ideal": checked("g512 dec", ref.bc1_decode(enc, 512, 512), orc.bc1_decode(enc, 512, 512)),
    }

    # 512^2 sweep of every level, mode and interpolator (LeastSquares x Nvidia excluded: reference UB)
    img = syn.block_mix(512, 512, workload=2, stream=1)
    sweep = {}
    for L in range(20):
        for mn, m in MODES.items():
            for iname, it in INTERPS.items():
                if it == 2 and oracle.Reference().level_params(L, m)[1] == 0:
                    continue
                p = BC1Params(level=L, color_mode=m, interpolator=it)
                sweep[f"L{L}_{mn}_{iname}"] = checked(f"sweep L{L}", ref.bc1_encode(img, 512, 512, p), orc.bc1_encode(img, 512, 512, p))
    hashes["mix_512_sweep"] = {"input": {"gen": "block_mix", "w": 512, "h": 512, "workload": 2, "stream": 1,
                                         "sha256": sha(img)}, "bc1": sweep}
    hashes["hazard_mix"] = hazard_entry(ref, orc)
    print(f"512 cases done in {time.time() - t0:.0f}s", flush=True)

    ce, rep = {}, {}
    if not args.skip_full:
        img = syn.block_mix(4096, 4096)
        runs = {}
        for L in (0, 10, 18):
            for mn, m in MODES.items():
                for iname, it in INTERPS.items():
                    p = BC1Params(level=L, color_mode=m, interpolator=it)
                    r = ref.bc1_encode(img, 4096, 4096, p)
                    orc.ce_reset()
                    o = orc.bc1_encode(img, 4096, 4096, p)
                    ce[f"L{L}_{mn}_{iname}"] = orc.ce_count() / (1024 * 1024)
                    rep[f"L{L}_{mn}_{iname}"] = orc.ce_repeated_count() / (1024 * 1024)
                    runs[f"L{L}_{mn}_{iname}"] = checked(f"4096 L{L} {mn} {iname}", r, o)
                    print(f"  4096 L{L} {mn} {iname} ({time.time() - t0:.0f}s)", flush=True)
        hashes["mix_4096"] = {"input": {"gen": "block_mix", "w": 4096, "h": 4096, "sha256": sha(img)}, "bc1": runs}

        img = syn.alpha_mix(8192, 8192)
        e3 = ref.bc3_encode(img, 8192, 8192, BC1Params(level=5))
        entry = {"input": {"gen": "alpha_mix", "w": 8192, "h": 8192, "sha256": sha(img)},
                 "bc3_L5_ideal": checked("bc3", e3, orc.bc3_encode(img, 8192, 8192, BC1Params(level=5))),
                 "bc3_decode_ideal": checked("bc3 dec", ref.bc3_decode(e3, 8192, 8192), orc.bc3_decode(e3, 8192, 8192))}
        for c in (0, 1, 3):
            e4 = ref.bc4_encode(img, 8192, 8192, c)
            entry[f"bc4_ch{c}"] = checked(f"bc4 {c}", e4, orc.bc4_encode(img, 8192, 8192, c))
            entry[f"bc4_decode_ch{c}"] = checked(f"bc4 dec {c}", ref.bc4_decode(e4, 8192, 8192, c), orc.bc4_decode(e4, 8192, 8192, c))
        hashes["alpha_8192"] = entry
        print(f"  8192 bc3/bc4 ({time.time() - t0:.0f}s)", flush=True)

        img = syn.normal_map(8192, 8192)
        e5 = ref.bc5_encode(img, 8192, 8192, 0, 1)
        hashes["normal_8192"] = {"input": {"gen": "normal_map", "w": 8192, "h": 8192, "sha256": sha(img)},
                                 "bc5_01": checked("bc5", e5, orc.bc5_encode(img, 8192, 8192, 0, 1)),
                                 "bc5_decode_01": checked("bc5 dec", ref.bc5_decode(e5, 8192, 8192, 0, 1),
                                                          orc.bc5_decode(e5, 8192, 8192, 0, 1))}
        write_ce_counts(ce, rep)

    with open(os.path.join(HERE, "ref_hashes.json"), "w") as f:
        json.dump(hashes, f, indent=1)
    print(f"done in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
