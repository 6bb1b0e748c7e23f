"""The seeded images and encoder settings of the DDS golden files (shared by
make_dds_golden.py, which runs the reference, and the tests, which run this
package). Encoder settings are plain data so either package's classes can be
built from them."""

from __future__ import annotations

import numpy as np


def image(name: str):
    """The PIL image of a case (seeded; RGBA unless the case says RGB)."""
    import os
    import sys

    from PIL import Image

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    import workloads as syn

    c = CASES[name]
    w, h = c["size"]
    if c["content"] == "alpha_mix":
        px = syn.alpha_mix(w, h, workload=11, stream=c["seed"])
    elif c["content"] == "normal_map":
        px = syn.normal_map(w, h, workload=11, stream=c["seed"])
    else:
        px = syn.block_mix(w, h, workload=11, stream=c["seed"])
    px = np.ascontiguousarray(px[:h, :w])
    img = Image.fromarray(px, "RGBA")
    return img.convert("RGB") if c.get("mode") == "RGB" else img


# encoder: (format, args) — BC1 (level, color mode name), BC3 (level,), BC4 (channel,), BC5 (chan0, chan1)
CASES = {
    "bc1_l5_37x21": {"size": (37, 21), "content": "alpha_mix", "seed": 1, "encoder": ("BC1", (5, "FourColor")), "four_cc": "DXT1"},
    "bc1_l10_three_64x64_rgb": {"size": (64, 64), "content": "block_mix", "seed": 2, "mode": "RGB",
                                "encoder": ("BC1", (10, "ThreeColor")), "four_cc": "DXT1"},
    "bc1_l18_black_45x30": {"size": (45, 30), "content": "block_mix", "seed": 3,
                            "encoder": ("BC1", (18, "ThreeColorBlack")), "four_cc": "DXT1"},
    "bc3_l5_64x40": {"size": (64, 40), "content": "alpha_mix", "seed": 4, "encoder": ("BC3", (5,)), "four_cc": "DXT5"},
    "bc3_l9_5x130_mips3": {"size": (5, 130), "content": "alpha_mix", "seed": 5, "encoder": ("BC3", (9,)),
                           "four_cc": "DXT5", "mip_count": 3},
    "bc4_ch0_33x17": {"size": (33, 17), "content": "block_mix", "seed": 6, "encoder": ("BC4", (0,)), "four_cc": "ATI1"},
    "bc4_ch3_31x31": {"size": (31, 31), "content": "alpha_mix", "seed": 7, "encoder": ("BC4", (3,)), "four_cc": "ATI1"},
    "bc5_40x40": {"size": (40, 40), "content": "normal_map", "seed": 8, "encoder": ("BC5", (0, 1)), "four_cc": "ATI2"},
    "bc1_l1_1x1": {"size": (1, 1), "content": "block_mix", "seed": 9, "encoder": ("BC1", (1, "FourColor")), "four_cc": "DXT1"},
}


def make_encoder(pkg, enc):
    """An encoder of package ``pkg`` (a module with s3tc.bc1..bc5) for the case's settings."""
    fmt, args = enc
    if fmt == "BC1":
        E = pkg.s3tc.bc1.BC1Encoder
        return E(args[0], getattr(E.ColorMode, args[1]))
    if fmt == "BC3":
        return pkg.s3tc.bc3.BC3Encoder(*args)
    if fmt == "BC4":
        return pkg.s3tc.bc4.BC4Encoder(*args)
    return pkg.s3tc.bc5.BC5Encoder(*args)


# command-line cases: (input case name, input mode, argv after the program name, output name)
CLI_INPUTS = {
    "cli_rgba": {"size": (40, 24), "content": "alpha_mix", "seed": 21},
    "cli_rgb": {"size": (36, 20), "content": "block_mix", "seed": 22, "mode": "RGB"},
}
CLI_ENCODE = [
    ("cli_rgb", ["encode", "bc1", "-l", "5"], "bc1_l5"),
    ("cli_rgb", ["encode", "bc1", "-l", "12", "-b", "-F"], "bc1_l12_black_noflip"),
    ("cli_rgba", ["encode", "bc3", "-l", "6"], "bc3_l6"),
    ("cli_rgb", ["encode", "bc3", "-l", "4", "-n"], "bc3_l4_normal"),
    ("cli_rgba", ["encode", "bc4"], "bc4"),
    ("cli_rgb", ["encode", "bc5", "-F"], "bc5_noflip"),
    ("cli_rgba", ["encode", "auto", "-l", "3"], "auto_alpha"),
    ("cli_rgb", ["encode", "auto", "-l", "3", "-4"], "auto_opaque_4color"),
]


def cli_image(name: str):
    """The seeded PIL image of a command-line input."""
    CASES[name] = dict(CLI_INPUTS[name], encoder=None, four_cc=None)
    try:
        return image(name)
    finally:
        del CASES[name]
