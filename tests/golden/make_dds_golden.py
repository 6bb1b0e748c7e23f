"""Generate tests/golden/dds/: DDS files written by the reference's own Python
``quicktex.dds.encode`` (its pybind11 module built from its sources by
``make -C oracle pymod``), for the seeded cases of dds_cases.py, plus the sha256
of every level the reference's ``dds.read(...).decode_all()`` returns.

    make -C oracle pymod REF=<reference root> &&
        QT_REFERENCE_ROOT=<reference root> python tests/golden/make_dds_golden.py

Only runs where the reference source tree exists. Writes nothing there: it is
imported with bytecode caching off.
"""

from __future__ import annotations

import hashlib
import json
import os
import sys

sys.dont_write_bytecode = True
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("QT_REFERENCE_ROOT", "")  # root of the reference source tree (required)


def main():
    if not REF:
        raise SystemExit("set QT_REFERENCE_ROOT to the root of the reference source tree")
    sys.path[:0] = [os.path.join(ROOT, "oracle", "_ref"), REF, HERE]
    import quicktex
    import quicktex.dds as rdds

    import dds_cases

    assert os.path.dirname(quicktex.__file__).startswith(REF), quicktex.__file__
    out = os.path.join(HERE, "dds")
    os.makedirs(out, exist_ok=True)
    manifest = {}
    for name, c in dds_cases.CASES.items():
        img = dds_cases.image(name)
        enc = dds_cases.make_encoder(quicktex, c["encoder"])
        f = rdds.encode(img, enc, c["four_cc"], c.get("mip_count"))
        path = os.path.join(out, name + ".dds")
        f.save(path)
        back = rdds.read(path)
        levels = [hashlib.sha256(im.tobytes()).hexdigest() for im in back.decode_all()]
        data = open(path, "rb").read()
        manifest[name] = {"file_sha256": hashlib.sha256(data).hexdigest(), "bytes": len(data),
                          "mips": back.mipmap_count, "decoded_level_sha256": levels}
        print(name, len(data), back.mipmap_count)
    # the reference's command line (click commands run in-process) on seeded PNG inputs
    import tempfile

    from click.testing import CliRunner
    from quicktex.__main__ import main as ref_main

    cli = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name in dds_cases.CLI_INPUTS:
            dds_cases.cli_image(name).save(os.path.join(tmp, name + ".png"))
        for src, argv, tag in dds_cases.CLI_ENCODE:
            work = os.path.join(tmp, tag)  # -o names a directory unless the file already exists
            os.makedirs(work)
            r = CliRunner().invoke(ref_main, argv + ["-o", work, os.path.join(tmp, src + ".png")], catch_exceptions=False)
            assert r.exit_code == 0, r.output
            dst = os.path.join(out, "cli_" + tag + ".dds")
            with open(os.path.join(work, src + ".dds"), "rb") as fi, open(dst, "wb") as fo:
                fo.write(fi.read())
            r = CliRunner().invoke(ref_main, ["decode", "-o", work, os.path.join(work, src + ".dds")], catch_exceptions=False)
            assert r.exit_code == 0, r.output
            png = os.path.join(work, src + ".png")
            from PIL import Image

            with Image.open(png) as im:
                px = im.convert("RGBA").tobytes()
            data = open(dst, "rb").read()
            cli[tag] = {"file_sha256": hashlib.sha256(data).hexdigest(), "decoded_png_pixels_sha256": hashlib.sha256(px).hexdigest()}
            print("cli", tag, len(data))
    with open(os.path.join(out, "manifest.json"), "w") as fh:
        json.dump({"generator": "quicktex (reference) dds.encode / dds.read(...).decode_all() and its click command "
                                "line, pybind11 module built from its sources", "cases": manifest, "cli": cli}, fh, indent=1)


if __name__ == "__main__":
    main()
