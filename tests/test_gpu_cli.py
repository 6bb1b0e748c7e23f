"""GPU: the command line (python -m quicktex_b200) writes the DDS files the
reference's command line wrote for the same inputs and options
(tests/golden/dds/cli_*.dds), decodes them to the reference's pixels, and gives
each file the same bytes when many files go through one invocation (one launch)."""

import hashlib
import json
import os
import shutil
import sys

import pytest
from click.testing import CliRunner

from quicktex_b200.cli import main

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "dds")
CLI = json.load(open(os.path.join(GOLD, "manifest.json")))["cli"]
sys.path.insert(0, os.path.join(HERE, "golden"))
import dds_cases  # noqa: E402


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli_in")
    for name in dds_cases.CLI_INPUTS:
        dds_cases.cli_image(name).save(d / (name + ".png"))
    return d


@pytest.mark.parametrize("src,argv,tag", dds_cases.CLI_ENCODE, ids=[t for _, _, t in dds_cases.CLI_ENCODE])
def test_cli_encode_and_decode_match_reference(inputs, tmp_path, src, argv, tag):
    from PIL import Image

    r = CliRunner().invoke(main, argv + ["-o", str(tmp_path), str(inputs / (src + ".png"))], catch_exceptions=False)
    assert r.exit_code == 0, r.output
    data = (tmp_path / (src + ".dds")).read_bytes()
    assert data == open(os.path.join(GOLD, "cli_" + tag + ".dds"), "rb").read()
    assert hashlib.sha256(data).hexdigest() == CLI[tag]["file_sha256"]
    r = CliRunner().invoke(main, ["decode", "-o", str(tmp_path), str(tmp_path / (src + ".dds"))], catch_exceptions=False)
    assert r.exit_code == 0, r.output
    with Image.open(tmp_path / (src + ".png")) as im:
        assert hashlib.sha256(im.convert("RGBA").tobytes()).hexdigest() == CLI[tag]["decoded_png_pixels_sha256"]


def test_many_files_one_invocation(inputs, tmp_path):
    """Six inputs (copies of the two seeded images) in one call: every output equals the single-file one."""
    files = []
    for k in range(3):
        for name in dds_cases.CLI_INPUTS:
            p = tmp_path / f"{name}_{k}.png"
            shutil.copy(inputs / (name + ".png"), p)
            files.append(p)
    out = tmp_path / "out"
    out.mkdir()
    r = CliRunner().invoke(main, ["encode", "auto", "-l", "3", "-o", str(out)] + [str(f) for f in files],
                           catch_exceptions=False)
    assert r.exit_code == 0, r.output
    gold = {"cli_rgba": "auto_alpha", "cli_rgb": None}
    for f in files:
        data = (out / (f.stem + ".dds")).read_bytes()
        name = f.stem.rsplit("_", 1)[0]
        if gold[name]:
            assert data == open(os.path.join(GOLD, "cli_" + gold[name] + ".dds"), "rb").read()
        assert data == (out / (name + "_0.dds")).read_bytes()
    r = CliRunner().invoke(main, ["decode", "-x", "png", "-o", str(out)] + [str(out / (f.stem + ".dds")) for f in files],
                           catch_exceptions=False)
    assert r.exit_code == 0, r.output
    assert len(list(out.glob("*.png"))) == len(files)
