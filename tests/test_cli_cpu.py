"""CPU: the command line's host-side rules, as the reference's
(quicktex/cli/common.py): where outputs go, which extensions decode accepts,
and the argument errors raised before any device work."""

import pathlib

import click
import pytest
from click.testing import CliRunner

from quicktex_b200.cli import common, main


def test_path_pairs(tmp_path):
    a, b = tmp_path / "a.png", tmp_path / "b.png"
    a.write_bytes(b"x")
    b.write_bytes(b"x")
    # in place, with the suffix
    assert common.path_pairs([str(a)], None, "_s", ".dds") == [(a, tmp_path / "a_s.dds")]
    # into a directory (a path that is not an existing file counts as a directory)
    out = tmp_path / "out"
    assert common.path_pairs([str(a), str(b)], str(out), "", ".dds") == [(a, out / "a.dds"), (b, out / "b.dds")]
    # into an existing file: one input only
    f = tmp_path / "x.dds"
    f.write_bytes(b"")
    assert common.path_pairs([str(a)], str(f), "_ignored", ".dds") == [(a, f)]
    with pytest.raises(click.BadOptionUsage):
        common.path_pairs([str(a), str(b)], str(f), "", ".dds")
    with pytest.raises(click.BadArgumentUsage):
        common.path_pairs([], None, "", ".dds")


def test_decoded_extension_validation():
    assert common.validate_decoded_extension(None, None, "png") == ".png"
    assert common.validate_decoded_extension(None, None, ".png") == ".png"
    with pytest.raises(click.BadParameter):
        common.validate_decoded_extension(None, None, ".notanimage")


def test_cli_help_and_argument_errors(tmp_path):
    r = CliRunner().invoke(main, ["--help"])
    assert r.exit_code == 0 and "encode" in r.output and "decode" in r.output
    for cmd in (["encode", "bc1"], ["encode", "bc3"], ["encode", "bc4"], ["encode", "bc5"], ["encode", "auto"], ["decode"]):
        r = CliRunner().invoke(main, cmd + ["--help"])
        assert r.exit_code == 0, cmd
    r = CliRunner().invoke(main, ["encode", "bc1", str(tmp_path / "missing.png")])
    assert r.exit_code == 2  # click: the input does not exist
    r = CliRunner().invoke(main, ["encode", "bc1", "-l", "19", str(tmp_path)])
    assert r.exit_code == 2  # level range 0..18, as the reference's option
    png = tmp_path / "img.png"
    png.write_bytes(b"not a dds")
    r = CliRunner().invoke(main, ["decode", str(png)])
    assert r.exit_code != 0 and "is not a DDS file" in r.output
