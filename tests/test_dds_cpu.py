"""CPU: DDS files written by the reference (tests/golden/dds, made by
make_dds_golden.py) parse with this package's dds.read, and tobytes() writes
them back byte for byte; the header fields follow the reference's rules."""

import hashlib
import json
import os

import pytest

from quicktex_b200 import dds
from quicktex_b200.image_utils import mip_sizes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dds")
MANIFEST = json.load(open(os.path.join(GOLD, "manifest.json")))["cases"]


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_read_and_write_back(name):
    path = os.path.join(GOLD, name + ".dds")
    data = open(path, "rb").read()
    assert hashlib.sha256(data).hexdigest() == MANIFEST[name]["file_sha256"]
    f = dds.read(path)
    assert f.mipmap_count == MANIFEST[name]["mips"] == len(f.textures)
    assert [t.size for t in f.textures] == mip_sizes(f.size, f.mipmap_count)
    assert f.pitch == f.textures[0].nbytes
    assert f.tobytes() == data
    multi = f.mipmap_count > 1
    assert (dds.DDSFlags.MIPMAPCOUNT in f.flags) == multi
    assert bool(f.caps[0] & dds.Caps0.MIPMAP) == multi


def test_read_rejects_bad_files(tmp_path):
    p = tmp_path / "x.dds"
    p.write_bytes(b"NOPE" + bytes(124))
    with pytest.raises(AssertionError):
        dds.read(p)
    good = open(os.path.join(GOLD, "bc1_l5_37x21.dds"), "rb").read()
    p.write_bytes(good[:-5])
    with pytest.raises(AssertionError):
        dds.read(p)
