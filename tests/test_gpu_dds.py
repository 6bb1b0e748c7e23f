"""GPU: mip chains and DDS files. The device resize equals Pillow's BILINEAR
resize (image_utils.resize_no_premultiply) byte for byte; dds.encode (mip chain
resized on the device, all levels in one batch launch) writes exactly the files
the reference's dds.encode wrote (tests/golden/dds); decode_all returns the
levels the reference decodes."""

import hashlib
import json
import os
import sys

import numpy as np
import pytest

import quicktex_b200
from quicktex_b200 import dds
from quicktex_b200.image_utils import mip_sizes, resize_device, resize_no_premultiply

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "dds")
MANIFEST = json.load(open(os.path.join(GOLD, "manifest.json")))["cases"]
sys.path.insert(0, os.path.join(HERE, "golden"))
import dds_cases  # noqa: E402


@pytest.mark.parametrize("w,h", [(37, 21), (64, 64), (5, 130), (130, 1), (1, 9), (1000, 700), (257, 513)])
def test_device_resize_matches_pillow(w, h):
    import torch
    from PIL import Image

    rng = np.random.default_rng(w * 7 + h)
    rgba = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    img = Image.fromarray(rgba, "RGBA")
    src = torch.from_numpy(rgba.reshape(-1).copy()).cuda()
    s = torch.cuda.current_stream()
    sizes = mip_sizes((w, h)) + [(w + 3, max(1, h // 3)), (max(1, w // 5), h + 2)]  # and an up/down mix
    for dw, dh in sizes:
        dst = torch.empty(dw * dh * 4, dtype=torch.uint8, device="cuda")
        resize_device(src.data_ptr(), w, h, dst.data_ptr(), dw, dh, s.cuda_stream)
        ref = np.asarray(resize_no_premultiply(img, (dw, dh)))
        assert np.array_equal(dst.cpu().numpy().reshape(dh, dw, 4), ref), (w, h, dw, dh)


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_encode_writes_the_reference_file(name):
    c = dds_cases.CASES[name]
    enc = dds_cases.make_encoder(quicktex_b200, c["encoder"])
    f = dds.encode(dds_cases.image(name), enc, c["four_cc"], c.get("mip_count"))
    data = f.tobytes()
    assert data == open(os.path.join(GOLD, name + ".dds"), "rb").read()
    assert f.mipmap_count == MANIFEST[name]["mips"]


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_decode_all_matches_reference(name):
    f = dds.read(os.path.join(GOLD, name + ".dds"))
    levels = f.decode_all()
    assert [hashlib.sha256(im.tobytes()).hexdigest() for im in levels] == MANIFEST[name]["decoded_level_sha256"]
    assert f.decode(0).tobytes() == levels[0].tobytes()
