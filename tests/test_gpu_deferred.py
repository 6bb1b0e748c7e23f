"""GPU: the three-pass encoder of large BC1/BC3 textures at levels with
EndpointSearch (solid blocks written by the split pass, searches queued per
colour mode and run by the refill kernel) gives, block for block, the oracle's
output. A block depends only on its own 16 texels, so block-aligned crops of
the large texture, encoded by the oracle, pin the corresponding blocks; the
crops are chosen so that all three search queues (four-colour, three-colour,
three-colour + black) are exercised, and BC3's colour half is checked at its
offset."""

import numpy as np
import pytest

import quicktex_b200.synth as syn
from oracle import BC1Params
from quicktex_b200 import capi

pytestmark = pytest.mark.gpu

SIDE = 2048  # 262,144 blocks: above the deferred-search threshold (two searches per resident lane)
CROPS = [(0, 0), (1024, 512), (1984, 1984), (640, 1600)]  # (x, y) texel offsets, 64x64 each


def _device_encode(fn, img, params, bsz):
    """Through the device entry point: one launch over the whole texture."""
    import torch

    d_in = torch.from_numpy(img.reshape(-1).copy()).cuda()
    d_out = torch.empty((SIDE // 4) ** 2 * bsz, dtype=torch.uint8, device="cuda")
    fn(d_in.data_ptr(), SIDE, SIDE, params, d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return d_out.cpu().numpy().tobytes()


def _crop_blocks(full_blocks, bsz, x, y, n=16):
    bw = SIDE // 4
    rows = [full_blocks[((y // 4 + r) * bw + x // 4) * bsz: ((y // 4 + r) * bw + x // 4 + n) * bsz] for r in range(n)]
    return b"".join(rows)


@pytest.mark.parametrize("level,mode,interp", [(18, 0x04, 0), (18, 0x03, 2), (18, 0x13, 1), (14, 0x04, 3), (17, 0x03, 0)])
def test_bc1_deferred_search_matches_oracle(oracle_lib, level, mode, interp):
    img = np.ascontiguousarray(syn.block_mix(SIDE, SIDE, workload=14, stream=level + mode))
    p = capi.params_for_level(level, mode, interp)
    out = _device_encode(capi.bc1_encode_device, img, p, 8)
    assert capi.bc1_encode(img, SIDE, SIDE, p) == out  # the banded host path, bands above the threshold too
    for x, y in CROPS:
        crop = np.ascontiguousarray(img[y:y + 64, x:x + 64])
        exp = oracle_lib.bc1_encode(crop, 64, 64, BC1Params(level=level, color_mode=mode, interpolator=interp))
        assert _crop_blocks(out, 8, x, y) == exp, (level, mode, interp, x, y)


def test_bc3_deferred_search_matches_oracle(oracle_lib):
    img = np.ascontiguousarray(syn.alpha_mix(SIDE, SIDE, workload=14, stream=99))
    p = capi.params_for_level(18, capi.FOUR_COLOR, 2)
    out = _device_encode(capi.bc3_encode_device, img, p, 16)
    assert capi.bc3_encode(img, SIDE, SIDE, p) == out
    for x, y in CROPS:
        crop = np.ascontiguousarray(img[y:y + 64, x:x + 64])
        exp = oracle_lib.bc3_encode(crop, 64, 64, BC1Params(level=18, color_mode=capi.FOUR_COLOR, interpolator=2))
        assert _crop_blocks(out, 16, x, y) == exp, (x, y)
