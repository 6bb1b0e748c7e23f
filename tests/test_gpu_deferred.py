"""GPU: the multi-pass encoder of large BC1/BC3 textures at levels with
EndpointSearch (solid blocks written by the split pass, the second cluster-fit
pass of level 18 queued for the blocks it can change, searches queued per
colour mode and run by the refill kernel) gives, block for block, the oracle's
output. A block depends only on its own 16 texels, so block-aligned crops of
the large texture, encoded by the oracle, pin the corresponding blocks; the
crops are chosen so that all three search queues (four-colour, three-colour,
three-colour + black) are exercised, and BC3's colour half is checked at its
offset."""

import numpy as np
import pytest

import workloads as syn
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


@pytest.mark.parametrize("mode,interp", [(0x04, 0), (0x03, 2), (0x13, 3)])
def test_bc1_level18_whole_texture_matches_oracle(oracle_lib, mode, interp):
    """Every block of a 2048^2 texture at level 18, through all five passes (split, encoder,
    the second cluster-fit pass for the blocks it can change, search, and the selectors of the
    searches that moved), against the oracle."""
    img = np.ascontiguousarray(syn.block_mix(SIDE, SIDE, workload=14, stream=18 + mode + interp))
    p = capi.params_for_level(18, mode, interp)
    assert capi.bc1_encode_kernels(SIDE, SIDE, p) == 5
    out = _device_encode(capi.bc1_encode_device, img, p, 8)
    exp = oracle_lib.bc1_encode(img, SIDE, SIDE, BC1Params(level=18, color_mode=mode, interpolator=interp))
    if out != exp:
        a, b = np.frombuffer(out, np.uint64), np.frombuffer(exp, np.uint64)
        bad = np.flatnonzero(a != b)
        raise AssertionError(f"{bad.size} of {a.size} blocks differ, first at block {bad[0]}")


def test_bc3_level18_whole_texture_matches_oracle(oracle_lib):
    img = np.ascontiguousarray(syn.alpha_mix(SIDE, SIDE, workload=14, stream=181))
    p = capi.params_for_level(18, capi.FOUR_COLOR, 0)
    out = _device_encode(capi.bc3_encode_device, img, p, 16)
    exp = oracle_lib.bc3_encode(img, SIDE, SIDE, BC1Params(level=18, color_mode=capi.FOUR_COLOR, interpolator=0))
    assert out == exp


def test_encode_kernel_count():
    """qt_bc1_encode_kernels reports the passes one device call launches: the encoder alone on
    small textures, the split pass first from 16384 blocks, the search pass and the pass that
    finishes the searches that moved on top of that for levels with EndpointSearch once the
    texture holds two searches per resident lane, and the second cluster-fit pass as its own
    kernel at levels with two of them (level 18)."""
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    side_defer = 4 * int(np.ceil(np.sqrt(2 * sms * 4 * 128)))
    p18, p10 = capi.params_for_level(18), capi.params_for_level(10)
    assert capi.bc1_encode_kernels(64, 64, p18) == 1
    assert capi.bc1_encode_kernels(508, 508, p18) == 1  # 127^2 = 16129 blocks
    assert capi.bc1_encode_kernels(512, 512, p18) == 2  # 16384 blocks
    assert capi.bc1_encode_kernels(side_defer, side_defer, p10) == 2
    assert capi.bc1_encode_kernels(side_defer, side_defer, p18) == 5
    assert capi.bc1_encode_kernels(SIDE, SIDE, capi.params_for_level(13)) == 4
    assert capi.bc1_encode_kernels(SIDE, SIDE, capi.params_for_level(17)) == 4
    assert capi.bc1_encode_kernels(SIDE, SIDE, capi.params_for_level(18)) == 5
    with pytest.raises(capi.QtError) as e:
        capi.bc1_encode_kernels(0, 64, p18)
    assert e.value.code == 1


@pytest.mark.parametrize("side,level,mode", [(256, 18, 0x04), (2048, 10, 0x04), (2048, 17, 0x03), (2048, 18, 0x13)])
def test_encode_kernel_count_matches_launches(side, level, mode):
    """The kernels one qt_bc1_encode_device call launches, as the CUDA profiler records them, are the
    number qt_bc1_encode_kernels reports (the figure bench.py counts launches with)."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    img = np.ascontiguousarray(syn.block_mix(side, side, workload=14, stream=side + level))
    p = capi.params_for_level(level, mode, 0)
    d_in = torch.from_numpy(img.reshape(-1).copy()).cuda()
    d_out = torch.empty((side // 4) ** 2 * 8, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    capi.bc1_encode_device(d_in.data_ptr(), side, side, p, d_out.data_ptr(), stream)  # warm-up
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        capi.bc1_encode_device(d_in.data_ptr(), side, side, p, d_out.data_ptr(), stream)
        torch.cuda.synchronize()
    launched = [e.name for e in prof.events() if "k_bc1_" in e.name]
    assert len(launched) == capi.bc1_encode_kernels(side, side, p), launched
