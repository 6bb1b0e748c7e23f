"""GPU: the host-buffer entry points on textures large enough to be cut into
bands (uploads, kernels and downloads pipelined over two streams) return the
same bytes as the device entry points on the whole texture, for every format,
with and without ragged right and bottom edges (the wrap rule reaches across
bands there)."""

import ctypes

import numpy as np
import pytest

import workloads as syn
from quicktex_b200 import capi

pytestmark = pytest.mark.gpu

SIZES = [(2048, 2048), (2051, 2047), (4096, 1030), (1500, 3001)]


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()


@pytest.mark.parametrize("w,h", SIZES)
def test_banded_encode_equals_device(w, h):
    import torch

    L = capi.lib()
    img = np.ascontiguousarray(syn.alpha_mix(w, h, workload=12, stream=w + h)[:h, :w])
    d_in = _dev(img)
    nb = ((w + 3) // 4) * ((h + 3) // 4)
    s = torch.cuda.current_stream()
    p0 = capi.params_for_level(0)
    p3 = capi.params_for_level(3)
    # EndpointSearch settings on >= ~151k blocks take the parted host path: bands encoded to
    # their first cluster-fit pass as they arrive, then one pass over the shared queues
    p13 = capi.params_for_level(13, 0x03, 2)
    p18 = capi.params_for_level(18, 0x13, 0)
    cases = [
        ("bc1 L13", 8, lambda src, dst: L.qt_bc1_encode_host(src, w, h, ctypes.byref(p13), dst),
         lambda src, dst: L.qt_bc1_encode_device(src, w, h, ctypes.byref(p13), dst, capi._vp(s.cuda_stream))),
        ("bc3 L18", 16, lambda src, dst: L.qt_bc3_encode_host(src, w, h, ctypes.byref(p18), dst),
         lambda src, dst: L.qt_bc3_encode_device(src, w, h, ctypes.byref(p18), dst, capi._vp(s.cuda_stream))),
        ("bc1", 8, lambda src, dst: L.qt_bc1_encode_host(src, w, h, ctypes.byref(p0), dst),
         lambda src, dst: L.qt_bc1_encode_device(src, w, h, ctypes.byref(p0), dst, capi._vp(s.cuda_stream))),
        ("bc3", 16, lambda src, dst: L.qt_bc3_encode_host(src, w, h, ctypes.byref(p3), dst),
         lambda src, dst: L.qt_bc3_encode_device(src, w, h, ctypes.byref(p3), dst, capi._vp(s.cuda_stream))),
        ("bc4", 8, lambda src, dst: L.qt_bc4_encode_host(src, w, h, 3, dst),
         lambda src, dst: L.qt_bc4_encode_device(src, w, h, 3, dst, capi._vp(s.cuda_stream))),
        ("bc5", 16, lambda src, dst: L.qt_bc5_encode_host(src, w, h, 0, 1, dst),
         lambda src, dst: L.qt_bc5_encode_device(src, w, h, 0, 1, dst, capi._vp(s.cuda_stream))),
    ]
    for name, bsz, host_fn, dev_fn in cases:
        out_h = np.empty(nb * bsz, np.uint8)
        capi.check(host_fn(capi._vp(img.ctypes.data), capi._vp(out_h.ctypes.data)))
        d_out = torch.empty(nb * bsz, dtype=torch.uint8, device="cuda")
        capi.check(dev_fn(capi._vp(d_in.data_ptr()), capi._vp(d_out.data_ptr())))
        assert np.array_equal(out_h, d_out.cpu().numpy()), (name, w, h)


@pytest.mark.parametrize("w,h", SIZES)
def test_banded_decode_equals_device(w, h):
    import torch

    L = capi.lib()
    nb = ((w + 3) // 4) * ((h + 3) // 4)
    rng = np.random.default_rng(w * 3 + h)
    s = torch.cuda.current_stream()
    for fmt, bsz in ((1, 8), (3, 16), (4, 8), (5, 16)):
        blocks = rng.integers(0, 256, nb * bsz, dtype=np.uint8)
        d_blocks = _dev(blocks)
        out_h = np.empty(w * h * 4, np.uint8)
        d_out = torch.empty(w * h * 4, dtype=torch.uint8, device="cuda")
        bp, hp, dp, sp = capi._vp(blocks.ctypes.data), capi._vp(out_h.ctypes.data), capi._vp(d_out.data_ptr()), capi._vp(s.cuda_stream)
        dbp = capi._vp(d_blocks.data_ptr())
        if fmt == 1:
            capi.check(L.qt_bc1_decode_host(bp, w, h, 2, 1, hp))
            capi.check(L.qt_bc1_decode_device(dbp, w, h, 2, 1, dp, sp))
        elif fmt == 3:
            capi.check(L.qt_bc3_decode_host(bp, w, h, 3, hp))
            capi.check(L.qt_bc3_decode_device(dbp, w, h, 3, dp, sp))
        elif fmt == 4:
            capi.check(L.qt_bc4_decode_host(bp, w, h, 1, hp))
            capi.check(L.qt_bc4_decode_device(dbp, w, h, 1, dp, sp))
        else:
            capi.check(L.qt_bc5_decode_host(bp, w, h, 2, 0, hp))
            capi.check(L.qt_bc5_decode_device(dbp, w, h, 2, 0, dp, sp))
        assert np.array_equal(out_h, d_out.cpu().numpy()), (fmt, w, h)


@pytest.mark.parametrize("w,h", [(2048, 2049), (2900, 2701)])
def test_banded_search_encode_equals_device(w, h):
    """Settings with EndpointSearch cut the texture into bands of at least the deferred-search
    threshold, each twice the last: 2048x2049 gives two bands, 2900x2701 three. Both have a ragged
    bottom edge, whose last band wraps to rows of the first (on the other stream for two bands)."""
    import torch

    L = capi.lib()
    img = np.ascontiguousarray(syn.alpha_mix(w, h, workload=14, stream=w * 7 + h)[:h, :w])
    d_in = _dev(img)
    nb = ((w + 3) // 4) * ((h + 3) // 4)
    s = torch.cuda.current_stream()
    p18 = capi.params_for_level(18, capi.THREE_COLOR, 2)
    p13 = capi.params_for_level(13)
    cases = [
        ("bc1 L18", 8, lambda src, dst: L.qt_bc1_encode_host(src, w, h, ctypes.byref(p18), dst),
         lambda src, dst: L.qt_bc1_encode_device(src, w, h, ctypes.byref(p18), dst, capi._vp(s.cuda_stream))),
        ("bc3 L13", 16, lambda src, dst: L.qt_bc3_encode_host(src, w, h, ctypes.byref(p13), dst),
         lambda src, dst: L.qt_bc3_encode_device(src, w, h, ctypes.byref(p13), dst, capi._vp(s.cuda_stream))),
    ]
    for name, bsz, host_fn, dev_fn in cases:
        out_h = np.empty(nb * bsz, np.uint8)
        capi.check(host_fn(capi._vp(img.ctypes.data), capi._vp(out_h.ctypes.data)))
        d_out = torch.empty(nb * bsz, dtype=torch.uint8, device="cuda")
        capi.check(dev_fn(capi._vp(d_in.data_ptr()), capi._vp(d_out.data_ptr())))
        assert np.array_equal(out_h, d_out.cpu().numpy()), (name, w, h)


@pytest.mark.parametrize("pieces", range(2, 13))
def test_staged_copy_of_uneven_length(pieces):
    """A pageable buffer is copied into the pinned staging chunk by up to 12 threads in
    64-byte-aligned pieces. Lengths of pieces x 512 KiB + 4 bytes split unevenly (the
    even share is itself a multiple of 64): the last 4 bytes (the texture's last texel
    on upload, the decoded texture's last texel on download) must arrive too."""
    import torch

    L = capi.lib()
    w, h = 1, pieces * 131072 + 1  # w * h * 4 = pieces * 524288 + 4 bytes
    img = np.random.default_rng(pieces).integers(0, 256, (h, w, 4), dtype=np.uint8)
    nb = (h + 3) // 4
    s = capi._vp(torch.cuda.current_stream().cuda_stream)
    p0 = capi.params_for_level(0)
    out_h = np.empty(nb * 8, np.uint8)
    capi.check(L.qt_bc1_encode_host(capi._vp(img.ctypes.data), w, h, ctypes.byref(p0), capi._vp(out_h.ctypes.data)))
    d_in, d_out = _dev(img), torch.empty(nb * 8, dtype=torch.uint8, device="cuda")
    capi.check(L.qt_bc1_encode_device(capi._vp(d_in.data_ptr()), w, h, ctypes.byref(p0), capi._vp(d_out.data_ptr()), s))
    assert np.array_equal(out_h, d_out.cpu().numpy())
    rgba_h = np.full(w * h * 4, 0xA5, np.uint8)
    capi.check(L.qt_bc1_decode_host(capi._vp(out_h.ctypes.data), w, h, 0, 1, capi._vp(rgba_h.ctypes.data)))
    d_rgba = torch.full((w * h * 4,), 0xA5, dtype=torch.uint8, device="cuda")
    capi.check(L.qt_bc1_decode_device(capi._vp(d_out.data_ptr()), w, h, 0, 1, capi._vp(d_rgba.data_ptr()), s))
    assert np.array_equal(rgba_h, d_rgba.cpu().numpy())


@pytest.mark.parametrize("pinned", [False, True])
def test_parted_search_encode_equals_device(pinned):
    """The parted host path (EndpointSearch settings on >= ~151k blocks) with pinned and
    with pageable host buffers, on a ragged texture whose last band waits for band 0."""
    import torch

    L = capi.lib()
    w, h = 2051, 2047
    img = np.ascontiguousarray(syn.block_mix(w, h, workload=7))
    nb = ((w + 3) // 4) * ((h + 3) // 4)
    s = capi._vp(torch.cuda.current_stream().cuda_stream)
    d_in = _dev(img)
    for level, mode, interp in ((18, 0x04, 0), (16, 0x03, 3)):
        p = capi.params_for_level(level, mode, interp)
        if pinned:
            h_in = torch.from_numpy(img.reshape(-1)).pin_memory()
            h_out = torch.zeros(nb * 8, dtype=torch.uint8).pin_memory()
            src, dst = capi._vp(h_in.data_ptr()), capi._vp(h_out.data_ptr())
        else:
            out_np = np.zeros(nb * 8, np.uint8)
            src, dst = capi._vp(img.ctypes.data), capi._vp(out_np.ctypes.data)
        capi.check(L.qt_bc1_encode_host(src, w, h, ctypes.byref(p), dst))
        got = h_out.numpy() if pinned else out_np
        d_out = torch.empty(nb * 8, dtype=torch.uint8, device="cuda")
        capi.check(L.qt_bc1_encode_device(capi._vp(d_in.data_ptr()), w, h, ctypes.byref(p), capi._vp(d_out.data_ptr()), s))
        assert np.array_equal(got, d_out.cpu().numpy()), (level, mode, interp, pinned)
