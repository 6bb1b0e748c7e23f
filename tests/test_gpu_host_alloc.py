"""GPU: qt_host_alloc hands out pinned host memory for blocks of 256 KiB and more (ordinary
memory below), reuses freed blocks of the same size class, and the drop-in texture classes
keep their texels in it, so their encodes copy with the copy engines directly and give the
same bytes as the device entry point."""

import ctypes

import numpy as np
import pytest

import workloads as syn
from quicktex_b200 import capi

pytestmark = pytest.mark.gpu

HOST, UNREGISTERED = 1, 0  # cudaMemoryType


def _mem_type(addr: int) -> int:
    from cuda import cudart

    err, attrs = cudart.cudaPointerGetAttributes(addr)
    assert err == cudart.cudaError_t.cudaSuccess, err
    return int(attrs.type)


def _alloc(n: int) -> int:
    p = ctypes.c_void_p()
    capi.check(capi.lib().qt_host_alloc(n, ctypes.byref(p)))
    return p.value


def test_large_blocks_are_pinned_and_reused():
    import torch

    torch.cuda.init()
    L = capi.lib()
    big = _alloc(64 << 20)
    assert _mem_type(big) == HOST
    small = _alloc(100 << 10)
    assert _mem_type(small) == UNREGISTERED
    L.qt_host_free(ctypes.c_void_p(big))
    again = _alloc((64 << 20) - 1000)  # the same size class comes back from the cache
    assert again == big
    L.qt_host_free(ctypes.c_void_p(again))
    L.qt_host_free(ctypes.c_void_p(small))


def test_dropin_textures_are_pinned_and_encode_like_device():
    import torch

    import quicktex_b200 as qt
    from quicktex_b200.s3tc.bc1 import BC1Encoder

    w, h = 2048, 1030
    img = np.ascontiguousarray(syn.block_mix(w, h, workload=5))
    tex = qt.RawTexture.frombytes(img.tobytes(), w, h)
    assert _mem_type(np.frombuffer(memoryview(tex), np.uint8).ctypes.data) == HOST
    for level in (0, 18):
        out = BC1Encoder(level).encode(tex)
        assert _mem_type(np.frombuffer(memoryview(out), np.uint8).ctypes.data) == HOST
        p = capi.params_for_level(level)
        d_in = torch.from_numpy(img.reshape(-1)).cuda()
        d_out = torch.empty(out.nbytes, dtype=torch.uint8, device="cuda")
        capi.bc1_encode_device(d_in.data_ptr(), w, h, p, d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert out.tobytes() == d_out.cpu().numpy().tobytes(), level
