"""CPU tests of the C-ABI library: it loads, exports every symbol the public
header declares, resolves level presets like the reference, and rejects bad
arguments with the reference's error classes before touching a GPU."""

import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from quicktex_b200 import capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "quicktex_cuda.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(qt_\w+)\s*\(", text, re.M)))


def test_header_exports():
    names = declared_symbols()
    assert len(names) >= 20
    assert set(names) == set(capi.EXPORTS)
    lib = capi.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert b"sm_100a" in lib.qt_version()


@pytest.mark.parametrize("mode", [capi.FOUR_COLOR, capi.THREE_COLOR, capi.THREE_COLOR_BLACK])
def test_level_presets_match_oracle(oracle_lib, mode):
    keys = ["error_mode", "endpoint_mode", "two_ls_passes", "two_ep_passes", "two_cf_passes", "exhaustive",
            "search_rounds", "orderings4", "orderings3", "power_iterations"]
    for level in range(20):
        p = capi.params_for_level(level, mode, capi.NVIDIA)
        assert [getattr(p, k) for k in keys] == oracle_lib.level_params(level, mode), level
        assert p.color_mode == mode and p.interpolator == capi.NVIDIA


def test_level_presets_match_reference(reference_lib):
    for level in range(20):
        p = capi.params_for_level(level)
        got = [p.error_mode, p.endpoint_mode, p.two_ls_passes, p.two_ep_passes, p.two_cf_passes, p.exhaustive,
               p.search_rounds, p.orderings4, p.orderings3, p.power_iterations]
        assert got == reference_lib.level_params(level, 4), level


def test_validate_clamps():
    p = capi.params_for_level(5, orderings4=0, orderings3=99, power_iterations=1)
    assert (p.orderings4, p.orderings3, p.power_iterations) == (1, 32, 4)


def test_argument_errors():
    lib = capi.lib()
    p = capi.BC1Params()
    with pytest.raises(capi.QtError) as e:
        capi.params_for_level(20)
    assert e.value.code == capi.QT_ERR_ARG and "Level out of range" in str(e.value)
    assert lib.qt_bc1_params_for_level(5, 0x10, 0, ctypes.byref(p)) == capi.QT_ERR_ARG
    assert lib.qt_bc1_params_for_level(5, 0x04, 4, ctypes.byref(p)) == capi.QT_ERR_ARG
    buf = np.zeros(64, np.uint8)
    good = capi.params_for_level(5)
    assert lib.qt_bc1_encode_host(capi._p(buf), 0, 4, ctypes.byref(good), capi._p(buf)) == capi.QT_ERR_ARG
    assert b"width" in lib.qt_last_error()
    assert lib.qt_bc4_encode_host(capi._p(buf), 4, 4, 4, capi._p(buf)) == capi.QT_ERR_ARG
    assert b"Channel" in lib.qt_last_error()
    assert lib.qt_bc1_decode_host(capi._p(buf), 4, 4, 9, 0, capi._p(buf)) == capi.QT_ERR_ARG
    assert lib.qt_bc1_encode_device(None, 4, 4, ctypes.byref(good), None, None) == capi.QT_ERR_ARG
    # misaligned device pointers are rejected before any launch
    assert lib.qt_bc1_encode_device(ctypes.c_void_p(4096 + 2), 4, 4, ctypes.byref(good), ctypes.c_void_p(8192), None) == capi.QT_ERR_ARG
    # batch helpers check their arguments before touching a device
    from quicktex_b200 import batch

    L = batch._lib()
    assert L.qt_batch_reserve(None, 1, 1) == capi.QT_ERR_ARG
    assert L.qt_copy_async(None, 1, None) == capi.QT_ERR_ARG
    assert L.qt_copy_async(None, 0, None) == capi.QT_OK
    rows = np.array([[0, 4096, 16]], np.uint64)
    assert L.qt_copy_async(ctypes.c_void_p(rows.ctypes.data), 1, None) == capi.QT_ERR_ARG
    assert b"NULL" in lib.qt_last_error()


def test_error_message_is_thread_local():
    import threading

    lib = capi.lib()
    seen = {}

    def worker():
        lib.qt_bc4_encode_host(None, 4, 4, 9, None)
        seen["t"] = lib.qt_last_error()

    lib.qt_bc1_params_for_level(99, 4, 0, ctypes.byref(capi.BC1Params()))
    th = threading.Thread(target=worker)
    th.start()
    th.join()
    assert b"Level" in lib.qt_last_error()
    assert seen["t"] != lib.qt_last_error()


def test_server_argument_errors():
    """The serving entry points check their arguments before touching a device."""
    from quicktex_b200 import serve

    L = serve._lib()
    h = ctypes.c_void_p()
    assert L.qt_server_create(0, 1 << 20, 0, 1024, 64, ctypes.byref(h)) == capi.QT_ERR_ARG  # no slots
    assert L.qt_server_create(0, 0, 2, 1024, 64, ctypes.byref(h)) == capi.QT_ERR_ARG        # no budget
    assert L.qt_server_create(0, 1 << 20, 2, 1024, 64, None) == capi.QT_ERR_ARG
    n = ctypes.c_size_t()
    assert L.qt_server_submit(None, None, None, 1) == capi.QT_ERR_ARG
    assert L.qt_server_poll(None, None, None, None, 0, 0, ctypes.byref(n)) == capi.QT_ERR_ARG
    assert L.qt_server_get_stats(None, None) == capi.QT_ERR_ARG
    assert L.qt_server_destroy(None) == capi.QT_OK
    import time

    assert abs(L.qt_server_clock() - time.monotonic()) < 1.0


def test_host_alloc_without_gpu_is_ordinary_memory():
    """qt_host_alloc hands out writable blocks of every size even where no pinned memory can
    be had (this machine has no GPU); qt_host_free takes them back and ignores NULL and
    foreign pointers."""
    L = capi.lib()
    blocks = []
    for n in (0, 1, 4095, 4096, 300 << 10, 5 << 20):
        p = ctypes.c_void_p()
        assert L.qt_host_alloc(n, ctypes.byref(p)) == 0
        assert p.value
        if n:
            buf = (ctypes.c_uint8 * n).from_address(p.value)
            ctypes.memset(p.value, 0x5A, n)
            assert buf[0] == 0x5A and buf[n - 1] == 0x5A
        blocks.append(p)
    for p in blocks:
        L.qt_host_free(p)
    L.qt_host_free(None)
    foreign = ctypes.create_string_buffer(16)
    L.qt_host_free(ctypes.cast(foreign, ctypes.c_void_p))
    assert L.qt_host_alloc(16, None) != 0
    p = ctypes.c_void_p()
    assert L.qt_host_alloc(ctypes.c_size_t(-1).value, ctypes.byref(p)) == capi.QT_ERR_OOM and not p.value


def test_texture_storage_round_trips_on_cpu(qt):
    """The drop-in textures keep their bytes in qt_host_alloc blocks: construction, the
    reference's fills and bytes round trips hold without a GPU."""
    t = qt.RawTexture(3, 2)
    assert t.tobytes() == bytes([0, 0, 0, 255] * 6)
    data = bytes(range(256)) * 4
    r = qt.RawTexture.frombytes(data, 16, 16)
    assert r.tobytes() == data and bytes(memoryview(r)) == data
    from quicktex_b200.s3tc.bc1 import BC1Texture

    b = BC1Texture(9, 5)
    assert b.tobytes() == bytes(8 * 3 * 2)
