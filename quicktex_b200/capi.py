"""ctypes binding of the C-ABI in ``include/quicktex_cuda.h``.

This is how a non-C++ caller drives ``libquicktex_cuda.so``; the parity tests
and the benchmark use it to call through the boundary exactly as such a caller
would. Host-buffer calls take numpy ``uint8`` arrays (or anything exposing the
buffer protocol); device calls take raw device pointers (ints) and a
``cudaStream_t`` (int, 0 = legacy default stream).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import library_path

QT_OK, QT_ERR_ARG, QT_ERR_OOM, QT_ERR_CUDA, QT_ERR_TIMEOUT, QT_ERR_RANGE, QT_ERR_STATE = range(7)
FOUR_COLOR, THREE_COLOR, THREE_COLOR_BLACK = 0x04, 0x03, 0x13
IDEAL, IDEAL_ROUND, NVIDIA, AMD = 0, 1, 2, 3

# every symbol include/quicktex_cuda.h declares
EXPORTS = (
    "qt_bc1_params_for_level", "qt_bc1_params_validate", "qt_init", "qt_last_error", "qt_version",
    "qt_bc1_encode_host", "qt_bc1_encode_device", "qt_bc3_encode_host", "qt_bc3_encode_device",
    "qt_bc4_encode_host", "qt_bc4_encode_device", "qt_bc5_encode_host", "qt_bc5_encode_device",
    "qt_bc1_decode_host", "qt_bc1_decode_device", "qt_bc3_decode_host", "qt_bc3_decode_device",
    "qt_bc4_decode_host", "qt_bc4_decode_device", "qt_bc5_decode_host", "qt_bc5_decode_device",
    "qt_batch_create", "qt_batch_destroy", "qt_batch_set_rules", "qt_batch_set_grid", "qt_batch_set_threads", "qt_batch_run",
    "qt_batch_last_tiles", "qt_batch_reserve", "qt_copy_async", "qt_batch_run_noalloc", "qt_batch_run_plain",
    "qt_server_create", "qt_server_destroy", "qt_server_set_rules", "qt_server_set_grid", "qt_server_set_threads",
    "qt_server_submit",
    "qt_server_poll", "qt_server_get_stats", "qt_server_clock",
    "qt_resize_bilinear_device", "qt_flip_swizzle_device", "qt_bc1_encode_kernels", "qt_host_alloc", "qt_host_free",
)


class BC1Params(ctypes.Structure):
    """``qt_bc1_params``: resolved BC1 settings."""

    _fields_ = [
        ("color_mode", ctypes.c_int32), ("interpolator", ctypes.c_int32), ("error_mode", ctypes.c_int32),
        ("endpoint_mode", ctypes.c_int32), ("two_ls_passes", ctypes.c_int32), ("two_ep_passes", ctypes.c_int32),
        ("two_cf_passes", ctypes.c_int32), ("exhaustive", ctypes.c_int32), ("search_rounds", ctypes.c_uint32),
        ("orderings4", ctypes.c_uint32), ("orderings3", ctypes.c_uint32), ("power_iterations", ctypes.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class QtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None
_vp, _i = ctypes.c_void_p, ctypes.c_int


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python quicktex_b200/build.py`")
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(BC1Params)
        sig = {
            "qt_bc1_params_for_level": [ctypes.c_uint, _i, _i, P],
            "qt_bc1_params_validate": [P],
            "qt_init": [_i],
            "qt_bc1_encode_host": [_vp, _i, _i, P, _vp],
            "qt_bc3_encode_host": [_vp, _i, _i, P, _vp],
            "qt_bc4_encode_host": [_vp, _i, _i, _i, _vp],
            "qt_bc5_encode_host": [_vp, _i, _i, _i, _i, _vp],
            "qt_bc1_encode_device": [_vp, _i, _i, P, _vp, _vp],
            "qt_bc3_encode_device": [_vp, _i, _i, P, _vp, _vp],
            "qt_bc1_encode_kernels": [_i, _i, P, ctypes.POINTER(_i)],
            "qt_bc4_encode_device": [_vp, _i, _i, _i, _vp, _vp],
            "qt_bc5_encode_device": [_vp, _i, _i, _i, _i, _vp, _vp],
            "qt_bc1_decode_host": [_vp, _i, _i, _i, _i, _vp],
            "qt_bc3_decode_host": [_vp, _i, _i, _i, _vp],
            "qt_bc4_decode_host": [_vp, _i, _i, _i, _vp],
            "qt_bc5_decode_host": [_vp, _i, _i, _i, _i, _vp],
            "qt_bc1_decode_device": [_vp, _i, _i, _i, _i, _vp, _vp],
            "qt_bc3_decode_device": [_vp, _i, _i, _i, _vp, _vp],
            "qt_bc4_decode_device": [_vp, _i, _i, _i, _vp, _vp],
            "qt_bc5_decode_device": [_vp, _i, _i, _i, _i, _vp, _vp],
            "qt_resize_bilinear_device": [_vp, _i, _i, _vp, _i, _i, _vp],
            "qt_flip_swizzle_device": [_vp, _i, _i, _vp, _i, _i, _i, _vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _i
        L.qt_last_error.restype = ctypes.c_char_p
        L.qt_version.restype = ctypes.c_char_p
        L.qt_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(_vp)]
        L.qt_host_alloc.restype = _i
        L.qt_host_free.argtypes = [_vp]
        L.qt_host_free.restype = None
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != QT_OK:
        raise QtError(rc, lib().qt_last_error().decode())


def params_for_level(level: int = 5, color_mode: int = FOUR_COLOR, interpolator: int = IDEAL, **overrides) -> BC1Params:
    """``qt_bc1_params_for_level`` then optional field overrides (validated/clamped)."""
    p = BC1Params()
    check(lib().qt_bc1_params_for_level(level, color_mode, interpolator, ctypes.byref(p)))
    if overrides:
        for k, v in overrides.items():
            if v is not None:
                setattr(p, k, int(v))
        check(lib().qt_bc1_params_validate(ctypes.byref(p)))
    return p


def nblocks(w: int, h: int) -> int:
    return ((w + 3) // 4) * ((h + 3) // 4)


def _u8(a) -> np.ndarray:
    a = np.ascontiguousarray(a if isinstance(a, np.ndarray) else np.frombuffer(bytes(a), np.uint8))
    return a.reshape(-1).view(np.uint8)


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


# ---- host-buffer entry points -------------------------------------------------
def bc1_encode(rgba, w: int, h: int, params: BC1Params) -> bytes:
    src, out = _u8(rgba), np.empty(nblocks(w, h) * 8, np.uint8)
    check(lib().qt_bc1_encode_host(_p(src), w, h, ctypes.byref(params), _p(out)))
    return out.tobytes()


def bc3_encode(rgba, w: int, h: int, params: BC1Params) -> bytes:
    src, out = _u8(rgba), np.empty(nblocks(w, h) * 16, np.uint8)
    check(lib().qt_bc3_encode_host(_p(src), w, h, ctypes.byref(params), _p(out)))
    return out.tobytes()


def bc4_encode(rgba, w: int, h: int, channel: int = 3) -> bytes:
    src, out = _u8(rgba), np.empty(nblocks(w, h) * 8, np.uint8)
    check(lib().qt_bc4_encode_host(_p(src), w, h, channel, _p(out)))
    return out.tobytes()


def bc5_encode(rgba, w: int, h: int, c0: int = 0, c1: int = 1) -> bytes:
    src, out = _u8(rgba), np.empty(nblocks(w, h) * 16, np.uint8)
    check(lib().qt_bc5_encode_host(_p(src), w, h, c0, c1, _p(out)))
    return out.tobytes()


def bc1_decode(blocks, w: int, h: int, interpolator: int = IDEAL, write_alpha: bool = False) -> bytes:
    src, out = _u8(blocks), np.empty(w * h * 4, np.uint8)
    check(lib().qt_bc1_decode_host(_p(src), w, h, interpolator, int(write_alpha), _p(out)))
    return out.tobytes()


def bc3_decode(blocks, w: int, h: int, interpolator: int = IDEAL) -> bytes:
    src, out = _u8(blocks), np.empty(w * h * 4, np.uint8)
    check(lib().qt_bc3_decode_host(_p(src), w, h, interpolator, _p(out)))
    return out.tobytes()


def bc4_decode(blocks, w: int, h: int, channel: int = 3) -> bytes:
    src, out = _u8(blocks), np.empty(w * h * 4, np.uint8)
    check(lib().qt_bc4_decode_host(_p(src), w, h, channel, _p(out)))
    return out.tobytes()


def bc5_decode(blocks, w: int, h: int, c0: int = 0, c1: int = 1) -> bytes:
    src, out = _u8(blocks), np.empty(w * h * 4, np.uint8)
    check(lib().qt_bc5_decode_host(_p(src), w, h, c0, c1, _p(out)))
    return out.tobytes()


# ---- device entry points (pointers are ints) ------------------------------------
def bc1_encode_device(d_rgba: int, w: int, h: int, params: BC1Params, d_out: int, stream: int = 0) -> None:
    check(lib().qt_bc1_encode_device(_vp(d_rgba), w, h, ctypes.byref(params), _vp(d_out), _vp(stream)))


def bc3_encode_device(d_rgba: int, w: int, h: int, params: BC1Params, d_out: int, stream: int = 0) -> None:
    check(lib().qt_bc3_encode_device(_vp(d_rgba), w, h, ctypes.byref(params), _vp(d_out), _vp(stream)))


def bc1_encode_kernels(w: int, h: int, params: BC1Params) -> int:
    """Kernels one bc1/bc3 device encode call of a w x h texture launches on the current device."""
    n = ctypes.c_int(0)
    check(lib().qt_bc1_encode_kernels(w, h, ctypes.byref(params), ctypes.byref(n)))
    return n.value


def bc4_encode_device(d_rgba: int, w: int, h: int, channel: int, d_out: int, stream: int = 0) -> None:
    check(lib().qt_bc4_encode_device(_vp(d_rgba), w, h, channel, _vp(d_out), _vp(stream)))


def bc5_encode_device(d_rgba: int, w: int, h: int, c0: int, c1: int, d_out: int, stream: int = 0) -> None:
    check(lib().qt_bc5_encode_device(_vp(d_rgba), w, h, c0, c1, _vp(d_out), _vp(stream)))


def bc1_decode_device(d_blocks: int, w: int, h: int, interpolator: int, write_alpha: bool, d_out: int, stream: int = 0) -> None:
    check(lib().qt_bc1_decode_device(_vp(d_blocks), w, h, interpolator, int(write_alpha), _vp(d_out), _vp(stream)))
