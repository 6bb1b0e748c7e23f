"""CPU oracle for the S3TC encode/decode path — TEST INFRASTRUCTURE ONLY.

Two checkers live here, and nothing in the product may import, link or call
either of them (only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / reference legs do):

* ``Oracle`` wraps ``_build/libqtoracle.so``, built from ``qt_oracle.c``: a
  plain-C restatement of the reference algorithm, function by function, each
  citing the reference ``file:line`` it follows.
* ``Reference`` wraps ``_ref/libqtref.so``: the UNMODIFIED reference sources
  (drewcassidy/quicktex ``quicktex/*.cpp``, ``quicktex/s3tc/**/*.cpp``)
  compiled where they lie by ``oracle/Makefile``, driven through
  ``ref_harness.cpp``. It pins the restatement: the CPU tests check
  ``Oracle`` against ``Reference`` and against the golden vectors in
  ``tests/golden``.

Both expose the same calls, on numpy ``uint8`` arrays:

    bc1_encode(rgba, w, h, params) -> bytes      bc1_decode(blocks, w, h, interp, write_alpha) -> rgba
    bc3_encode(rgba, w, h, params) -> bytes      bc3_decode(blocks, w, h, interp) -> rgba
    bc4_encode(rgba, w, h, channel) -> bytes     bc4_decode(blocks, w, h, channel) -> rgba
    bc5_encode(rgba, w, h, c0, c1) -> bytes      bc5_decode(blocks, w, h, c0, c1) -> rgba

``params`` is a ``BC1Params`` (level preset plus advanced overrides).
"""

from __future__ import annotations

import ctypes
import dataclasses
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libqtoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqtref.so")
ORDER_TABLES = os.path.join(os.path.dirname(HERE), "quicktex_b200", "data", "bc1_order_tables.bin")

# Reference enum values (BC1Encoder.h:57-100, Interpolator.h:30).
FOUR_COLOR, THREE_COLOR, THREE_COLOR_BLACK = 0x04, 0x03, 0x13
ERR_NONE, ERR_FASTER, ERR_CHECK2, ERR_FULL = 0, 1, 2, 3
EP_LEAST_SQUARES, EP_BOUNDING_BOX, EP_BOUNDING_BOX_INT, EP_PCA = 0, 1, 2, 3
IDEAL, IDEAL_ROUND, NVIDIA, AMD = 0, 1, 2, 3


@dataclasses.dataclass
class BC1Params:
    """A BC1 encoder configuration: a level preset, a colour mode, an
    interpolator and optional advanced overrides (None keeps the preset)."""

    level: int = 5
    color_mode: int = FOUR_COLOR
    interpolator: int = IDEAL
    error_mode: Optional[int] = None
    endpoint_mode: Optional[int] = None
    two_ls_passes: Optional[bool] = None
    two_ep_passes: Optional[bool] = None
    two_cf_passes: Optional[bool] = None
    exhaustive: Optional[bool] = None
    search_rounds: Optional[int] = None
    orderings4: Optional[int] = None
    orderings3: Optional[int] = None
    power_iterations: Optional[int] = None

    def overrides(self):
        vals = [self.error_mode, self.endpoint_mode, self.two_ls_passes, self.two_ep_passes,
                self.two_cf_passes, self.exhaustive, self.search_rounds, self.orderings4,
                self.orderings3, self.power_iterations]
        return (ctypes.c_int * 10)(*[-1 if v is None else int(v) for v in vals])


def build(force: bool = False, ref_root: Optional[str] = None) -> None:
    """Compile the checkers (``make -C oracle``). The reference checker is built
    only when ``ref_root`` (else ``QT_REFERENCE_ROOT`` from the environment)
    names a reference source tree."""
    ref_root = ref_root or os.environ.get("QT_REFERENCE_ROOT")
    targets = ["oracle"]
    if ref_root and os.path.isdir(os.path.join(ref_root, "quicktex")):
        targets.append("ref")
    cmd = ["make", "-C", HERE] + ([f"REF={ref_root}"] if "ref" in targets else []) + (["-B"] if force else []) + targets
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)


_vp = ctypes.c_void_p
_i = ctypes.c_int


def _nblocks(w, h):
    return ((w + 3) // 4) * ((h + 3) // 4)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _as_u8(buf) -> np.ndarray:
    a = np.ascontiguousarray(np.frombuffer(bytes(buf), np.uint8) if not isinstance(buf, np.ndarray) else buf)
    assert a.dtype == np.uint8
    return a.reshape(-1)


class _Lib:
    prefix = ""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"checker library missing: {path} (run oracle.build())")
        self.lib = ctypes.CDLL(path)
        p = self.prefix
        sig = {
            "bc1_encode": [_vp, _i, _i, _i, _i, _i, _vp, _vp, _i],
            "bc3_encode": [_vp, _i, _i, _i, _i, _vp, _i],
            "bc4_encode": [_vp, _i, _i, _i, _vp, _i],
            "bc5_encode": [_vp, _i, _i, _i, _i, _vp, _i],
            "bc1_decode": [_vp, _i, _i, _i, _i, _vp],
            "bc3_decode": [_vp, _i, _i, _i, _vp],
            "bc4_decode": [_vp, _i, _i, _i, _vp],
            "bc5_decode": [_vp, _i, _i, _i, _i, _vp],
            "bc1_level_params": [_i, _i, _vp],
            "set_threads": [_i],
        }
        for name, args in sig.items():
            f = getattr(self.lib, p + name)
            f.argtypes = args
            f.restype = None if name == "set_threads" else _i
        # getattr (not lib[...]) so the restype sticks to the cached function object
        getattr(self.lib, p + "last_error").restype = ctypes.c_char_p
        getattr(self.lib, p + "num_threads").restype = _i

    def _call(self, name, *args):
        rc = getattr(self.lib, self.prefix + name)(*args)
        if rc != 0:
            raise RuntimeError(getattr(self.lib, self.prefix + "last_error")().decode())

    def set_threads(self, n: int) -> None:
        getattr(self.lib, self.prefix + "set_threads")(int(n))

    def num_threads(self) -> int:
        return getattr(self.lib, self.prefix + "num_threads")()

    def level_params(self, level: int, color_mode: int = FOUR_COLOR):
        out = (ctypes.c_int * 10)()
        self._call("bc1_level_params", level, color_mode, out)
        return list(out)

    # mode 0: as-shipped Encode loop; mode 1: OpenMP over every block.
    def bc1_encode(self, rgba, w, h, params: BC1Params = BC1Params(), mode: int = 1) -> bytes:
        src = _as_u8(rgba)
        out = np.zeros(_nblocks(w, h) * 8, np.uint8)
        self._call("bc1_encode", _ptr(src), w, h, params.level, params.color_mode, params.interpolator,
                   params.overrides(), _ptr(out), mode)
        return out.tobytes()

    def bc3_encode(self, rgba, w, h, params: BC1Params = BC1Params(), mode: int = 1) -> bytes:
        src = _as_u8(rgba)
        out = np.zeros(_nblocks(w, h) * 16, np.uint8)
        self._call("bc3_encode", _ptr(src), w, h, params.level, params.interpolator, _ptr(out), mode)
        return out.tobytes()

    def bc4_encode(self, rgba, w, h, channel: int = 3, mode: int = 1) -> bytes:
        src = _as_u8(rgba)
        out = np.zeros(_nblocks(w, h) * 8, np.uint8)
        self._call("bc4_encode", _ptr(src), w, h, channel, _ptr(out), mode)
        return out.tobytes()

    def bc5_encode(self, rgba, w, h, c0: int = 0, c1: int = 1, mode: int = 1) -> bytes:
        src = _as_u8(rgba)
        out = np.zeros(_nblocks(w, h) * 16, np.uint8)
        self._call("bc5_encode", _ptr(src), w, h, c0, c1, _ptr(out), mode)
        return out.tobytes()

    def bc1_decode(self, blocks, w, h, interp: int = IDEAL, write_alpha: bool = False) -> bytes:
        src = _as_u8(blocks)
        out = np.zeros(w * h * 4, np.uint8)
        self._call("bc1_decode", _ptr(src), w, h, interp, int(write_alpha), _ptr(out))
        return out.tobytes()

    def bc3_decode(self, blocks, w, h, interp: int = IDEAL) -> bytes:
        src = _as_u8(blocks)
        out = np.zeros(w * h * 4, np.uint8)
        self._call("bc3_decode", _ptr(src), w, h, interp, _ptr(out))
        return out.tobytes()

    def bc4_decode(self, blocks, w, h, channel: int = 3) -> bytes:
        src = _as_u8(blocks)
        out = np.zeros(w * h * 4, np.uint8)
        self._call("bc4_decode", _ptr(src), w, h, channel, _ptr(out))
        return out.tobytes()

    def bc5_decode(self, blocks, w, h, c0: int = 0, c1: int = 1) -> bytes:
        src = _as_u8(blocks)
        out = np.zeros(w * h * 4, np.uint8)
        self._call("bc5_decode", _ptr(src), w, h, c0, c1, _ptr(out))
        return out.tobytes()


class Reference(_Lib):
    """The unmodified reference codec (``oracle/_ref/libqtref.so``)."""

    prefix = "ref_"

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        self.lib.ref_time_encode.argtypes = [_i, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i]
        self.lib.ref_time_encode.restype = ctypes.c_double
        self.lib.ref_time_decode.argtypes = [_i, _vp, _i, _i, _i, _i, _i, _i, _i]
        self.lib.ref_time_decode.restype = ctypes.c_double

    # CPU baseline timing: seconds of the fastest of `reps` runs (after one untimed run) of one
    # encode/decode, with the codec, its tables and the input built beforehand. mode 0: the
    # reference's own Encode/Decode loop as shipped; mode 1: OpenMP over EncodeBlock/DecodeBlock.
    def time_encode(self, fmt: int, rgba, w, h, params: BC1Params = BC1Params(), c0: int = 0, c1: int = 1,
                    mode: int = 0, reps: int = 1) -> float:
        src = _as_u8(rgba)
        t = self.lib.ref_time_encode(fmt, _ptr(src), w, h, params.level, params.color_mode, params.interpolator,
                                     c0, c1, mode, reps)
        if t < 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return t

    def time_decode(self, fmt: int, blocks, w, h, interp: int = IDEAL, c0: int = 0, c1: int = 1, mode: int = 0,
                    reps: int = 1) -> float:
        src = _as_u8(blocks)
        t = self.lib.ref_time_decode(fmt, _ptr(src), w, h, interp, c0, c1, mode, reps)
        if t < 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return t


class Oracle(_Lib):
    """The plain-C restatement (``oracle/_build/libqtoracle.so``)."""

    prefix = "qo_"

    def __init__(self, path: str = ORACLE_SO, tables: str = ORDER_TABLES):
        super().__init__(path)
        self.lib.qo_ce_count.restype = ctypes.c_ulonglong
        self.lib.qo_ce_repeated_count.restype = ctypes.c_ulonglong
        self.lib.qo_init.argtypes = [ctypes.c_char_p]
        self.lib.qo_init.restype = _i
        if self.lib.qo_init(tables.encode()) != 0:
            raise RuntimeError(self.lib.qo_last_error().decode())


    def ce_count(self) -> int:
        """Candidate evaluations (SSD + select of one texel vs one palette colour)
        performed by the encodes since the last ``ce_reset``."""
        return int(self.lib.qo_ce_count())

    def ce_repeated_count(self) -> int:
        """Of ``ce_count``, the evaluations in second four-colour cluster-fit passes that repeat
        the first pass's trials (same start hash and texel order, or zero error), which cannot
        change the result."""
        return int(self.lib.qo_ce_repeated_count())

    def ce_reset(self) -> None:
        self.lib.qo_ce_reset()


def reference_available() -> bool:
    return os.path.exists(REF_SO)
