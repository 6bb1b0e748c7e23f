"""Batched persistent encode/decode (C-ABI ``qt_batch_*``).

Many textures of uneven sizes, formats (BC1/BC3/BC4/BC5), operations
(encode/decode) and levels run as ONE persistent kernel launch replayed from a
CUDA graph: each texture is cut into tiles of consecutive blocks, the tiles are
queued heaviest-first in device memory, and warps pull tiles (one block per
lane) until the queue is empty. Tile sizes and per-block costs per (op, format, level) come from
the tuning table written by ``quicktex_b200.autotune`` (``data/batch_tuning.json``).

Every output is byte-identical to the single-texture entry points: the batch
changes only the launch model.

    jobs = [Job.encode("bc1", rgba, w, h, level=18), Job.decode("bc4", blocks, w, h, channel=0), ...]
    outs = run_jobs(jobs)            # list of bytes, one per job
"""

from __future__ import annotations

import ctypes
import dataclasses
import json
import os
from typing import Optional, Sequence

import numpy as np

from . import capi

QT_OP_ENCODE, QT_OP_DECODE = 0, 1
FORMATS = {"bc1": 1, "bc3": 3, "bc4": 4, "bc5": 5}
BLOCK_BYTES = {1: 8, 3: 16, 4: 8, 5: 16}
TUNING_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "batch_tuning.json")


class BatchItem(ctypes.Structure):
    """``qt_batch_item``."""

    _fields_ = [
        ("op", ctypes.c_int32), ("format", ctypes.c_int32), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
        ("src", ctypes.c_void_p), ("dst", ctypes.c_void_p), ("params", capi.BC1Params),
        ("chan0", ctypes.c_int32), ("chan1", ctypes.c_int32), ("interpolator", ctypes.c_int32),
        ("write_alpha", ctypes.c_int32),
    ]


ITEM_DTYPE = np.dtype(BatchItem)  # the same layout as a numpy record


class TileRule(ctypes.Structure):
    """``qt_tile_rule``."""

    _fields_ = [("op", ctypes.c_int32), ("format", ctypes.c_int32), ("level", ctypes.c_int32),
                ("tile_blocks", ctypes.c_uint32), ("cost_per_block", ctypes.c_float)]


_sigs_done = False


def _lib():
    global _sigs_done
    L = capi.lib()
    if not _sigs_done:
        L.qt_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.qt_batch_destroy.argtypes = [ctypes.c_void_p]
        L.qt_batch_set_rules.argtypes = [ctypes.c_void_p, ctypes.POINTER(TileRule), ctypes.c_size_t]
        L.qt_batch_set_grid.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.qt_batch_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.qt_batch_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(BatchItem), ctypes.c_size_t, ctypes.c_void_p]
        L.qt_batch_last_tiles.argtypes = [ctypes.c_void_p]
        L.qt_batch_last_tiles.restype = ctypes.c_size_t
        L.qt_batch_reserve.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t]
        L.qt_copy_async.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        L.qt_batch_run_plain.argtypes = [ctypes.POINTER(BatchItem), ctypes.c_size_t, ctypes.c_void_p]
        for n in ("qt_batch_create", "qt_batch_destroy", "qt_batch_set_rules", "qt_batch_set_grid", "qt_batch_set_threads", "qt_batch_run",
                  "qt_batch_reserve", "qt_copy_async", "qt_batch_run_plain"):
            getattr(L, n).restype = ctypes.c_int
        _sigs_done = True
    return L


def load_tuning(path: str = TUNING_PATH) -> Optional[dict]:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


class Batch:
    """One batch queue (device buffers + captured graph) on one device."""

    def __init__(self, device: int = 0, tuning: Optional[dict] = None, use_default_tuning: bool = True):
        self.device = device
        h = ctypes.c_void_p()
        capi.check(_lib().qt_batch_create(device, ctypes.byref(h)))
        self.handle = h
        if tuning is None and use_default_tuning:
            tuning = load_tuning()
        if tuning:
            self.apply_tuning(tuning)

    def apply_tuning(self, tuning: dict) -> None:
        rules = tuning.get("rules", [])
        self.set_rules(rules)
        if tuning.get("threads_per_cta"):
            self.set_threads(int(tuning["threads_per_cta"]))
        if tuning.get("ctas_per_sm"):
            self.set_grid(int(tuning["ctas_per_sm"]))

    def set_rules(self, rules: Sequence[dict]) -> None:
        arr = (TileRule * max(1, len(rules)))()
        for i, r in enumerate(rules):
            arr[i] = TileRule(r["op"], r["format"], r.get("level", -1), r["tile_blocks"], r["cost_per_block"])
        capi.check(_lib().qt_batch_set_rules(self.handle, arr, len(rules)))

    def set_grid(self, ctas_per_sm: int) -> None:
        capi.check(_lib().qt_batch_set_grid(self.handle, ctas_per_sm))

    def set_threads(self, threads_per_cta: int) -> None:
        """Threads per CTA of the persistent kernel (32, 64 or 128)."""
        capi.check(_lib().qt_batch_set_threads(self.handle, threads_per_cta))

    def reserve(self, items: int, tiles: int) -> None:
        """Size the queue now so runs within these limits never reallocate it."""
        capi.check(_lib().qt_batch_reserve(self.handle, items, tiles))

    def run(self, items, stream: int = 0) -> None:
        """``items``: a sequence of ``BatchItem`` or an ``ITEM_DTYPE`` array."""
        if isinstance(items, np.ndarray):
            assert items.dtype == ITEM_DTYPE and items.flags.c_contiguous
            arr = ctypes.cast(ctypes.c_void_p(items.ctypes.data), ctypes.POINTER(BatchItem))
        else:
            arr = (BatchItem * max(1, len(items)))(*items)
        capi.check(_lib().qt_batch_run(self.handle, arr, len(items), ctypes.c_void_p(stream)))

    def last_tiles(self) -> int:
        return int(_lib().qt_batch_last_tiles(self.handle))

    def close(self) -> None:
        if self.handle:
            _lib().qt_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
class Job:
    """One texture to encode or decode."""

    op: int
    fmt: int
    width: int
    height: int
    data: np.ndarray  # RGBA8 texels (encode) or blocks (decode), uint8
    params: Optional[capi.BC1Params] = None
    chan0: int = 0
    chan1: int = 1
    interpolator: int = 0
    write_alpha: bool = False

    @staticmethod
    def encode(fmt: str, rgba, width: int, height: int, level: int = 5, color_mode: int = capi.FOUR_COLOR,
               interpolator: int = 0, channel: int = 3, chan0: int = 0, chan1: int = 1, params=None) -> "Job":
        f = FORMATS[fmt]
        if f in (1, 3) and params is None:
            params = capi.params_for_level(level, color_mode if f == 1 else capi.FOUR_COLOR, interpolator)
        c0, c1 = (channel, channel) if f == 4 else (chan0, chan1)
        return Job(QT_OP_ENCODE, f, width, height, np.ascontiguousarray(rgba, np.uint8).reshape(-1), params, c0, c1)

    @staticmethod
    def decode(fmt: str, blocks, width: int, height: int, interpolator: int = 0, write_alpha: bool = False,
               channel: int = 3, chan0: int = 0, chan1: int = 1) -> "Job":
        f = FORMATS[fmt]
        c0, c1 = (channel, channel) if f == 4 else (chan0, chan1)
        data = np.frombuffer(bytes(blocks), np.uint8) if not isinstance(blocks, np.ndarray) else blocks.reshape(-1)
        return Job(QT_OP_DECODE, f, width, height, data, None, c0, c1, interpolator, write_alpha)

    @property
    def nblocks(self) -> int:
        return ((self.width + 3) // 4) * ((self.height + 3) // 4)

    @property
    def out_bytes(self) -> int:
        return self.nblocks * BLOCK_BYTES[self.fmt] if self.op == QT_OP_ENCODE else self.width * self.height * 4

    def item(self, src: int, dst: int) -> BatchItem:
        it = BatchItem()
        it.op, it.format, it.width, it.height = self.op, self.fmt, self.width, self.height
        it.src, it.dst = src, dst
        if self.params is not None:
            it.params = self.params
        it.chan0, it.chan1, it.interpolator, it.write_alpha = self.chan0, self.chan1, self.interpolator, int(self.write_alpha)
        return it

    def record(self) -> np.void:
        """This job's ``qt_batch_item`` as an ``ITEM_DTYPE`` record with NULL buffers (cached)."""
        r = self.__dict__.get("_record")
        if r is None:
            r = np.frombuffer(bytes(self.item(0, 0)), ITEM_DTYPE)[0]
            self.__dict__["_record"] = r
        return r


def items_array(jobs: Sequence[Job], src, dst) -> np.ndarray:
    """``qt_batch_item`` array for ``jobs`` with buffer addresses ``src``/``dst`` (sequences of ints)."""
    arr = np.empty(len(jobs), ITEM_DTYPE)
    for k, j in enumerate(jobs):
        arr[k] = j.record()
    arr["src"] = src
    arr["dst"] = dst
    return arr


def copy_async(copies: np.ndarray, stream: int = 0) -> None:
    """``copies``: uint64 array of shape (n, 3) rows (dst, src, bytes); one
    cudaMemcpyAsync per row on ``stream`` (``qt_copy_async``)."""
    c = np.ascontiguousarray(copies, np.uint64)
    assert c.ndim == 2 and c.shape[1] == 3
    capi.check(_lib().qt_copy_async(ctypes.c_void_p(c.ctypes.data), len(c), ctypes.c_void_p(stream)))


def _align(n: int, a: int = 256) -> int:
    return (n + a - 1) // a * a


class Arena:
    """All jobs' inputs packed into one device buffer (and outputs into another),
    filled from one pinned host buffer: one upload and one download per batch."""

    def __init__(self, jobs: Sequence[Job], device: int = 0):
        import torch

        self.jobs = list(jobs)
        self.in_off, self.out_off = [], []
        ni = no = 0
        for j in self.jobs:
            self.in_off.append(ni)
            self.out_off.append(no)
            ni += _align(j.data.nbytes)
            no += _align(j.out_bytes)
        self.in_bytes, self.out_bytes = ni, no
        dev = torch.device("cuda", device)
        self.h_in = torch.empty(max(ni, 1), dtype=torch.uint8).pin_memory()
        self.h_out = torch.empty(max(no, 1), dtype=torch.uint8).pin_memory()
        hin = self.h_in.numpy()
        for j, o in zip(self.jobs, self.in_off):
            hin[o:o + j.data.nbytes] = j.data
        self.d_in = torch.empty(max(ni, 1), dtype=torch.uint8, device=dev)
        self.d_out = torch.empty(max(no, 1), dtype=torch.uint8, device=dev)

    def upload(self, stream=None):
        self.d_in.copy_(self.h_in, non_blocking=True)

    def download(self):
        self.h_out.copy_(self.d_out, non_blocking=True)

    def items(self) -> list[BatchItem]:
        bi, bo = self.d_in.data_ptr(), self.d_out.data_ptr()
        return [j.item(bi + a, bo + b) for j, a, b in zip(self.jobs, self.in_off, self.out_off)]

    def outputs(self) -> list[bytes]:
        ho = self.h_out.numpy()
        return [ho[o:o + j.out_bytes].tobytes() for j, o in zip(self.jobs, self.out_off)]


class PipelinedRun:
    """An arena's whole round trip (upload, persistent launch, download) cut into ``chunks``
    consecutive groups of textures of about equal block counts, each with its own queue. Chunk
    k's upload runs on a copy stream, its launch on a compute stream after that upload, its
    download on a second copy stream after that launch: the uploads of later chunks and the
    downloads of earlier ones overlap the launches. ``run()`` returns with every output in the
    arena's pinned host buffer."""

    def __init__(self, arena: "Arena", chunks: int = 4, device: int = 0, tuning: Optional[dict] = None):
        import torch

        self.arena = arena
        n = len(arena.jobs)
        total = sum(j.nblocks for j in arena.jobs)
        cuts, acc = [0], 0
        for k, j in enumerate(arena.jobs):
            acc += j.nblocks
            if len(cuts) < chunks and acc >= total * len(cuts) / chunks and k + 1 < n:
                cuts.append(k + 1)
        cuts.append(n)
        self.groups = [(a, b) for a, b in zip(cuts, cuts[1:]) if b > a]
        items = arena.items()
        self.items = [items[a:b] for a, b in self.groups]
        ends_in = arena.in_off[1:] + [arena.in_bytes]
        ends_out = arena.out_off[1:] + [arena.out_bytes]
        self.ranges = [(arena.in_off[a], ends_in[b - 1], arena.out_off[a], ends_out[b - 1]) for a, b in self.groups]
        self.batches = [Batch(device, tuning=tuning) for _ in self.groups]
        dev = torch.device("cuda", device)
        self.up, self.comp, self.down = (torch.cuda.Stream(dev) for _ in range(3))
        self.ev_up = [torch.cuda.Event() for _ in self.groups]
        self.ev_run = [torch.cuda.Event() for _ in self.groups]

    def run(self) -> None:
        import torch

        a = self.arena
        for (i0, i1, _, _), ev in zip(self.ranges, self.ev_up):
            with torch.cuda.stream(self.up):
                a.d_in[i0:i1].copy_(a.h_in[i0:i1], non_blocking=True)
            ev.record(self.up)
        for b, items, eu, er in zip(self.batches, self.items, self.ev_up, self.ev_run):
            self.comp.wait_event(eu)
            b.run(items, self.comp.cuda_stream)
            er.record(self.comp)
        for (_, _, o0, o1), er in zip(self.ranges, self.ev_run):
            self.down.wait_event(er)
            with torch.cuda.stream(self.down):
                a.h_out[o0:o1].copy_(a.d_out[o0:o1], non_blocking=True)
        self.down.synchronize()

    def close(self) -> None:
        for b in self.batches:
            b.close()


def run_plain_native(items: Sequence[BatchItem], stream: int = 0) -> None:
    """The same work with one single-texture device entry point call per texture,
    issued by the library's own C++ loop (``qt_batch_run_plain``): the launch model
    the batch replaces, with no interpreter in the loop."""
    L = _lib()
    arr = (BatchItem * len(items))(*items)
    capi.check(L.qt_batch_run_plain(arr, len(items), ctypes.c_void_p(stream)))


def run_plain(items: Sequence[BatchItem], stream: int = 0) -> None:
    """The same work with one launch per texture through the single-texture
    device entry points, each called from Python (``run_plain_native`` issues the
    same calls from C++)."""
    for it in items:
        f, p = it.format, ctypes.byref(it.params)
        src, dst, w, h, s = ctypes.c_void_p(it.src), ctypes.c_void_p(it.dst), it.width, it.height, ctypes.c_void_p(stream)
        L = capi.lib()
        if it.op == QT_OP_ENCODE:
            rc = (L.qt_bc1_encode_device(src, w, h, p, dst, s) if f == 1 else
                  L.qt_bc3_encode_device(src, w, h, p, dst, s) if f == 3 else
                  L.qt_bc4_encode_device(src, w, h, it.chan0, dst, s) if f == 4 else
                  L.qt_bc5_encode_device(src, w, h, it.chan0, it.chan1, dst, s))
        else:
            rc = (L.qt_bc1_decode_device(src, w, h, it.interpolator, it.write_alpha, dst, s) if f == 1 else
                  L.qt_bc3_decode_device(src, w, h, it.interpolator, dst, s) if f == 3 else
                  L.qt_bc4_decode_device(src, w, h, it.chan0, dst, s) if f == 4 else
                  L.qt_bc5_decode_device(src, w, h, it.chan0, it.chan1, dst, s))
        capi.check(rc)


def run_plain_host(arena: "Arena") -> None:
    """Every texture through its own host-buffer C-ABI call (upload, launch,
    download and wait per texture): the per-texture launch model end to end."""
    L = capi.lib()
    hi, ho = arena.h_in.data_ptr(), arena.h_out.data_ptr()
    for j, a, b in zip(arena.jobs, arena.in_off, arena.out_off):
        src, dst, w, h = ctypes.c_void_p(hi + a), ctypes.c_void_p(ho + b), j.width, j.height
        if j.op == QT_OP_ENCODE:
            p = ctypes.byref(j.params) if j.params is not None else None
            rc = (L.qt_bc1_encode_host(src, w, h, p, dst) if j.fmt == 1 else
                  L.qt_bc3_encode_host(src, w, h, p, dst) if j.fmt == 3 else
                  L.qt_bc4_encode_host(src, w, h, j.chan0, dst) if j.fmt == 4 else
                  L.qt_bc5_encode_host(src, w, h, j.chan0, j.chan1, dst))
        else:
            rc = (L.qt_bc1_decode_host(src, w, h, j.interpolator, int(j.write_alpha), dst) if j.fmt == 1 else
                  L.qt_bc3_decode_host(src, w, h, j.interpolator, dst) if j.fmt == 3 else
                  L.qt_bc4_decode_host(src, w, h, j.chan0, dst) if j.fmt == 4 else
                  L.qt_bc5_decode_host(src, w, h, j.chan0, j.chan1, dst))
        capi.check(rc)


def run_jobs(jobs: Sequence[Job], device: int = 0, batch: Optional[Batch] = None) -> list[bytes]:
    """Upload, one persistent launch, download; returns each job's output bytes."""
    import torch

    torch.cuda.set_device(device)
    arena = Arena(jobs, device)
    stream = torch.cuda.current_stream()
    arena.upload()
    own = batch is None
    b = batch or Batch(device)
    try:
        b.run(arena.items(), stream.cuda_stream)
        arena.download()
        stream.synchronize()
    finally:
        if own:
            b.close()
    return arena.outputs()
