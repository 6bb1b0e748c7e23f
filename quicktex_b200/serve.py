"""Serving: continuous batching of encode/decode requests on one GPU.

``Server`` is the Python face of the native serving loop ``qt_server_*``
(csrc/qt_server.cpp); the loop itself runs on a C++ worker thread, outside the
interpreter lock:

* **Admission by memory budget.** Request payloads and results live in one
  device arena of ``memory_budget`` bytes (first fit). A waiting request joins
  a batch only when its bytes fit the largest free range; otherwise it waits
  until a running batch returns its memory. A request larger than the whole
  budget fails at once with ``MemoryError``.
* **Continuous batching.** ``slots`` batches can be in flight at once, each on
  its own CUDA stream with its own ``qt_batch`` queue (sized up front for
  ``max_batch_blocks`` / ``max_batch_requests``, so it never reallocates).
  Whenever a slot is free the worker folds the waiting requests, in arrival
  order, into the next persistent launch: requests that arrive while others
  run are admitted as soon as a slot and memory free up, and their work
  overlaps on the device with the batches still running.
* **Copies.** Each payload is uploaded from, and each result downloaded into,
  host memory by one asynchronous copy on the batch's stream. Give a request a
  pinned response buffer (``out=``) and its result lands there with no further
  copy; without one, the future resolves to ``bytes``.

The integer block output does not depend on what else is in a batch: every
request's bytes equal those of the single-texture call (tests check this).
"""

from __future__ import annotations

import concurrent.futures
import ctypes
import threading
import time
from typing import Optional, Sequence

import numpy as np

from . import capi
from .batch import BatchItem, Job, TileRule, items_array, load_tuning


class _Stats(ctypes.Structure):
    """``qt_server_stats``."""

    _fields_ = [("batches", ctypes.c_uint64), ("requests_done", ctypes.c_uint64), ("blocks_done", ctypes.c_uint64),
                ("max_inflight", ctypes.c_uint32), ("pending", ctypes.c_uint32), ("inflight", ctypes.c_uint32),
                ("slots", ctypes.c_uint32)]


_sigs_done = False


def _lib():
    global _sigs_done
    L = capi.lib()
    if not _sigs_done:
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L.qt_server_create.argtypes = [ctypes.c_int, sz, ctypes.c_int, sz, sz, ctypes.POINTER(vp)]
        L.qt_server_destroy.argtypes = [vp]
        L.qt_server_set_rules.argtypes = [vp, ctypes.POINTER(TileRule), sz]
        L.qt_server_set_grid.argtypes = [vp, ctypes.c_int]
        L.qt_server_set_threads.argtypes = [vp, ctypes.c_int]
        L.qt_server_submit.argtypes = [vp, ctypes.POINTER(BatchItem), vp, sz]
        L.qt_server_poll.argtypes = [vp, vp, vp, vp, sz, ctypes.c_int64, ctypes.POINTER(sz)]
        L.qt_server_get_stats.argtypes = [vp, ctypes.POINTER(_Stats)]
        L.qt_server_clock.argtypes = []
        L.qt_server_clock.restype = ctypes.c_double
        for n in ("qt_server_create", "qt_server_destroy", "qt_server_set_rules", "qt_server_set_grid", "qt_server_set_threads",
                  "qt_server_submit", "qt_server_poll", "qt_server_get_stats"):
            getattr(L, n).restype = ctypes.c_int
        _sigs_done = True
    return L


class _PinnedPool:
    """First-fit allocator over one pinned host buffer: the response buffers of
    requests submitted without ``out`` (a download into pageable memory would
    make the batch's copies synchronous)."""

    ALIGN = 256

    def __init__(self, nbytes: int):
        import torch

        self.buf = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
        self.np = self.buf.numpy()
        self.free = [(0, nbytes)]  # sorted (offset, length)
        self.lock = threading.Lock()

    def take(self, n: int):
        n = (n + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        with self.lock:
            for i, (off, ln) in enumerate(self.free):
                if ln >= n:
                    self.free[i:i + 1] = [] if ln == n else [(off + n, ln - n)]
                    return off, n
        return None

    def give(self, off: int, n: int) -> None:
        with self.lock:
            fl = sorted(self.free + [(off, n)])
            merged = [fl[0]]
            for o, ln in fl[1:]:
                if merged[-1][0] + merged[-1][1] == o:
                    merged[-1] = (merged[-1][0], merged[-1][1] + ln)
                else:
                    merged.append((o, ln))
            self.free = merged


class Request:
    __slots__ = ("job", "future", "t_arrival", "t_done", "out", "buf", "pooled")

    def __init__(self, job: Job, t_arrival: float, out: Optional[np.ndarray] = None, pool: Optional[_PinnedPool] = None):
        if out is not None and (out.dtype != np.uint8 or out.nbytes < job.out_bytes or not out.flags.c_contiguous
                                or not out.flags.writeable):
            raise ValueError(f"out must be a writable contiguous uint8 array of at least {job.out_bytes} bytes")
        self.job = job
        self.future = concurrent.futures.Future()
        self.future.request = self
        self.t_arrival = t_arrival
        self.t_done = None
        self.out = out
        self.pooled = None
        if out is not None:
            self.buf = out
        else:
            got = pool.take(job.out_bytes) if pool is not None else None
            if got is not None:
                self.pooled = got
                self.buf = pool.np[got[0]: got[0] + job.out_bytes]
            else:  # pool full: a pageable buffer (correct, but its download is synchronous)
                self.buf = np.empty(job.out_bytes, np.uint8)

    def result(self):
        n = self.job.out_bytes
        return self.buf[:n].tobytes() if self.out is None else self.out[:n]


class Server:
    """Continuous-batching encode/decode server on one GPU."""

    def __init__(self, device: int = 0, memory_budget: int = 16 << 30, slots: int = 3,
                 max_batch_blocks: int = 1 << 22, max_batch_requests: int = 8192, tuning=None,
                 response_pool_bytes: int = 256 << 20):
        L = _lib()
        self._pool_bytes = response_pool_bytes
        self._pool: Optional[_PinnedPool] = None  # pinned on first use
        h = ctypes.c_void_p()
        capi.check(L.qt_server_create(device, memory_budget, slots, max_batch_blocks, max_batch_requests,
                                      ctypes.byref(h)))
        self.handle = h
        self.device = device
        tuning = load_tuning() if tuning is None else tuning
        if tuning:
            rules = tuning.get("rules", [])
            arr = (TileRule * max(1, len(rules)))()
            for i, r in enumerate(rules):
                arr[i] = TileRule(r["op"], r["format"], r.get("level", -1), r["tile_blocks"], r["cost_per_block"])
            capi.check(L.qt_server_set_rules(h, arr, len(rules)))
            if tuning.get("threads_per_cta"):
                capi.check(L.qt_server_set_threads(h, int(tuning["threads_per_cta"])))
            if tuning.get("ctas_per_sm"):
                capi.check(L.qt_server_set_grid(h, int(tuning["ctas_per_sm"])))
        # completion times come on CLOCK_MONOTONIC; latencies are measured against time.perf_counter
        self._clock_offset = time.perf_counter() - L.qt_server_clock()
        self._lock = threading.Lock()
        self._inflight: dict[int, Request] = {}
        self._next_tag = 1
        self._closing = False
        self._poller = threading.Thread(target=self._poll_loop, name="quicktex-serve-poll", daemon=True)
        self._poller.start()

    # ---- client side --------------------------------------------------------
    def submit(self, job: Job, t_arrival: Optional[float] = None, out: Optional[np.ndarray] = None
               ) -> concurrent.futures.Future:
        """Queue a request. ``t_arrival`` (perf_counter seconds) defaults to now;
        latency is measured from it. Without ``out`` the future resolves to the
        output as ``bytes``; with ``out`` (a uint8 array, pinned for an
        asynchronous copy) the result is copied from the device straight into it
        and the future resolves to ``out[:job.out_bytes]``. The job's payload and
        ``out`` must not change until the future is done."""
        return self.submit_many([job], [t_arrival], [out])[0]

    def submit_many(self, jobs: Sequence[Job], t_arrivals=None, outs=None) -> list:
        """``submit`` for several requests in one native call."""
        n = len(jobs)
        if n == 0:
            return []
        now = time.perf_counter()
        t_arrivals = [now] * n if t_arrivals is None else [now if t is None else t for t in t_arrivals]
        outs = [None] * n if outs is None else outs
        if self._pool is None and self._pool_bytes > 0 and any(o is None for o in outs):
            self._pool = _PinnedPool(self._pool_bytes)
        reqs = [Request(j, t, o, self._pool) for j, t, o in zip(jobs, t_arrivals, outs)]
        items = items_array(jobs, [j.data.ctypes.data for j in jobs], [r.buf.ctypes.data for r in reqs])
        with self._lock:
            if self._closing:
                raise RuntimeError("the server is closed")
            t0 = self._next_tag
            self._next_tag += n
            for k, r in enumerate(reqs):
                self._inflight[t0 + k] = r
        tags = np.arange(t0, t0 + n, dtype=np.uint64)
        rc = _lib().qt_server_submit(self.handle, ctypes.cast(items.ctypes.data, ctypes.POINTER(BatchItem)),
                                     tags.ctypes.data, n)
        if rc:
            with self._lock:
                for k in range(n):
                    self._inflight.pop(t0 + k, None)
            capi.check(rc)
        return [r.future for r in reqs]

    def close(self) -> None:
        """Finish every submitted request, then release the server."""
        if self.handle is None:
            return
        with self._lock:
            self._closing = True
        self._poller.join()
        self._final_stats = self.stats()
        _lib().qt_server_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- statistics -------------------------------------------------------------
    def stats(self) -> dict:
        """Batches launched, requests and blocks done, most batches in flight at once, ... (kept after close)."""
        if self.handle is None:
            return dict(self._final_stats)
        s = _Stats()
        capi.check(_lib().qt_server_get_stats(self.handle, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _Stats._fields_}

    @property
    def batches(self) -> int:
        return self.stats()["batches"]

    @property
    def blocks_done(self) -> int:
        return self.stats()["blocks_done"]

    @property
    def max_inflight_seen(self) -> int:
        return self.stats()["max_inflight"]

    # ---- completions ----------------------------------------------------------------
    def _poll_loop(self) -> None:
        L = _lib()
        cap = 4096
        tags, status, t_done = np.empty(cap, np.uint64), np.empty(cap, np.int32), np.empty(cap, np.float64)
        got = ctypes.c_size_t()
        while True:
            capi.check(L.qt_server_poll(self.handle, tags.ctypes.data, status.ctypes.data, t_done.ctypes.data, cap,
                                        20_000, ctypes.byref(got)))
            k = got.value
            if k:
                tl, sl, dl = tags[:k].tolist(), status[:k].tolist(), t_done[:k].tolist()
                with self._lock:
                    rs = [self._inflight.pop(t) for t in tl]
                for r, s, t in zip(rs, sl, dl):
                    r.t_done = t + self._clock_offset
                    res = r.result() if s == capi.QT_OK else None
                    if r.pooled is not None:  # result copied out (or failed): the pinned range is free again
                        self._pool.give(*r.pooled)
                        r.pooled, r.buf = None, None
                    if s == capi.QT_OK:
                        r.future.set_result(res)
                    elif s == capi.QT_ERR_RANGE:
                        r.future.set_exception(MemoryError("request exceeds the server's memory budget"))
                    else:
                        r.future.set_exception(capi.QtError(s, "request failed on the device"))
                continue
            with self._lock:
                if self._closing and not self._inflight:
                    return


def latency_stats(futures) -> dict:
    lat = np.array([(f.request.t_done - f.request.t_arrival) * 1e3 for f in futures])
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "requests": int(len(lat))}
