"""Serving: continuous batching of encode/decode requests on one GPU.

A ``Server`` accepts requests at any time (``submit`` returns a future) and
runs them through the batched persistent path:

* **Admission by memory budget.** Input and output buffers come from one
  pre-reserved device arena (``memory_budget`` bytes, first-fit free list). A
  request is admitted into a batch only when its bytes fit; otherwise it waits
  until a running batch returns its memory.
* **Continuous batching.** ``slots`` batches can be in flight at once, each on
  its own CUDA stream with its own ``qt_batch`` queue. Whenever a slot is free
  the worker folds every waiting request that fits (up to ``max_batch_blocks``)
  into the next persistent launch, so requests that arrive while others run on
  the GPU are admitted as soon as a slot and memory free up, and their work
  overlaps on the device with the batches still running.
* **Resident buffers.** Nothing is allocated per request: device memory is
  carved from the arena, each slot's queue is sized for the largest batch at
  start-up (``qt_batch_reserve``), and the download buffer is pinned and reused.
  Request payloads are copied straight from the caller's buffers (pinned for
  asynchronous copies) by ``qt_copy_async``, one call per batch.

The integer block output does not depend on what else is in a batch: every
request's bytes equal those of the single-texture call (tests check this).
"""

from __future__ import annotations

import collections
import concurrent.futures
import threading
import time
from typing import Optional

import numpy as np

from .batch import Batch, Job, copy_async, items_array


def _event(stream):
    import torch

    e = torch.cuda.Event()
    e.record(stream)
    return e


class DeviceArena:
    """First-fit free list over one device buffer (the memory budget)."""

    ALIGN = 256

    def __init__(self, nbytes: int, device: int):
        import torch

        self.buf = torch.empty(nbytes, dtype=torch.uint8, device=torch.device("cuda", device))
        self.base = self.buf.data_ptr()
        self.size = nbytes
        self.free = [(0, nbytes)]  # sorted (offset, length)
        self.in_use = 0

    def alloc(self, n: int) -> Optional[int]:
        n = (n + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        for i, (off, ln) in enumerate(self.free):
            if ln >= n:
                if ln == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (off + n, ln - n)
                self.in_use += n
                return off
        return None

    def release(self, off: int, n: int) -> None:
        n = (n + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        self.in_use -= n
        fl = self.free
        fl.append((off, n))
        fl.sort()
        merged = []
        for o, l in fl:
            if merged and merged[-1][0] + merged[-1][1] == o:
                merged[-1] = (merged[-1][0], merged[-1][1] + l)
            else:
                merged.append((o, l))
        self.free = merged


class Request:
    __slots__ = ("job", "future", "t_arrival", "t_done", "out", "out_off")

    def __init__(self, job: Job, t_arrival: float, out: Optional[np.ndarray] = None):
        if out is not None and (out.dtype != np.uint8 or out.nbytes < job.out_bytes or not out.flags.c_contiguous):
            raise ValueError(f"out must be a contiguous uint8 array of at least {job.out_bytes} bytes")
        self.job = job
        self.future = concurrent.futures.Future()
        self.t_arrival = t_arrival
        self.t_done = None
        self.out = out
        self.out_off = 0


class _Slot:
    def __init__(self, device: int, tuning=None):
        import torch

        self.stream = torch.cuda.Stream(device=device)
        self.batch = Batch(device, tuning=tuning)
        self.event = None
        self.reqs: list[Request] = []
        self.region = None  # (offset, nbytes) in the arena
        self.h_out = None  # pinned download buffer, reused
        self.h_out_np = None

    def host_out(self, n: int) -> np.ndarray:
        import torch

        if self.h_out is None or self.h_out.numel() < n:
            self.h_out = torch.empty(max(n, 1 << 20) * 2, dtype=torch.uint8).pin_memory()
            self.h_out_np = self.h_out.numpy()
        return self.h_out_np


class Server:
    """Continuous-batching encode/decode server on one GPU."""

    def __init__(self, device: int = 0, memory_budget: int = 16 << 30, slots: int = 3,
                 max_batch_blocks: int = 1 << 22, max_batch_requests: int = 8192, tuning=None):
        import torch

        torch.cuda.set_device(device)
        self.device = device
        self.arena = DeviceArena(memory_budget, device)
        self.slots = [_Slot(device, tuning) for _ in range(slots)]
        for s in self.slots:  # queues sized for the largest batch up front: no reallocation while serving
            s.batch.reserve(max_batch_requests, max_batch_blocks // 32 + max_batch_requests)
        self.max_batch_blocks = max_batch_blocks
        self.max_batch_requests = max_batch_requests
        self.pending: collections.deque[Request] = collections.deque()
        self.cv = threading.Condition()
        self.running = True
        self.batches = 0
        self.blocks_done = 0
        self.max_inflight_seen = 0
        self.worker = threading.Thread(target=self._loop, name="quicktex-serve", daemon=True)
        self.worker.start()

    # ---- client side --------------------------------------------------------
    def submit(self, job: Job, t_arrival: Optional[float] = None, out: Optional[np.ndarray] = None
               ) -> concurrent.futures.Future:
        """Queue a request. ``t_arrival`` (perf_counter seconds) defaults to now;
        latency is measured from it. Without ``out`` the future resolves to the
        output as ``bytes``; with ``out`` (a uint8 array, pinned for an
        asynchronous copy) the result is copied from the device straight into it
        and the future resolves to ``out[:job.out_bytes]``."""
        r = Request(job, time.perf_counter() if t_arrival is None else t_arrival, out)
        r.future.request = r
        with self.cv:
            self.pending.append(r)
            self.cv.notify()
        return r.future

    def submit_many(self, jobs, t_arrivals, outs=None) -> list:
        """``submit`` for several requests under one lock."""
        reqs = [Request(j, t, o) for j, t, o in zip(jobs, t_arrivals, outs if outs is not None else [None] * len(jobs))]
        for r in reqs:
            r.future.request = r
        with self.cv:
            self.pending.extend(reqs)
            self.cv.notify()
        return [r.future for r in reqs]

    def close(self) -> None:
        with self.cv:
            self.running = False
            self.cv.notify()
        self.worker.join()
        for s in self.slots:
            s.batch.close()

    # ---- worker ---------------------------------------------------------------
    def _launch(self, slot: _Slot, reqs: list[Request]) -> None:
        """One batch on ``slot``'s stream: payload uploads and result downloads
        (one copy per request each, issued from C), one persistent launch."""
        n = len(reqs)
        jobs = [r.job for r in reqs]
        in_b = np.fromiter((j.data.nbytes for j in jobs), np.int64, n)
        out_b = np.fromiter((j.out_bytes for j in jobs), np.int64, n)
        a = DeviceArena.ALIGN
        in_al, out_al = (in_b + a - 1) // a * a, (out_b + a - 1) // a * a
        in_off, out_off = np.cumsum(in_al) - in_al, np.cumsum(out_al) - out_al
        n_in, n_out = int(in_al.sum()), int(out_al.sum())
        off = self.arena.alloc(n_in + n_out)
        assert off is not None  # reserved by the caller
        base = self.arena.base + off
        src = (base + in_off).astype(np.uint64)
        dst = (base + n_in + out_off).astype(np.uint64)
        copies = np.empty((n, 3), np.uint64)
        copies[:, 0] = src
        copies[:, 1] = np.fromiter((j.data.ctypes.data for j in jobs), np.uint64, n)
        copies[:, 2] = in_b
        stream = slot.stream.cuda_stream
        copy_async(copies, stream)
        slot.batch.run(items_array(jobs, src, dst), stream)
        # results: into the request's own buffer, else into the slot's pinned buffer
        host = slot.host_out(n_out)
        hbase = host.ctypes.data
        copies[:, 1] = dst
        copies[:, 2] = out_b
        for k, (r, o) in enumerate(zip(reqs, out_off.tolist())):
            r.out_off = o
            copies[k, 0] = hbase + o if r.out is None else r.out.ctypes.data
        copy_async(copies, stream)
        slot.event = _event(slot.stream)
        slot.reqs = reqs
        slot.region = (off, n_in + n_out)
        self.batches += 1

    def _complete(self, slot: _Slot) -> None:
        t = time.perf_counter()
        host = slot.h_out_np
        for r in slot.reqs:
            n = r.job.out_bytes
            out = host[r.out_off: r.out_off + n].tobytes() if r.out is None else r.out[:n]
            r.t_done = t
            self.blocks_done += r.job.nblocks
            r.future.set_result(out)
        self.arena.release(*slot.region)
        slot.reqs, slot.region, slot.event = [], None, None

    def _take(self) -> list[Request]:
        """Admit waiting requests, FIFO, while they fit in the free memory and the batch cap."""
        reqs, nbytes, blocks = [], 0, 0
        free = self.arena.size - self.arena.in_use
        largest = max((l for _, l in self.arena.free), default=0)
        while self.pending:
            r = self.pending[0]
            need = DeviceArena.ALIGN * ((r.job.data.nbytes + 255) // 256 + (r.job.out_bytes + 255) // 256)
            if reqs and (blocks + r.job.nblocks > self.max_batch_blocks or len(reqs) >= self.max_batch_requests):
                break
            if nbytes + need > min(free, largest):
                break
            reqs.append(self.pending.popleft())
            nbytes += need
            blocks += r.job.nblocks
        return reqs

    def _loop(self) -> None:
        import torch

        torch.cuda.set_device(self.device)
        while True:
            busy = [s for s in self.slots if s.event is not None]
            for s in busy:
                if s.event.query():
                    self._complete(s)
            free_slots = [s for s in self.slots if s.event is None]
            inflight = len(self.slots) - len(free_slots)
            with self.cv:
                if not self.running and not self.pending and inflight == 0:
                    return
                reqs = self._take() if (free_slots and self.pending) else []
                if not reqs and inflight == 0:
                    if self.pending and not self.arena.in_use:  # a request larger than the whole budget
                        r = self.pending.popleft()
                        r.future.set_exception(MemoryError("request exceeds the server's memory budget"))
                        continue
                    self.cv.wait(timeout=0.001)
                    continue
            if reqs:
                self._launch(free_slots[0], reqs)
                self.max_inflight_seen = max(self.max_inflight_seen, inflight + 1)
            else:
                time.sleep(20e-6)


def latency_stats(futures) -> dict:
    lat = np.array([(f.request.t_done - f.request.t_arrival) * 1e3 for f in futures])
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "requests": int(len(lat))}
