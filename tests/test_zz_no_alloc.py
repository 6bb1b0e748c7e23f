"""GPU: qt_batch_run_noalloc, the batched path for callers that may not
allocate device memory when they encode (engines with a fixed device budget,
latency-critical loops that cannot take cudaMalloc's synchronisation).

Called through the C-ABI, it must give the same bytes as the allocating
entry point qt_batch_run (bit-exact, the tolerance of every test here) on two
calls in a row with different work, and refuse requests beyond its fixed size.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

import workloads as syn
from quicktex_b200 import capi
from quicktex_b200.batch import Arena, BatchItem, Job, run_jobs

pytestmark = pytest.mark.gpu


def _jobs(seed: int, n: int):
    rng = np.random.default_rng(seed)
    pool = syn.alpha_mix(160, 160, workload=9, stream=20 + seed)
    jobs = []
    for _ in range(n):
        w, h = int(rng.integers(1, 150)), int(rng.integers(1, 150))
        fmt = ["bc1", "bc3", "bc4", "bc5"][int(rng.integers(0, 4))]
        img = np.ascontiguousarray(pool[:h, :w])
        if rng.random() < 0.25:
            nb = ((w + 3) // 4) * ((h + 3) // 4) * (16 if fmt in ("bc3", "bc5") else 8)
            jobs.append(Job.decode(fmt, rng.integers(0, 256, nb, dtype=np.uint8), w, h,
                                   interpolator=int(rng.integers(0, 4)), write_alpha=bool(rng.integers(0, 2)),
                                   channel=int(rng.integers(0, 4))))
        else:
            jobs.append(Job.encode(fmt, img, w, h, level=int(rng.choice([0, 5, 10, 18])),
                                   color_mode=int(rng.choice([0x04, 0x03, 0x13])), interpolator=int(rng.integers(0, 4)),
                                   channel=int(rng.integers(0, 4)), chan0=1, chan1=3))
    return jobs


def _run_noalloc(jobs):
    import torch

    lib = capi.lib()
    lib.qt_batch_run_noalloc.argtypes = [ctypes.POINTER(BatchItem), ctypes.c_size_t, ctypes.c_void_p]
    lib.qt_batch_run_noalloc.restype = ctypes.c_int
    arena = Arena(jobs)
    arena.upload()
    items = arena.items()
    arr = (BatchItem * len(items))(*items)
    stream = torch.cuda.current_stream()
    capi.check(lib.qt_batch_run_noalloc(arr, len(items), ctypes.c_void_p(stream.cuda_stream)))
    arena.download()
    stream.synchronize()
    return arena.outputs()


def test_noalloc_matches_qt_batch_run_on_two_calls():
    for seed, n in ((11, 40), (12, 25)):  # two calls in a row, different work each time
        jobs = _jobs(seed, n)
        assert _run_noalloc(jobs) == run_jobs(jobs)


def test_noalloc_rejects_more_items_than_its_limit():
    lib = capi.lib()
    lib.qt_batch_run_noalloc.argtypes = [ctypes.POINTER(BatchItem), ctypes.c_size_t, ctypes.c_void_p]
    lib.qt_batch_run_noalloc.restype = ctypes.c_int
    n = 1025  # QT_NOALLOC_MAX_ITEMS + 1
    arr = (BatchItem * n)()
    rc = lib.qt_batch_run_noalloc(arr, n, None)
    assert rc == capi.QT_ERR_ARG
    assert b"1024" in lib.qt_last_error()
