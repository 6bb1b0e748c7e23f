"""GPU: qt_batch_run_noalloc, the batched path for callers that may not
allocate device memory when they encode (engines with a fixed device budget,
latency-critical loops that cannot take cudaMalloc's synchronisation).

Called through the C-ABI, it must give the same bytes as the allocating
entry point qt_batch_run and as the oracle (bit-exact, the tolerance of every
test here) on two calls in a row with different work; with exactly its item
limit; with more tiles than its fixed queue holds, so that it coarsens them;
and it must refuse requests beyond its fixed size or with invalid textures.
Every output buffer starts filled with a sentinel, so a block or texel the
call skipped cannot pass by matching stale bytes.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

import workloads as syn
from oracle import BC1Params
from quicktex_b200 import capi
from quicktex_b200.batch import Arena, BatchItem, Job, run_jobs

pytestmark = pytest.mark.gpu

MAX_ITEMS, MAX_TILES = 1024, 16384  # QT_NOALLOC_MAX_ITEMS, QT_NOALLOC_MAX_TILES
SENTINEL = 0xA5


def _lib():
    lib = capi.lib()
    lib.qt_batch_run_noalloc.argtypes = [ctypes.POINTER(BatchItem), ctypes.c_size_t, ctypes.c_void_p]
    lib.qt_batch_run_noalloc.restype = ctypes.c_int
    return lib


def _jobs(seed: int, n: int, max_side: int = 150):
    """Mixed encode/decode jobs with their oracle specs."""
    rng = np.random.default_rng(seed)
    pool = syn.alpha_mix(max_side + 10, max_side + 10, workload=9, stream=20 + seed)
    jobs, specs = [], []
    for _ in range(n):
        w, h = int(rng.integers(1, max_side)), int(rng.integers(1, max_side))
        fmt = ["bc1", "bc3", "bc4", "bc5"][int(rng.integers(0, 4))]
        img = np.ascontiguousarray(pool[:h, :w])
        if rng.random() < 0.25:
            nb = ((w + 3) // 4) * ((h + 3) // 4) * (16 if fmt in ("bc3", "bc5") else 8)
            blocks = rng.integers(0, 256, nb, dtype=np.uint8)
            it, wa, ch = int(rng.integers(0, 4)), bool(rng.integers(0, 2)), int(rng.integers(0, 4))
            jobs.append(Job.decode(fmt, blocks, w, h, interpolator=it, write_alpha=wa, channel=ch, chan0=1, chan1=3))
            specs.append(("decode", fmt, blocks, w, h, it, wa, ch))
        else:
            level, mode = int(rng.choice([0, 5, 10, 18])), int(rng.choice([0x04, 0x03, 0x13]))
            it, ch = int(rng.integers(0, 4)), int(rng.integers(0, 4))
            jobs.append(Job.encode(fmt, img, w, h, level=level, color_mode=mode, interpolator=it, channel=ch,
                                   chan0=1, chan1=3))
            specs.append(("encode", fmt, img, w, h, level, mode, it, ch))
    return jobs, specs


def _oracle(orc, spec) -> bytes:
    if spec[0] == "decode":
        _, fmt, blocks, w, h, it, wa, ch = spec
        return {"bc1": lambda: orc.bc1_decode(blocks, w, h, it, wa), "bc3": lambda: orc.bc3_decode(blocks, w, h, it),
                "bc4": lambda: orc.bc4_decode(blocks, w, h, ch), "bc5": lambda: orc.bc5_decode(blocks, w, h, 1, 3)}[fmt]()
    _, fmt, img, w, h, level, mode, it, ch = spec
    return {"bc1": lambda: orc.bc1_encode(img, w, h, BC1Params(level=level, color_mode=mode, interpolator=it)),
            "bc3": lambda: orc.bc3_encode(img, w, h, BC1Params(level=level, interpolator=it)),
            "bc4": lambda: orc.bc4_encode(img, w, h, ch), "bc5": lambda: orc.bc5_encode(img, w, h, 1, 3)}[fmt]()


def _run_noalloc(jobs):
    import torch

    arena = Arena(jobs)
    arena.upload()
    arena.d_out.fill_(SENTINEL)
    items = arena.items()
    arr = (BatchItem * len(items))(*items)
    stream = torch.cuda.current_stream()
    capi.check(_lib().qt_batch_run_noalloc(arr, len(items), ctypes.c_void_p(stream.cuda_stream)))
    arena.download()
    stream.synchronize()
    return arena.outputs()


def _check(jobs, specs, orc, outs=None):
    outs = _run_noalloc(jobs) if outs is None else outs
    assert outs == run_jobs(jobs)
    for k, (o, s) in enumerate(zip(outs, specs)):
        assert bytes(o) == bytes(_oracle(orc, s)), (k, s[:2], s[3:5])


def test_noalloc_matches_qt_batch_run_and_oracle_on_two_calls(oracle_lib):
    for seed, n in ((11, 40), (12, 25)):  # two calls in a row, different work each time
        jobs, specs = _jobs(seed, n)
        _check(jobs, specs, oracle_lib)


def test_noalloc_at_its_item_limit(oracle_lib):
    jobs, specs = _jobs(13, MAX_ITEMS, max_side=24)
    _check(jobs, specs, oracle_lib)


def test_noalloc_coarsens_tiles_beyond_its_queue(oracle_lib):
    # nine 1024x1024 BC1 level-13 textures: 65,536 blocks each in 32-block tiles (EndpointSearch
    # settings) = 18,432 tiles, more than the fixed queue's 16,384, so the call coarsens them
    side, n = 1024, 9
    jobs, specs = [], []
    for k in range(n):
        img = syn.block_mix(side, side, workload=9, stream=40 + k)
        mode, it = (0x04, 0x03, 0x13)[k % 3], k % 4
        jobs.append(Job.encode("bc1", img, side, side, level=13, color_mode=mode, interpolator=it))
        specs.append(("encode", "bc1", img, side, side, 13, mode, it, 0))
    assert n * (side // 4) ** 2 // 32 > MAX_TILES
    _check(jobs, specs, oracle_lib)


def test_noalloc_rejects_more_items_than_its_limit():
    lib = _lib()
    n = MAX_ITEMS + 1
    arr = (BatchItem * n)()
    rc = lib.qt_batch_run_noalloc(arr, n, None)
    assert rc == capi.QT_ERR_ARG
    assert b"1024" in lib.qt_last_error()


def test_noalloc_rejects_invalid_and_oversized_textures():
    """Checked on the host before any size is used or anything is uploaded:
    the buffers below are never dereferenced."""
    lib = _lib()
    good = Job.encode("bc4", np.zeros(64, np.uint8), 4, 4).item(256, 256)
    for w, h, msg in ((-4, 8, b"width"), (8, 0, b"height"), (1 << 18, 1 << 18, b"too large")):
        bad = Job.encode("bc4", np.zeros(64, np.uint8), 4, 4).item(256, 256)
        bad.width, bad.height = w, h
        arr = (BatchItem * 2)(good, bad)
        assert lib.qt_batch_run_noalloc(arr, 2, None) == capi.QT_ERR_ARG
        assert msg in lib.qt_last_error()
