"""GPU: the batched persistent path returns, for every texture of a mixed
batch, exactly the bytes of the single-texture entry points (and of the
oracle): formats BC1/BC3/BC4/BC5, encode and decode, levels 0..19, all colour
modes and interpolators, sizes 1..300 including non-multiples of 4."""

import numpy as np
import pytest

import workloads as syn
from oracle import BC1Params
from quicktex_b200 import capi
from quicktex_b200.batch import Batch, Job, run_jobs, run_plain, run_plain_native, Arena

pytestmark = pytest.mark.gpu


def make_jobs(seed: int, n: int):
    rng = np.random.default_rng(seed)
    pool = syn.alpha_mix(320, 320, workload=9, stream=seed)
    jobs, refs = [], []
    for i in range(n):
        w, h = int(rng.integers(1, 300)), int(rng.integers(1, 300))
        if rng.random() < 0.3:
            w, h = int(rng.integers(1, 9)), int(rng.integers(1, 9))
        fmt = ["bc1", "bc3", "bc4", "bc5"][int(rng.integers(0, 4))]
        y0, x0 = int(rng.integers(0, 320 - h + 1)), int(rng.integers(0, 320 - w + 1))
        img = np.ascontiguousarray(pool[y0:y0 + h, x0:x0 + w])
        if rng.random() < 0.3:  # decode job of random block bytes
            nb = ((w + 3) // 4) * ((h + 3) // 4) * (16 if fmt in ("bc3", "bc5") else 8)
            blocks = rng.integers(0, 256, nb, dtype=np.uint8)
            it, wa = int(rng.integers(0, 4)), bool(rng.integers(0, 2))
            ch, c0, c1 = int(rng.integers(0, 4)), int(rng.integers(0, 4)), int(rng.integers(0, 4))
            jobs.append(Job.decode(fmt, blocks, w, h, interpolator=it, write_alpha=wa, channel=ch, chan0=c0, chan1=c1))
            refs.append(("decode", fmt, blocks, w, h, it, wa, ch, c0, c1))
        else:
            level = int(rng.choice([0, 1, 5, 9, 10, 14, 18, 19]))
            mode = int(rng.choice([0x04, 0x03, 0x13]))
            it = int(rng.integers(0, 4))
            ch, c0, c1 = int(rng.integers(0, 4)), int(rng.integers(0, 4)), int(rng.integers(0, 4))
            jobs.append(Job.encode(fmt, img, w, h, level=level, color_mode=mode, interpolator=it, channel=ch, chan0=c0, chan1=c1))
            refs.append(("encode", fmt, img, w, h, level, mode, it, ch, c0, c1))
    return jobs, refs


def single(ref):
    if ref[0] == "decode":
        _, fmt, blocks, w, h, it, wa, ch, c0, c1 = ref
        return {"bc1": lambda: capi.bc1_decode(blocks, w, h, it, wa), "bc3": lambda: capi.bc3_decode(blocks, w, h, it),
                "bc4": lambda: capi.bc4_decode(blocks, w, h, ch), "bc5": lambda: capi.bc5_decode(blocks, w, h, c0, c1)}[fmt]()
    _, fmt, img, w, h, level, mode, it, ch, c0, c1 = ref
    return {"bc1": lambda: capi.bc1_encode(img, w, h, capi.params_for_level(level, mode, it)),
            "bc3": lambda: capi.bc3_encode(img, w, h, capi.params_for_level(level, capi.FOUR_COLOR, it)),
            "bc4": lambda: capi.bc4_encode(img, w, h, ch), "bc5": lambda: capi.bc5_encode(img, w, h, c0, c1)}[fmt]()


def test_batch_matches_single_texture_calls():
    jobs, refs = make_jobs(1, 80)
    outs = run_jobs(jobs)
    for i, (o, r) in enumerate(zip(outs, refs)):
        assert o == single(r), (i, r[:2], r[3:5])


def test_batch_matches_oracle(oracle_lib):
    jobs, refs = make_jobs(2, 40)
    outs = run_jobs(jobs)
    for o, r in zip(outs, refs):
        if r[0] != "encode" or r[1] != "bc1":
            continue
        _, fmt, img, w, h, level, mode, it, *_ = r
        assert o == oracle_lib.bc1_encode(img, w, h, BC1Params(level=level, color_mode=mode, interpolator=it))


def test_graph_replay_growth_and_plain_path():
    import torch

    b = Batch(0)
    for seed, n in ((3, 5), (4, 120), (5, 30)):  # the queue grows (re-capture) and shrinks
        jobs, refs = make_jobs(seed, n)
        arena = Arena(jobs)
        arena.upload()
        s = torch.cuda.current_stream()
        b.run(arena.items(), s.cuda_stream)
        assert b.last_tiles() >= n
        arena.download()
        s.synchronize()
        batched = arena.outputs()
        arena.d_out.zero_()
        run_plain(arena.items(), s.cuda_stream)
        arena.download()
        s.synchronize()
        assert arena.outputs() == batched
        arena.d_out.fill_(0xA5)
        run_plain_native(arena.items(), s.cuda_stream)  # the same calls from the library's C++ loop
        arena.download()
        s.synchronize()
        assert arena.outputs() == batched
        for o, r in zip(batched, refs):
            assert o == single(r)
    b.close()


def test_batch_tuning_rules_keep_results():
    jobs, refs = make_jobs(6, 25)
    ref_out = run_jobs(jobs)
    b = Batch(0, use_default_tuning=False)
    b.set_rules([{"op": 0, "format": f, "level": -1, "tile_blocks": t, "cost_per_block": 1.0}
                 for f in (1, 3, 4, 5) for t in (3,)] + [{"op": 1, "format": f, "tile_blocks": 7, "cost_per_block": 0.5} for f in (1, 3, 4, 5)])
    b.set_grid(1)
    assert run_jobs(jobs, batch=b) == ref_out
    b.close()


def test_batch_rejects_bad_items():
    b = Batch(0)
    it = Job.encode("bc4", np.zeros(64, np.uint8), 4, 4).item(0, 0)
    with pytest.raises(capi.QtError):
        b.run([it])
    b.close()


def test_reserve_and_record_arrays():
    """A reserved queue runs batches within its size without reallocating, and
    items given as an ITEM_DTYPE array run exactly like BatchItem lists."""
    import torch

    from quicktex_b200.batch import items_array

    jobs, refs = make_jobs(7, 60)
    b = Batch(0)
    b.reserve(4096, 1 << 16)
    b.reserve(16, 16)  # never shrinks
    arena = Arena(jobs)
    arena.upload()
    s = torch.cuda.current_stream()
    arr = items_array(jobs, [it.src for it in arena.items()], [it.dst for it in arena.items()])
    b.run(arr, s.cuda_stream)
    arena.download()
    s.synchronize()
    for o, r in zip(arena.outputs(), refs):
        assert o == single(r)
    b.close()


def test_copy_async_round_trip():
    import torch

    from quicktex_b200.batch import copy_async

    rng = np.random.default_rng(11)
    sizes = [1, 7, 256, 4096, 100_003, 0]
    h_in = torch.empty(sum(sizes) + 4096, dtype=torch.uint8).pin_memory()
    h_out = torch.zeros_like(h_in).pin_memory()
    h_in.numpy()[:] = rng.integers(0, 256, h_in.numel(), dtype=np.uint8)
    d = torch.empty(h_in.numel(), dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream()
    rows, o = [], 0
    for n in sizes:
        rows.append([d.data_ptr() + o, h_in.data_ptr() + o, n])
        o += n
    copy_async(np.array(rows, np.uint64), s.cuda_stream)
    copy_async(np.array([[h_out.data_ptr(), d.data_ptr(), o]], np.uint64), s.cuda_stream)
    s.synchronize()
    assert np.array_equal(h_out.numpy()[:o], h_in.numpy()[:o])


def test_pipelined_round_trip_matches_one_launch():
    """PipelinedRun (chunks with their own queues, copies overlapping launches) gives every
    texture's bytes of a single persistent launch, on two runs in a row."""
    from quicktex_b200.batch import PipelinedRun

    jobs, refs = make_jobs(7, 90)
    ref_out = run_jobs(jobs)
    arena = Arena(jobs)
    pipe = PipelinedRun(arena, chunks=3)
    try:
        for _ in range(2):
            arena.h_out.fill_(0xA5)
            pipe.run()
            assert arena.outputs() == ref_out
    finally:
        pipe.close()
