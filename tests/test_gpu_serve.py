"""GPU: the continuous-batching server. Every request's result is the same
alone and in the mix; requests are folded into shared launches, batches
overlap on the device, and the memory budget admits requests as memory frees."""

import time

import numpy as np
import pytest

import workloads as syn
from quicktex_b200.batch import Job, run_jobs
from quicktex_b200.serve import Server, latency_stats

pytestmark = pytest.mark.gpu


def _jobs(seed, n, max_side=200):
    rng = np.random.default_rng(seed)
    pool = syn.alpha_mix(max_side, max_side, workload=9, stream=40 + seed)
    jobs = []
    for _ in range(n):
        w, h = int(rng.integers(1, max_side)), int(rng.integers(1, max_side))
        fmt = ["bc1", "bc3", "bc4", "bc5"][int(rng.integers(0, 4))]
        img = np.ascontiguousarray(pool[:h, :w])
        if rng.random() < 0.3:
            nb = ((w + 3) // 4) * ((h + 3) // 4) * (16 if fmt in ("bc3", "bc5") else 8)
            jobs.append(Job.decode(fmt, rng.integers(0, 256, nb, dtype=np.uint8), w, h, interpolator=int(rng.integers(0, 4))))
        else:
            jobs.append(Job.encode(fmt, img, w, h, level=int(rng.choice([0, 5, 10, 18])),
                                   color_mode=int(rng.choice([4, 3, 0x13])), interpolator=int(rng.integers(0, 4)), channel=0))
    return jobs


def test_results_same_alone_and_in_the_mix():
    jobs = _jobs(1, 120)
    alone = [run_jobs([j])[0] for j in jobs]
    srv = Server(memory_budget=8 << 20, slots=3, max_batch_blocks=4096)
    # all at once: the worker fills the free slots back to back, so batches overlap
    futs = srv.submit_many(jobs[:100]) + [srv.submit(j) for j in jobs[100:]]
    outs = [f.result(timeout=120) for f in futs]
    srv.close()
    assert outs == alone
    assert srv.batches < len(jobs)        # requests were folded into shared launches
    assert srv.max_inflight_seen >= 2     # batches overlapped on the device
    st = latency_stats(futs)
    assert st["requests"] == len(jobs) and st["p99_ms"] >= st["p50_ms"] > 0


def test_budget_admission_and_oversize_request():
    jobs = _jobs(2, 40, max_side=128)
    # a budget that holds only a few requests at a time: the rest wait for memory to free up
    srv = Server(memory_budget=1 << 20, slots=2)
    futs = [srv.submit(j) for j in jobs]
    big = Job.encode("bc1", np.zeros((1024, 1024, 4), np.uint8), 1024, 1024)  # 4 MiB + blocks > 1 MiB budget
    fbig = srv.submit(big)
    outs = [f.result(timeout=120) for f in futs]
    with pytest.raises(MemoryError):
        fbig.result(timeout=120)
    srv.close()
    assert outs == run_jobs(jobs)


def test_requests_arriving_while_busy_are_admitted():
    jobs = _jobs(3, 60)
    srv = Server(memory_budget=64 << 20, slots=2, max_batch_blocks=2048)
    futs = []
    for i, j in enumerate(jobs):  # a steady trickle while earlier batches run
        futs.append(srv.submit(j))
        if i % 10 == 9:
            time.sleep(0.002)
    outs = [f.result(timeout=120) for f in futs]
    srv.close()
    assert outs == run_jobs(jobs)
    assert srv.batches >= 2


def test_results_into_caller_buffers():
    """Requests with a response buffer (pinned or pageable) get the same bytes
    written straight into it; requests without one still get bytes."""
    import torch

    jobs = _jobs(4, 50)
    ref = run_jobs(jobs)
    pinned = torch.empty(sum(j.out_bytes + 256 for j in jobs), dtype=torch.uint8).pin_memory().numpy()
    outs, o = [], 0
    for k, j in enumerate(jobs):
        if k % 3 == 0:
            outs.append(None)
        elif k % 3 == 1:
            outs.append(pinned[o:o + j.out_bytes + 256])
            o += j.out_bytes + 256
        else:
            outs.append(np.empty(j.out_bytes, np.uint8))
    srv = Server(memory_budget=64 << 20, slots=2, max_batch_blocks=8192)
    futs = srv.submit_many(jobs, [time.perf_counter()] * len(jobs), outs)
    got = [f.result(timeout=120) for f in futs]
    srv.close()
    for g, r, out in zip(got, ref, outs):
        if out is None:
            assert isinstance(g, bytes) and g == r
        else:
            assert g.base is out or g is out or np.shares_memory(g, out)
            assert g.tobytes() == r
    with pytest.raises(ValueError):
        Server.submit(srv, jobs[0], out=np.empty(1, np.uint8))
