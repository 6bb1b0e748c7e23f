#!/usr/bin/env python3
"""Benchmark of the S3TC encode path on B200.

Workload (one "step"): BC1-encode one seeded 4096x4096 RGBA8 texture
(1,048,576 blocks; 40% gradient / 30% random / 20% two-colour edge / 10% solid
blocks) once for each of the 36 settings {level 0, 10, 18} x {four-colour,
three-colour, three-colour+black} x {Ideal, IdealRound, Nvidia, AMD}:
37.7 M blocks per step, every output bit-exact with the reference encoder
(checked by the parity tests against the committed reference hashes).

  value   Mblocks/s with the texture resident in HBM (device entry point
          qt_bc1_encode_device), L2 flushed between steps, CUDA-event timed.
  e2e     the same metric through the host-buffer entry point
          qt_bc1_encode_host from pinned host memory: every call copies the
          texture in and the blocks out.
  roofline  the BC1 encode kernels against the instruction issue rate (an
          INT32/FP32 issue-bound path, not HBM- or tensor-bound): warp
          instructions per block of each setting (ncu counts, WARP_INST_PER_BLOCK)
          x blocks / CUDA-event time, over SMs x 4 schedulers x clock. The older
          work model (10 lane-ops per oracle-counted candidate evaluation,
          tests/golden/ce_counts.json) rides along as "work_model".
  cpu_baseline  the unmodified reference encoder (oracle/_ref) on this host's
          cores, OpenMP as shipped, on a 512x512 crop of the same texture for
          each of the 36 settings.

Multi-GPU (torchrun, one process per GPU): every rank encodes its own replica
of the workload (the path shards by texture; no collective on the data path),
value = all ranks' blocks / max-over-ranks time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import collections
import gc
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BC1/BC3 encode Mblocks/s bit-exact, batched vs plain on 1 B200; serve p50/p99 ms"
LEVELS = (0, 10, 18)
MODES = (("four", 0x04), ("three", 0x03), ("three_black", 0x13))
INTERPS = (("ideal", 0), ("round", 1), ("nvidia", 2), ("amd", 3))
W = H = 4096
NB = (W // 4) * (H // 4)
SETTINGS = [(L, mn, m, iname, it) for L in LEVELS for mn, m in MODES for iname, it in INTERPS]


def configure(size: int, levels) -> None:
    """Profiling variants (--size / --levels); the default is the benchmark workload."""
    global W, H, NB, SETTINGS
    W = H = size
    NB = (W // 4) * (H // 4)
    SETTINGS = [(L, mn, m, iname, it) for L in levels for mn, m in MODES for iname, it in INTERPS]
    CONFIG["levels"] = list(levels)
    CONFIG["blocks_per_step"] = NB * len(SETTINGS)
    if size != 4096 or tuple(levels) != LEVELS:
        CONFIG["workload"] = f"bc1_encode_{size}x{size}_mix_{len(SETTINGS)}settings (profiling variant)"
CONFIG = {
    "workload": "bc1_encode_4096x4096_mix_36settings",
    "texture": "4096x4096 RGBA8, seeded block mix (40% gradient, 30% random, 20% edge, 10% solid)",
    "levels": list(LEVELS),
    "color_modes": [m for m, _ in MODES],
    "interpolators": [i for i, _ in INTERPS],
    "blocks_per_step": NB * len(SETTINGS),
    "l2": "flushed between steps (256 MiB write)",
}


# DRAM bytes per block of a level-18 encode call (split, encoder, second cluster-fit pass, search,
# finish), the setting class that holds ~80% of the step: the ncu capture summarised in
# profiles/k_bc1_L18_2048sq_pipeline.md (dram__bytes_read.sum + dram__bytes_write.sum of the five
# kernels = 92,676,096 B for 262,144 blocks). Each pass re-reads the block's texels.
BC1_DRAM_BYTES_PER_BLOCK = (16792832 + 18021376 + 2560 + 20707584 + 21565952 + 15585792) / 262144

# Warp instructions executed per block by one encode call of each setting: smsp__inst_executed.sum
# over the call's kernels divided by the texture's blocks, from the ncu launch list of the bench's
# own per-setting pass at 2048x2048 (a crop of the same texture, the same kernels: split + fast
# encoder, or the five-kernel level-18 pipeline), summarised in
# profiles/bench_2048sq_inst_per_block.md.
WARP_INST_PER_BLOCK: dict = {
    "L0_four_ideal": 121.0, "L0_four_round": 121.7, "L0_four_nvidia": 122.8, "L0_four_amd": 120.8,
    "L0_three_ideal": 188.3, "L0_three_round": 189.0, "L0_three_nvidia": 191.1, "L0_three_amd": 188.2,
    "L0_three_black_ideal": 190.1, "L0_three_black_round": 190.8, "L0_three_black_nvidia": 192.8, "L0_three_black_amd": 189.9,
    "L10_four_ideal": 443.9, "L10_four_round": 448.0, "L10_four_nvidia": 457.8, "L10_four_amd": 442.6,
    "L10_three_ideal": 593.0, "L10_three_round": 597.1, "L10_three_nvidia": 612.6, "L10_three_amd": 591.7,
    "L10_three_black_ideal": 594.8, "L10_three_black_round": 598.9, "L10_three_black_nvidia": 614.2, "L10_three_black_amd": 593.4,
    "L18_four_ideal": 3221.0, "L18_four_round": 3266.3, "L18_four_nvidia": 3678.5, "L18_four_amd": 3225.4,
    "L18_three_ideal": 3917.7, "L18_three_round": 3962.8, "L18_three_nvidia": 4511.4, "L18_three_amd": 3922.0,
    "L18_three_black_ideal": 3917.9, "L18_three_black_round": 3963.0, "L18_three_black_nvidia": 4515.0, "L18_three_black_amd": 3924.5,
}


def measure_hbm_paths(dev, stream, side: int = 16384, reps: int = 5):
    """The bandwidth-bound kernels on side^2 textures (16384^2 = 1 GiB of texels, far larger
    than L2): BC4 and BC5 encode, BC1, BC3, BC4 and BC5 decode; achieved = algorithmic bytes
    (64 B of texels + 8 or 16 B of blocks per block) / CUDA-event time."""
    import torch

    from quicktex_b200 import capi

    nb = (side // 4) ** 2
    rng = np.random.default_rng(7)
    tex = torch.from_numpy(rng.integers(0, 256, side * side * 4, dtype=np.uint8)).to(dev)
    blocks16 = torch.empty(nb * 16, dtype=torch.uint8, device=dev)
    out = torch.empty(side * side * 4, dtype=torch.uint8, device=dev)
    sptr = stream.cuda_stream
    L = capi.lib()
    cases = {
        "bc4_encode": (lambda: capi.check(L.qt_bc4_encode_device(capi._vp(tex.data_ptr()), side, side, 0, capi._vp(blocks16.data_ptr()), capi._vp(sptr))), nb * (64 + 8)),
        "bc5_encode": (lambda: capi.check(L.qt_bc5_encode_device(capi._vp(tex.data_ptr()), side, side, 0, 1, capi._vp(blocks16.data_ptr()), capi._vp(sptr))), nb * (64 + 16)),
        "bc1_decode": (lambda: capi.check(L.qt_bc1_decode_device(capi._vp(blocks16.data_ptr()), side, side, 0, 0, capi._vp(out.data_ptr()), capi._vp(sptr))), nb * (8 + 64)),
        "bc4_decode": (lambda: capi.check(L.qt_bc4_decode_device(capi._vp(blocks16.data_ptr()), side, side, 0, capi._vp(out.data_ptr()), capi._vp(sptr))), nb * (8 + 64)),
        "bc3_decode": (lambda: capi.check(L.qt_bc3_decode_device(capi._vp(blocks16.data_ptr()), side, side, 0, capi._vp(out.data_ptr()), capi._vp(sptr))), nb * (16 + 64)),
        "bc5_decode": (lambda: capi.check(L.qt_bc5_decode_device(capi._vp(blocks16.data_ptr()), side, side, 0, 1, capi._vp(out.data_ptr()), capi._vp(sptr))), nb * (16 + 64)),
    }
    res = {}
    for name, (fn, nbytes) in cases.items():
        fn()
        fn()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        ms = float(np.median(ts))
        res[name] = {"ms": ms, "gb_s": nbytes / (ms / 1e3) / 1e9, "mblocks_s": nb / (ms / 1e3) / 1e6}
    return res


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region. The sampler starts before the
    region and the region begins only after its first sample has arrived (nvidia-smi takes a
    while to start); only samples that arrive inside the region are summarised."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, period_ms: int = 100):
        self.index = index
        self.period_ms = period_ms
        self.proc = None
        self.samples = []  # (arrival time, line)

    def _reader(self):
        for line in self.proc.stdout:
            if line.strip():
                self.samples.append((time.perf_counter(), line))

    def __enter__(self):
        import threading

        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        if self.proc:
            self.thread = threading.Thread(target=self._reader, daemon=True)
            self.thread.start()
            t0 = time.perf_counter()
            while not self.samples and time.perf_counter() - t0 < 5.0:
                time.sleep(0.01)
        self.t_start = time.perf_counter()
        return self

    def __exit__(self, *a):
        self.t_end = time.perf_counter() + self.period_ms / 1e3  # the sample taken as the region ends
        if self.proc:
            time.sleep(self.period_ms / 1e3 * 1.5)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)
        self.lines = [l for t, l in self.samples if self.t_start <= t <= self.t_end]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def reduce_max(x: float, world: int) -> float:
    from quicktex_b200.shard import max_over_ranks

    return max_over_ranks(x) if world > 1 else x


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def cpu_reference_sample(img: np.ndarray, mode: int = 0, threads: int = 0, side: int = 512):
    """The reference encoder on a side x side crop for each of the 36 settings, encode only
    (encoder and input built beforehand). mode 0: its own Encode as shipped (BlockEncoder::Encode,
    OpenMP over block rows for BC1); mode 1: OpenMP over EncodeBlock. Returns
    (Mblocks/s, seconds, threads, kind)."""
    import oracle

    crop = np.ascontiguousarray(img[:side, :side])
    cores = threads or os.cpu_count() or 1
    if not oracle.reference_available():
        raise RuntimeError("the compiled reference (oracle/_ref/libqtref.so) is not built")
    ref = oracle.Reference()
    ref.set_threads(cores)
    secs = 0.0
    t0 = time.perf_counter()
    for L, _mn, m, _in, it in SETTINGS:
        secs += ref.time_encode(1, crop, side, side, oracle.BC1Params(level=L, color_mode=m, interpolator=it),
                                mode=mode, reps=1)
    wall = time.perf_counter() - t0
    ref.set_threads(os.cpu_count() or 1)
    return (side // 4) ** 2 * len(SETTINGS) / secs / 1e6, wall, cores, "reference"


def cpu_sweep_figures(img: np.ndarray) -> dict:
    """The other two CPU figures of the reference's timing plan for the sweep: OpenMP over
    EncodeBlock on the same 512x512 crops, and one thread on 128x128 crops."""
    omp, t1, cores, _ = cpu_reference_sample(img, mode=1)
    one, t2, _, _ = cpu_reference_sample(img, mode=1, threads=1, side=128)
    return {"omp_over_blocks": omp, "single_thread": one, "unit": "Mblocks/s", "cores": cores, "kind": "reference",
            "sample": "36 settings on 512x512 crops (one thread: 128x128 crops); encode only",
            "cpu_seconds": t1 + t2}


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    import oracle
    import workloads as syn

    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "the compiled reference (oracle/_ref/libqtref.so, "
                                                             "built by oracle/Makefile from the reference sources) "
                                                             "is missing"}), flush=True)
        return
    img = syn.block_mix(W, H)
    vals = []
    for i in range(args.warmup + args.steps):
        v, dt, cores, kind = cpu_reference_sample(img)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    sample = ("512x512 crop (16,384 blocks) of the workload texture for each of the 36 settings per step; "
              "the reference's own Encode as shipped (OpenMP over block rows), encode only")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mblocks/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 36 * 16384 / value / 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded PCG64 block mix)", "config": CONFIG,
        "cpu_baseline": {"value": value, "unit": "Mblocks/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "Mblocks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def roofline_line(issue, achieved_exec, achieved_ref, peak_tops, sms, peaks_kind) -> dict:
    """The sweep's roofline object. Bound: CUDA-core instruction issue (the BC1 encoder is neither
    HBM- nor tensor-bound: even level 0 moves 72 B per ~4.6k thread instructions). Primary figure:
    warp instructions issued per second (per-block counts from ncu x blocks / CUDA-event time)
    over SMs x 4 schedulers x clock, when the counts are present. Beside it, the algorithmic work
    model: 10 lane-ops per oracle-counted candidate evaluation over SMs x 128 lanes x clock (a
    work count, not an issue fraction: the kernels spend ~3 instructions per candidate evaluation,
    so it can pass 1.0 at level 18)."""
    work = {
        "achieved": achieved_exec, "peak": peak_tops, "unit": "Tlane-op/s", "frac": achieved_exec / peak_tops,
        "work": "10 lane-ops x oracle-counted candidate evaluations per block, less those in second "
                "cluster-fit passes that repeat the first pass's trials (skipped here with identical output)",
        "achieved_reference_work": achieved_ref, "frac_reference_work": achieved_ref / peak_tops,
        "peak_source": f"{sms} SMs x 128 lanes x sm_max_mhz ({peaks_kind})",
    }
    line = {"bound": "issue", "traffic": BC1_DRAM_BYTES_PER_BLOCK * NB,
            "traffic_source": "ncu dram bytes of the five kernels of one 2048^2 level-18 call, per block, "
                              "times this texture's blocks",
            "kernel": "BC1 encode call: qtk::k_bc1_split, then qtk::k_bc1_fast for settings without "
                      "EndpointSearch, or qtk::k_bc1_defer + qtk::k_bc1_cf2 + qtk::k_bc1_search + qtk::k_bc1_finish",
            "work_model": work}
    if issue:
        line.update({k: issue[k] for k in ("achieved", "peak", "unit", "frac", "by_level_frac", "source")})
        line["peak_source"] = f"{sms} SMs x 4 schedulers x sm_max_mhz ({peaks_kind})"
    else:
        line.update({"achieved": achieved_exec, "peak": peak_tops, "unit": "Tlane-op/s",
                     "frac": achieved_exec / peak_tops, "source": "work model (instruction counts not measured)"})
    return line


def run_ours(args, world, rank, local):
    import torch

    import workloads as syn
    from quicktex_b200 import capi

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    img = syn.block_mix(4096, 4096)[:H, :W] if W <= 4096 else syn.block_mix(W, H)
    img = np.ascontiguousarray(img)
    host_in = torch.from_numpy(img.reshape(-1)).pin_memory()
    d_in = host_in.to(dev)
    d_out = torch.empty(NB * 8, dtype=torch.uint8, device=dev)
    host_out = torch.empty(NB * 8, dtype=torch.uint8).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    params = [capi.params_for_level(L, m, it) for L, _mn, m, _in, it in SETTINGS]
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def step():
        for p in params:
            capi.bc1_encode_device(d_in.data_ptr(), W, H, p, d_out.data_ptr(), sptr)

    # per-setting kernel times (one pass, for the roofline and the level breakdown)
    per = []
    for p in params:
        capi.bc1_encode_device(d_in.data_ptr(), W, H, p, d_out.data_ptr(), sptr)
    torch.cuda.synchronize()
    for p in params:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        a.record(stream)
        capi.bc1_encode_device(d_in.data_ptr(), W, H, p, d_out.data_ptr(), sptr)
        b.record(stream)
        b.synchronize()
        per.append(a.elapsed_time(b))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            times.append((a, b))
        torch.cuda.synchronize()
    barrier(world)
    ms = sum(a.elapsed_time(b) for a, b in times) / args.steps
    ms = reduce_max(ms, world)
    blocks_step = NB * len(SETTINGS)
    value = world * blocks_step / (ms / 1e3) / 1e6

    # end to end through the host-buffer C-ABI call (pinned host memory in and out)
    hin, hout = host_in.numpy(), host_out.numpy()

    def e2e_step():
        for p in params:
            capi.check(capi.lib().qt_bc1_encode_host(capi._p(hin), W, H, capi.ctypes.byref(p), capi._p(hout)))

    e2e_value = None
    if not args.no_e2e:
        for _ in range(max(1, args.warmup)):
            e2e_step()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        e2e_s = reduce_max((time.perf_counter() - t0) / args.steps, world)
        e2e_value = world * blocks_step / e2e_s / 1e6

    # the same through the drop-in Python API: BC1Encoder(level, mode, interpolator).encode(RawTexture),
    # whose texels live in the RawTexture's own storage (pinned blocks from the library's cache)
    e2e_dropin = None
    if not args.no_e2e and world == 1:
        import quicktex_b200 as qt
        from quicktex_b200.s3tc.bc1 import BC1Encoder
        from quicktex_b200.s3tc.interpolator import Interpolator, InterpolatorAMD, InterpolatorNvidia, InterpolatorRound

        tex = qt.RawTexture.frombytes(img.tobytes(), W, H)
        interps = [Interpolator, InterpolatorRound, InterpolatorNvidia, InterpolatorAMD]
        mode_enum = {0x04: BC1Encoder.ColorMode.FourColor, 0x03: BC1Encoder.ColorMode.ThreeColor,
                     0x13: BC1Encoder.ColorMode.ThreeColorBlack}
        encoders = [BC1Encoder(L, mode_enum[m], interps[it]()) for L, _mn, m, _in, it in SETTINGS]
        for e in encoders[:3]:
            e.encode(tex)
        passes = []  # the host copies share the box's CPU cores: the median of three passes
        for _ in range(3):
            t0 = time.perf_counter()
            for e in encoders:
                e.encode(tex)
            passes.append(time.perf_counter() - t0)
        e2e_dropin = {"value": blocks_step / float(np.median(passes)) / 1e6, "unit": "Mblocks/s",
                      "passes_mblocks_s": [blocks_step / t / 1e6 for t in passes],
                      "path": "BC1Encoder(level, color_mode, interpolator).encode(RawTexture) for the 36 settings: "
                              "texels in the RawTexture's storage (pinned, from qt_host_alloc), blocks returned in a new "
                              "BC1Texture; median of 3 passes"}
        del tex

    # roofline: algorithmic lane-ops (10 per candidate evaluation) / kernel time
    peaks, peaks_kind = load_peaks()
    with open(os.path.join(ROOT, "tests", "golden", "ce_counts.json")) as f:
        counts = json.load(f)
    ce, ce_rep = counts["per_block"], counts["per_block_repeated"]
    # (profiling variants at levels without oracle counts report no CE figure)
    ops = sum(10.0 * ce.get(f"L{L}_{mn}_{iname}", 0.0) * NB for L, mn, _m, iname, _it in SETTINGS)
    # the reference's work less the second cluster-fit passes that repeat the first (skipped here)
    ops_exec = ops - sum(10.0 * ce_rep.get(f"L{L}_{mn}_{iname}", 0.0) * NB for L, mn, _m, iname, _it in SETTINGS)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_tops = sms * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    achieved = ops / (sum(per) / 1e3) / 1e12
    achieved_exec = ops_exec / (sum(per) / 1e3) / 1e12
    # the counter-based issue roofline: warp instructions issued per second over the SMs'
    # 4 schedulers x clock (one warp instruction per scheduler per cycle)
    issue = None
    if all(f"L{L}_{mn}_{iname}" in WARP_INST_PER_BLOCK for L, mn, _m, iname, _it in SETTINGS):
        peak_wi = sms * 4 * peaks.get("sm_max_mhz", 1965.0) * 1e6
        cls = {}
        for (L, mn, _m, iname, _it), t in zip(SETTINGS, per):
            c = cls.setdefault(f"L{L}", [0.0, 0.0])
            c[0] += WARP_INST_PER_BLOCK[f"L{L}_{mn}_{iname}"] * NB
            c[1] += t / 1e3
        tot_i, tot_t = sum(c[0] for c in cls.values()), sum(c[1] for c in cls.values())
        issue = {"achieved": tot_i / tot_t / 1e9, "peak": peak_wi / 1e9, "unit": "Gwarp-inst/s",
                 "frac": tot_i / tot_t / peak_wi,
                 "by_level_frac": {k: v[0] / v[1] / peak_wi for k, v in cls.items()},
                 "source": "warp instructions per block per setting (ncu smsp__inst_executed.sum at 2048^2) x this "
                           "texture's blocks / CUDA-event kernel time; peak = SMs x 4 schedulers x sm_max_mhz"}
    by_level = {}
    for (L, _mn, _m, _in, _it), t in zip(SETTINGS, per):
        by_level.setdefault(f"L{L}", [0.0, 0])
        by_level[f"L{L}"][0] += t
        by_level[f"L{L}"][1] += NB
    line = {
        "metric": METRIC, "value": value, "unit": "Mblocks/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded PCG64 block mix; no public corpus exists)", "config": CONFIG,
        "roofline": roofline_line(issue, achieved_exec, achieved, peak_tops, sms, peaks_kind),
        "by_level_mblocks_s": {k: v[1] / (v[0] / 1e3) / 1e6 for k, v in by_level.items()},
        "e2e": {"value": e2e_value, "unit": "Mblocks/s", "h2d_bytes_per_step": W * H * 4 * len(SETTINGS),
                "d2h_bytes_per_step": NB * 8 * len(SETTINGS)},
        "e2e_dropin": e2e_dropin,
        # per encode call, as the library reports it: the encoder, the split pass (>= 16384 blocks)
        # and, for settings with EndpointSearch on large textures, the search pass
        "gpu_launches": args.steps * sum(capi.bc1_encode_kernels(W, H, p) for p in params),
        "clocks": clk.summary(),
    }
    peaks_hbm = peaks.get("hbm_gbs", 6650.0)
    if not args.no_hbm:
        hbm = measure_hbm_paths(dev, stream)
        line["hbm_paths"] = {k: dict(v, frac_of_hbm=v["gb_s"] / peaks_hbm) for k, v in hbm.items()}
        line["hbm_paths"]["peak_gb_s"] = peaks_hbm
    if not args.no_batch:
        line["batched"] = measure_batched(args, dev, world)
    if not args.no_serve and world == 1:
        line["serve"] = measure_serving(args, dev)
    if not args.no_dds and world == 1:
        line["dds"] = measure_dds(args, dev)
    if not args.no_configs and world == 1:
        line["config_bc1_512_L5"] = measure_config1(dev, stream, flush)
        line["config_bc3_bc4_bc5_8192"] = measure_config3(dev, stream)
    if world == 1 and rank == 0 and not args.no_cpu:
        v, dt, cores, kind = cpu_reference_sample(img)
        line["cpu_baseline"] = {"value": v, "unit": "Mblocks/s", "cores": cores, "kind": kind,
                                "sample": f"512x512 crop x 36 settings, the reference's own Encode as shipped "
                                          f"(OpenMP), encode only, {dt:.1f} s"}
        line["cpu_figures"] = cpu_sweep_figures(img)
    if rank == 0:
        print(json.dumps(line), flush=True)


GOLDEN_HASHES = os.path.join(ROOT, "tests", "golden", "ref_hashes.json")


def _sha(b) -> str:
    import hashlib

    return hashlib.sha256(bytes(b)).hexdigest()


def _timed_each(fn, stream, reps: int, flush=None) -> float:
    """Median CUDA-event time (ms) of `fn` on `stream` over `reps` runs, L2 flushed before each
    run when `flush` (a device buffer larger than L2) is given."""
    import torch

    fn()
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def _wall_each(fn, reps: int) -> float:
    """Median wall time (ms) of `fn` (a call that returns with its result in host memory)."""
    fn()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)) * 1e3


def cpu_figures(fmt: int, img: np.ndarray, params=None, c0: int = 0, c1: int = 1, side: int = 0, single_side: int = 0,
                decode_blocks=None, reps: int = 1) -> dict:
    """The reference's CPU encoder (oracle/_ref, unmodified sources) three ways, as the reference's
    timing plan asks: as shipped (its own Encode: OpenMP for BC1 only, serial for BC3/BC4/BC5),
    OpenMP over EncodeBlock (the fair parallel figure), and one thread. Encode only (tables and
    input built beforehand), best of `reps` after one untimed run, on a `side`^2 crop (single
    thread: `single_side`^2). With `decode_blocks`, the same three for decoding them instead."""
    import oracle

    if not oracle.reference_available():
        return {"unavailable": "compiled reference (oracle/_ref) not built"}
    ref = oracle.Reference()
    cores = os.cpu_count() or 1
    params = params or oracle.BC1Params()
    h, w = img.shape[:2]
    side = side or min(w, h)
    single_side = single_side or side

    def rate(s, mode, threads):
        ref.set_threads(threads)
        nb = (s // 4) ** 2
        if decode_blocks is not None:
            bw = w // 4
            blk = decode_blocks.reshape(h // 4, bw, -1)[: s // 4, : s // 4].reshape(-1)
            t = ref.time_decode(fmt, np.ascontiguousarray(blk), s, s, params.interpolator, c0, c1, mode, reps)
        else:
            t = ref.time_encode(fmt, np.ascontiguousarray(img[:s, :s]), s, s, params, c0, c1, mode, reps)
        return nb / t / 1e6

    t0 = time.perf_counter()
    out = {"as_shipped": rate(side, 0, cores), "omp_over_blocks": rate(side, 1, cores),
           "single_thread": rate(single_side, 1, 1), "unit": "Mblocks/s", "cores": cores, "kind": "reference",
           "sample": f"{side}x{side} crop ({(side // 4) ** 2} blocks); one thread on {single_side}x{single_side}"}
    ref.set_threads(cores)
    out["cpu_seconds"] = time.perf_counter() - t0
    return out


def measure_config1(dev, stream, flush, reps: int = 20):
    """512x512 gradient + noise (10% solid blocks), BC1 level 5 four-colour Ideal encode, then
    decode. Device-resident through the C-ABI (CUDA events, L2 flushed before each run), and end
    to end through the drop-in Python API (BC1Encoder(5).encode(RawTexture) and
    BC1Decoder().decode, whose texels live in the textures' own pinned storage), beside the reference's CPU
    figures. Outputs are checked against the reference's committed digests."""
    import torch

    import quicktex_b200 as qt
    import workloads as syn
    from quicktex_b200 import capi
    from quicktex_b200.s3tc.bc1 import BC1Decoder, BC1Encoder

    side = 512
    nb = (side // 4) ** 2
    img = syn.gradient_noise(side, side)
    golden = json.load(open(GOLDEN_HASHES))["gradient_512"]
    d_in = torch.from_numpy(img.reshape(-1).copy()).to(dev)
    d_blk = torch.empty(nb * 8, dtype=torch.uint8, device=dev)
    d_dec = torch.empty(side * side * 4, dtype=torch.uint8, device=dev)
    p = capi.params_for_level(5)
    sp = stream.cuda_stream
    enc_fn = lambda: capi.bc1_encode_device(d_in.data_ptr(), side, side, p, d_blk.data_ptr(), sp)  # noqa: E731
    dec_fn = lambda: capi.bc1_decode_device(d_blk.data_ptr(), side, side, 0, False, d_dec.data_ptr(), sp)  # noqa: E731
    enc_ms = _timed_each(enc_fn, stream, reps, flush)
    dec_ms = _timed_each(dec_fn, stream, reps, flush)
    torch.cuda.synchronize()
    exact = (_sha(d_blk.cpu().numpy()) == golden["bc1_L5_four_ideal"] and
             _sha(d_dec.cpu().numpy()) == golden["bc1_decode_ideal"])

    tex = qt.RawTexture.frombytes(img.tobytes(), side, side)
    enc, dec = BC1Encoder(5), BC1Decoder()
    blocks = enc.encode(tex)
    exact = exact and _sha(blocks.tobytes()) == golden["bc1_L5_four_ideal"]
    e_enc = _wall_each(lambda: enc.encode(tex), reps)
    e_dec = _wall_each(lambda: dec.decode(blocks), reps)
    e_both = _wall_each(lambda: dec.decode(enc.encode(tex)), reps)
    peaks, kind = load_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    cpu_enc = cpu_figures(1, img, reps=5)
    cpu_dec = cpu_figures(1, img, decode_blocks=np.frombuffer(blocks.tobytes(), np.uint8), reps=5)
    return {
        "workload": "512x512 gradient + noise, 10% solid blocks; BC1 level 5 four-colour Ideal encode, then decode",
        "blocks": nb,
        "device": {"encode_mblocks_s": nb / enc_ms / 1e3, "decode_mblocks_s": nb / dec_ms / 1e3,
                   "encode_decode_mblocks_s": nb / (enc_ms + dec_ms) / 1e3, "encode_ms": enc_ms, "decode_ms": dec_ms,
                   "l2": "flushed before each run"},
        "e2e_dropin": {"encode_mblocks_s": nb / e_enc / 1e3, "decode_mblocks_s": nb / e_dec / 1e3,
                       "encode_decode_mblocks_s": nb / e_both / 1e3,
                       "path": "BC1Encoder(5).encode(RawTexture) / BC1Decoder().decode: the textures' own (pinned) storage, "
                               "copies and kernel launches inside the timed call"},
        "roofline": {"bound": "hbm", "encode_gb_s": nb * 72 / enc_ms / 1e6, "decode_gb_s": nb * 72 / dec_ms / 1e6,
                     "peak_gb_s": hbm, "encode_frac": nb * 72 / enc_ms / 1e6 / hbm,
                     "decode_frac": nb * 72 / dec_ms / 1e6 / hbm, "peak_source": kind,
                     "note": "1 MiB of texels: one launch of 256 CTAs, latency-bound, not bandwidth-bound"},
        "cpu_encode": cpu_enc, "cpu_decode": cpu_dec,
        "bit_exact_vs_reference": exact,
    }


def measure_config3(dev, stream, reps: int = 5):
    """8192x8192: BC3 level 5 (Ideal) of the colour block mix with the alpha mix (binary
    cutouts, ramps, noise), BC4 on channels 0, 1 and 3 of it, and BC5 (channels 0, 1) of the
    normal map of a sum of 8 Gaussian bumps; each decoded back. Device-resident (256 MiB inputs,
    larger than L2), CUDA events; BC3 and BC5 encode also end to end through the drop-in Python
    API from the textures' own (pinned) storage. Outputs checked against the reference's committed digests."""
    import torch

    import quicktex_b200 as qt
    import workloads as syn
    from quicktex_b200 import capi
    from quicktex_b200.s3tc.bc3 import BC3Encoder
    from quicktex_b200.s3tc.bc5 import BC5Encoder

    side = 8192
    nb = (side // 4) ** 2
    golden = json.load(open(GOLDEN_HASHES))
    ga, gn = golden.get("alpha_8192", {}), golden.get("normal_8192", {})
    peaks, kind = load_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    sp = stream.cuda_stream
    L = capi.lib()
    vp = capi._vp
    res, exact = {}, {}
    d_blk = torch.empty(nb * 16, dtype=torch.uint8, device=dev)
    d_out = torch.empty(side * side * 4, dtype=torch.uint8, device=dev)

    def leg(name, fn, nbytes, golden_key, golden_entry, out_tensor):
        ms = _timed_each(fn, stream, reps)
        torch.cuda.synchronize()
        block_bytes = 16 if name.startswith(("bc3", "bc5")) else 8
        n = nb * block_bytes if name.endswith("encode") else side * side * 4
        exact[name] = _sha(out_tensor[:n].cpu().numpy()) == golden_entry.get(golden_key)
        res[name] = {"ms": ms, "mblocks_s": nb / ms / 1e3, "gb_s": nbytes / ms / 1e6, "frac_of_hbm": nbytes / ms / 1e6 / hbm}

    img = syn.alpha_mix(side, side)
    d_in = torch.from_numpy(img.reshape(-1)).to(dev)
    p5 = capi.params_for_level(5)
    leg("bc3_L5_encode", lambda: capi.bc3_encode_device(d_in.data_ptr(), side, side, p5, d_blk.data_ptr(), sp),
        nb * 80, "bc3_L5_ideal", ga, d_blk)
    leg("bc3_decode", lambda: capi.check(L.qt_bc3_decode_device(vp(d_blk.data_ptr()), side, side, 0, vp(d_out.data_ptr()), vp(sp))),
        nb * 80, "bc3_decode_ideal", ga, d_out)
    for c in (0, 1, 3):
        leg(f"bc4_ch{c}_encode", lambda c=c: capi.check(L.qt_bc4_encode_device(vp(d_in.data_ptr()), side, side, c, vp(d_blk.data_ptr()), vp(sp))),
            nb * 72, f"bc4_ch{c}", ga, d_blk)
        leg(f"bc4_ch{c}_decode", lambda c=c: capi.check(L.qt_bc4_decode_device(vp(d_blk.data_ptr()), side, side, c, vp(d_out.data_ptr()), vp(sp))),
            nb * 72, f"bc4_decode_ch{c}", ga, d_out)
    tex = qt.RawTexture.frombytes(img.tobytes(), side, side)
    e3 = _wall_each(lambda: BC3Encoder(5).encode(tex), 2)
    cpu3 = cpu_figures(3, img, capi_params_to_oracle(5), side=2048, single_side=512)
    cpu4 = {c: cpu_figures(4, img, c0=c, side=2048, single_side=1024) for c in (0, 3)}
    del tex, img

    nm = syn.normal_map(side, side)
    d_in.copy_(torch.from_numpy(nm.reshape(-1)))
    leg("bc5_encode", lambda: capi.check(L.qt_bc5_encode_device(vp(d_in.data_ptr()), side, side, 0, 1, vp(d_blk.data_ptr()), vp(sp))),
        nb * 80, "bc5_01", gn, d_blk)
    leg("bc5_decode", lambda: capi.check(L.qt_bc5_decode_device(vp(d_blk.data_ptr()), side, side, 0, 1, vp(d_out.data_ptr()), vp(sp))),
        nb * 80, "bc5_decode_01", gn, d_out)
    tex = qt.RawTexture.frombytes(nm.tobytes(), side, side)
    e5 = _wall_each(lambda: BC5Encoder(0, 1).encode(tex), 2)
    cpu5 = cpu_figures(5, nm, c0=0, c1=1, side=2048, single_side=1024)
    del tex, nm
    return {
        "workload": "8192x8192: BC3 level 5 Ideal and BC4 channels {0,1,3} of the block mix with the alpha mix; "
                    "BC5 channels (0,1) of the Gaussian-bump normal map; and their decodes",
        "blocks": nb, "device": res, "peak_gb_s": hbm, "peak_source": kind,
        "algorithmic_bytes_per_block": {"bc3": 80, "bc5": 80, "bc4": 72},
        "e2e_dropin": {"bc3_L5_encode_mblocks_s": nb / e3 / 1e3, "bc5_encode_mblocks_s": nb / e5 / 1e3,
                       "path": "BC3Encoder(5) / BC5Encoder(0, 1).encode(RawTexture): the textures' own (pinned) storage, "
                               "copies and kernels inside the timed call"},
        "cpu": {"bc3_L5_encode": cpu3, "bc4_encode": cpu4, "bc5_encode": cpu5},
        "bit_exact_vs_reference": exact,
    }


def capi_params_to_oracle(level: int, color_mode: int = 0x04, interpolator: int = 0):
    import oracle

    return oracle.BC1Params(level=level, color_mode=color_mode, interpolator=interpolator)


def measure_batched(args, dev, world):
    """Mixed batch: 10,000 seeded textures (log-uniform sides 4..2048, 25% off the
    4-texel grid; BC1:BC3:BC4:BC5 = 4:3:2:1; levels uniform in {0,5,10,18};
    BC4 on channel 0, BC5 on channels 0,1) as one persistent CUDA-graph launch
    versus one launch per texture, device-resident; plus the persistent path
    with the upload and download of all textures inside the timed region."""
    import torch

    import workloads as syn
    from quicktex_b200.batch import Arena, Batch, Job, PipelinedRun, run_plain, run_plain_host, run_plain_native

    from quicktex_b200.shard import block_cost, max_over_ranks, shard

    items = syn.mixed_batch(args.batch_count)
    all_blocks = sum(((i.width + 3) // 4) * ((i.height + 3) // 4) for i in items)
    pools = syn.MixedBatchPools()
    jobs = [Job.encode(i.fmt, pools.texture(i), i.width, i.height, level=i.level, channel=0, chan0=0, chan1=1)
            for i in items]
    if world > 1:  # each rank encodes its cost-balanced share of the same batch
        rank = int(os.environ.get("RANK", "0"))
        jobs = [jobs[k] for k in shard(items, world, rank, lambda i: block_cost(i.width, i.height, i.fmt, i.level))]
    del pools
    nblocks = sum(j.nblocks for j in jobs)
    arena = Arena(jobs, dev.index)
    arena.upload()
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    citems = arena.items()
    batch = Batch(dev.index)

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return ts

    for _ in range(args.warmup):
        batch.run(citems, sptr)
    torch.cuda.synchronize()
    persistent = timed(lambda: batch.run(citems, sptr), args.steps)
    arena.download()
    torch.cuda.synchronize()
    out_persistent = arena.outputs()  # each texture's bytes (the alignment padding between them is not output)
    arena.d_out.zero_()
    run_plain_native(citems, sptr)
    torch.cuda.synchronize()
    plain = timed(lambda: run_plain_native(citems, sptr), max(1, args.steps // 2))
    arena.download()
    torch.cuda.synchronize()
    identical = out_persistent == arena.outputs()
    arena.d_out.zero_()
    plain_py = timed(lambda: run_plain(citems, sptr), max(1, args.steps // 4))
    arena.download()
    torch.cuda.synchronize()
    identical = identical and out_persistent == arena.outputs()

    def e2e():
        arena.upload()
        batch.run(citems, sptr)
        arena.download()

    e2e_seq_ms = timed(e2e, max(1, args.steps // 2))
    torch.cuda.synchronize()
    # the same round trip pipelined in 4 chunks (uploads and downloads overlap the launches):
    # wall clock, from pinned host inputs to every output in pinned host memory
    pipe = PipelinedRun(arena, chunks=4, device=dev.index)
    arena.h_out.zero_()
    pipe.run()
    identical = identical and out_persistent == arena.outputs()
    e2e_ms = []
    for _ in range(max(1, args.steps // 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pipe.run()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    pipe.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run_plain_host(arena)
    plain_e2e = (time.perf_counter() - t0) * 1e3
    pm, qm, em, ym, sm_ = (max_over_ranks(float(np.median(x))) for x in (persistent, plain, e2e_ms, plain_py, e2e_seq_ms))
    plain_e2e = max_over_ranks(plain_e2e)
    ntiles = batch.last_tiles()
    batch.close()
    return {
        "workload": f"{len(jobs)} textures, log-uniform 4..2048 sides (25% not multiples of 4), "
                    "BC1:BC3:BC4:BC5 = 4:3:2:1, levels {0,5,10,18}, encode",
        "blocks": all_blocks,
        "scaling": "strong (the batch is sharded across ranks)" if world > 1 else "single GPU",
        "persistent_mblocks_s": all_blocks / (pm / 1e3) / 1e6,
        "plain_mblocks_s": all_blocks / (qm / 1e3) / 1e6,
        "persistent_over_plain": qm / pm,
        "plain": "one single-texture device entry point call per texture from the library's C++ loop "
                 "(qt_batch_run_plain)",
        "plain_python_loop_mblocks_s": all_blocks / (ym / 1e3) / 1e6,
        "persistent_over_plain_python_loop": ym / pm,
        "persistent_e2e_mblocks_s": all_blocks / (em / 1e3) / 1e6,
        "persistent_e2e": "pinned host buffers in and out; 4 chunks, each its own queue, uploads and downloads "
                          "on two copy streams overlapping the launches (PipelinedRun)",
        "persistent_e2e_sequential_mblocks_s": all_blocks / (sm_ / 1e3) / 1e6,
        "plain_e2e_mblocks_s": all_blocks / (plain_e2e / 1e3) / 1e6,
        "persistent_over_plain_e2e": plain_e2e / em,
        "e2e_h2d_bytes": arena.in_bytes, "e2e_d2h_bytes": arena.out_bytes,
        "ms": {"persistent": pm, "plain": qm, "plain_python_loop": ym, "persistent_e2e": em, "plain_e2e": plain_e2e},
        "tiles": ntiles,
        "launches_per_step": {"persistent": 1, "plain": len(jobs)},
        "outputs_identical": identical,
    }


class _ResponseRing:
    """Response buffers of a serving front end: slices of one pinned ring, handed
    out in order; a slice is reused only after the request that held it is done."""

    def __init__(self, nbytes: int):
        import torch

        self.buf = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
        self.np = self.buf.numpy()
        self.size, self.pos = nbytes, 0
        self.held = collections.deque()  # (start, end, future), oldest first
        self.pending = []

    def take(self, n: int):
        n = (n + 255) // 256 * 256
        assert n <= self.size
        if self.pos + n > self.size:
            self.pos = 0
        while self.held and self.held[0][0] < self.pos + n and self.held[0][1] > self.pos:
            self.held.popleft()[2].result()  # back-pressure: wait for the oldest response still in use
        start, self.pos = self.pos, self.pos + n
        self.pending.append((start, start + n))
        return self.np[start:start + n]

    def hold(self, futures) -> None:
        self.held.extend((a, b, f) for (a, b), f in zip(self.pending, futures))
        self.pending = []


def measure_dds(args, dev):
    """Mip chains (DDS encode): 8 seeded 2048x2048 RGBA images, full chains (12 levels each),
    BC3 level 10. ``dds.encode_many``: upload once per image, every level resized on the
    device, all levels of all images in one persistent launch, download. Beside it, the
    reference's way on the same GPU: Pillow resize per level on the CPU, one encode call per
    level through the drop-in API. Wall-clock, end to end (PIL image in -> blocks in host
    memory); outputs compared. Plus the resize kernels alone for one chain (CUDA events)."""
    import torch

    import quicktex_b200 as qt
    import workloads as syn
    from PIL import Image

    from quicktex_b200 import dds, image_utils
    from quicktex_b200.s3tc.bc3 import BC3Encoder

    side, n = 2048, 8
    imgs = [Image.fromarray(np.ascontiguousarray(syn.alpha_mix(side, side, workload=13, stream=k)), "RGBA") for k in range(n)]
    enc = BC3Encoder(10)
    sizes = image_utils.mip_sizes((side, side))
    blocks = n * sum(((w + 3) // 4) * ((h + 3) // 4) for w, h in sizes)

    def ours():
        return dds.encode_many([dds.EncodeRequest(im, enc, "DXT5") for im in imgs])

    def per_level():
        out = []
        for im in imgs:
            levels = [im] + [image_utils.resize_no_premultiply(im, s) for s in sizes[1:]]
            out.append([enc.encode(qt.RawTexture.frombytes(lv.tobytes("raw", "RGBA"), *lv.size)) for lv in levels])
        return out

    def wall(fn, reps):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), r

    t_ours, files = wall(ours, 3)
    t_ref, texs = wall(per_level, 1)
    identical = all(bytes(a) == bytes(b) for f, ts in zip(files, texs) for a, b in zip(f.textures, ts))
    # the resize kernels alone: one chain from a device-resident 2048^2 image
    src = torch.from_numpy(np.asarray(imgs[0]).reshape(-1).copy()).to(dev)
    outs = [torch.empty(w * h * 4, dtype=torch.uint8, device=dev) for w, h in sizes[1:]]
    st = torch.cuda.current_stream(dev)
    def chain():
        for (w, h), o in zip(sizes[1:], outs):
            image_utils.resize_device(src.data_ptr(), side, side, o.data_ptr(), w, h, st.cuda_stream)
    chain()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(5):
        chain()
    b.record(st)
    b.synchronize()
    chain_ms = a.elapsed_time(b) / 5
    # algorithmic bytes per level: the source rows it reads once (all of them) plus its texels written
    resize_bytes = sum(side * side * 4 + w * h * 4 for w, h in sizes[1:])
    return {"workload": f"{n} x {side}x{side} RGBA, full mip chains ({len(sizes)} levels), BC3 level 10",
            "blocks": blocks, "encode_many_ms": t_ours * 1e3, "encode_many_mblocks_s": blocks / t_ours / 1e6,
            "per_level_calls_ms": t_ref * 1e3, "per_level_calls_mblocks_s": blocks / t_ref / 1e6,
            "speedup": t_ref / t_ours, "outputs_identical": identical,
            "resize_chain_ms": chain_ms, "resize_chain_gb_s": resize_bytes / (chain_ms / 1e3) / 1e9}


def measure_serving(args, dev):
    """Open-loop Poisson arrivals of encode (70%) / decode (30%) requests, sizes,
    formats and levels drawn as in the mixed batch, against the continuous-batching
    server (16 GiB device budget); latency = arrival -> result bytes on the host."""
    import torch

    import workloads as syn
    from quicktex_b200.batch import Job, run_jobs
    from quicktex_b200.serve import Server, latency_stats

    items = syn.mixed_batch(args.serve_pool, workload=5)
    pools = syn.MixedBatchPools(workload=5)
    enc = [Job.encode(i.fmt, pools.texture(i), i.width, i.height, level=i.level, channel=0, chan0=0, chan1=1)
           for i in items]
    del pools
    dec = [Job.decode({1: "bc1", 3: "bc3", 4: "bc4", 5: "bc5"}[j.fmt], np.frombuffer(o, np.uint8), j.width, j.height,
                      channel=0, chan0=0, chan1=1) for j, o in zip(enc, run_jobs(enc, dev.index))]
    # request payloads live in pinned host memory, as a serving front end would keep them
    total = sum(j.data.nbytes for j in enc + dec)
    pinned = torch.empty(total, dtype=torch.uint8).pin_memory().numpy()
    o = 0
    for j in enc + dec:
        n = j.data.nbytes
        pinned[o:o + n] = j.data
        j.data = pinned[o:o + n]
        o += n
    srv = Server(dev.index, memory_budget=16 << 30, slots=3)
    for f in [srv.submit(j) for j in enc[:8] + dec[:8]]:  # warm-up: graphs captured, tables resident
        f.result()
    ring = _ResponseRing(1 << 30)
    loads = []
    for rate, seconds in zip(args.serve_rates, args.serve_seconds):
        rng = np.random.default_rng(int(rate))
        n = max(1, int(rate * seconds))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        is_dec = rng.random(n) < 0.3
        pick = rng.integers(0, len(enc), n)
        jobs = [dec[p] if d else enc[p] for p, d in zip(pick, is_dec)]
        gc.collect()
        gc.disable()  # a latency-sensitive front end keeps collector pauses out of the request path
        blocks0, batches0 = srv.blocks_done, srv.batches
        t0 = time.perf_counter() + 0.01
        due_np = t0 + arrivals
        due_at = due_np.tolist()
        # the front end sleeps (releasing the GIL) until the next arrival, then hands
        # over every request due by now, each with its response buffer in a pinned
        # ring; latency counts from each scheduled arrival
        futs, k = [], 0
        while k < n:
            now = time.perf_counter()
            if due_at[k] > now:
                time.sleep(min(due_at[k] - now, 1e-3))
                continue
            k1 = int(np.searchsorted(due_np, now, side="right"))
            outs = [ring.take(j.out_bytes) for j in jobs[k:k1]]
            fs = srv.submit_many(jobs[k:k1], due_at[k:k1], outs)
            ring.hold(fs)
            futs += fs
            k = k1
        for f in futs:
            f.result()
        gc.enable()
        span = max(f.request.t_done for f in futs) - t0
        st = latency_stats(futs)
        st.update({"offered_rps": rate, "achieved_rps": n / span, "mblocks_s": (srv.blocks_done - blocks0) / span / 1e6,
                   "batches": srv.batches - batches0, "seconds_offered": seconds})
        loads.append(st)
    srv.close()
    return {"mix": "70% encode / 30% decode; sizes, formats and levels as the mixed batch; "
                   f"{len(enc)} distinct payloads in pinned host memory",
            "device_budget_gib": 16, "slots": 3, "max_inflight_seen": srv.max_inflight_seen, "loads": loads}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-plain leg")
    ap.add_argument("--batch-count", type=int, default=10000, help="textures in the batched leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-dds", action="store_true", help="skip the mip-chain (DDS) leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the 512^2 BC1 and 8192^2 BC3/BC4/BC5 legs")
    ap.add_argument("--no-hbm", action="store_true", help="skip the bandwidth-bound kernels on 16384^2 textures")
    ap.add_argument("--serve-pool", type=int, default=256, help="distinct request payloads")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[1000, 10000, 50000])
    ap.add_argument("--serve-seconds", type=float, nargs="+", default=[2.0, 2.0, 1.0])
    ap.add_argument("--size", type=int, default=4096, help="texture side (profiling variants only)")
    ap.add_argument("--levels", type=str, default="0,10,18", help="levels (profiling variants only)")
    ap.add_argument("--hbm-only", action="store_true",
                    help="profiling variant: only the bandwidth-bound kernels on --size^2 textures, one JSON line")
    args = ap.parse_args()
    if args.hbm_only:
        import torch

        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        res = measure_hbm_paths(dev, torch.cuda.current_stream(dev), side=args.size, reps=max(1, args.steps))
        print(json.dumps({"hbm_paths": res, "side": args.size}))
        return
    configure(args.size, tuple(int(x) for x in args.levels.split(",")))
    if args.impl == "reference":  # CPU only: rank 0 runs it, the other ranks exit without work
        run_reference_arm(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_init(args)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
