#!/usr/bin/env python
"""Benchmark of the pairwise SIFT brute-force matcher (dense int8 contraction workload).

Workload (N=1): one image pair of 32768 query x 32768 train 128-byte SIFT-like descriptors
(50% true overlap, noise sigma 10), matched bidirectionally with second-best distance, ratio
test 0.8 and cross-check flags. A step = squared norms of both sets + the fused tcgen05 matcher
(init, match, flags kernels) over inputs already resident in HBM. Inputs (8 MiB) are smaller than
L2, so L2 is flushed (a 256 MiB write) between timed steps, outside the timed region.

Multi-GPU: image pairs are independent, so each rank matches its own pair (weak scaling, no
collective on the data path); the step time is the max over ranks.

--impl reference: the reference has no CPU matcher; its CPU path is the exhaustive exact loop of
its kernel tests (test/bruteForceMatchKernelTest.cpp:140-164), restated in oracle/ and timed on
the host cores (all threads) on a bounded row sample of the same workload.
"""
import argparse
import copy
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUERY = 32768
N_TRAIN = 32768
OVERLAP = 0.5
SIGMA = 10.0
WORKLOAD = "bf_pair_32768x32768"
METRIC = "desc-pairs/s"


def _config():
    return {
        "workload": WORKLOAD,
        "n_query": N_QUERY,
        "n_train": N_TRAIN,
        "overlap": OVERLAP,
        "noise_sigma": SIGMA,
        "ratio": 0.8,
        "cross_check": True,
        "l2": "256 MiB flush write between timed steps (inputs 8 MiB < L2)",
        "parallelism": "independent pairs per rank (replicas)",
    }


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons in the background during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def mark(self, which):
        setattr(self, which, time.perf_counter())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t_begin", 0.0), getattr(self, "t_end", float("inf"))
        window = [ln for ts, ln in self.lines if t0 <= ts <= t1 + 0.06]
        if not window and self.lines:  # region shorter than one sampling period: nearest sample
            window = [min(self.lines, key=lambda x: abs(x[0] - t1))[1]]
        for ln in window:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(value, device="cpu"):
    """Largest value over all ranks of the default process group (the job's step time is its
    slowest rank's); the value itself when running alone."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(q, t, rows, threads, min_seconds=0.0):
    """Times the oracle port (exhaustive exact bidirectional loop) on `rows` query rows against the
    whole train set, repeated until `min_seconds` of CPU work have run. Returns (pairs/s, seconds)."""
    from oracle import oracle as orc
    orc.load()
    sub = np.ascontiguousarray(q[:rows])
    orc.bf_match(sub[:8], t, threads=threads)  # warm
    reps, t0 = 0, time.perf_counter()
    while True:
        orc.bf_match(sub, t, threads=threads)
        reps += 1
        dt = time.perf_counter() - t0
        if dt >= min_seconds:
            break
    return reps * rows * len(t) / dt, dt


def cpu_baseline_scalar(q, t, rows):
    """The reference test's plain loop (one thread, scalar bytes) on `rows` query rows against
    the whole train set. Returns (pairs/s, seconds)."""
    from oracle import oracle as orc
    sub = np.ascontiguousarray(q[:rows])
    t0 = time.perf_counter()
    orc.bf_match_scalar(sub, t)
    dt = time.perf_counter() - t0
    return rows * len(t) / dt, dt


def check_exact(q, t, best_a, best_b, second_a, flags_a, threads):
    """True when the matcher's outputs (forward and backward BestMatch, second-best distance, flag
    word; host tensors) equal the oracle's on the whole pair."""
    from oracle import oracle as orc
    global _ORACLE_PAIR
    if _ORACLE_PAIR is None or _ORACLE_PAIR[0] is not q:
        efwd, ebwd, esec = orc.bf_match(q, t, threads=threads)
        _ORACLE_PAIR = (q, efwd, ebwd, esec, orc.match_flags(efwd, esec, ebwd))
    _, efwd, ebwd, esec, eflg = _ORACLE_PAIR
    u32 = lambda x: x.numpy().view(np.uint32)
    return bool(np.array_equal(u32(best_a).reshape(-1, 2), efwd) and np.array_equal(u32(best_b).reshape(-1, 2), ebwd)
                and np.array_equal(u32(second_a), esec) and np.array_equal(u32(flags_a), eflg))


_ORACLE_PAIR = None


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def _cpu_sample(q, t, threads, seconds):
    """Rows per run so one run takes about `seconds` (whole pair when faster), and the timing."""
    rate, _ = cpu_baseline(q, t, 256, threads)
    rows = int(max(256, min(len(q), rate * seconds / len(t))))
    return rows, cpu_baseline(q, t, rows, threads, min_seconds=seconds)


def run_reference(args):
    import numpy as np  # noqa: F401
    from rapidsfm_b200 import synth
    ws, rank, _ = _dist_env()
    if rank != 0:
        return
    q, t, _ = synth.make_pair(N_QUERY, N_TRAIN, OVERLAP, SIGMA, seed=1)
    threads = os.cpu_count() or 1
    # each step: a bounded sample so the whole run stays near two minutes (whole pair per run
    # when one pass is that fast, else the leading query rows)
    per_step = min(10.0, max(0.3, 120.0 / max(1, args.steps)))
    rows, _ = _cpu_sample(q, t, threads, per_step)
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(q, t, min(rows, 256), threads)
    for _ in range(args.steps):
        v, _ = cpu_baseline(q, t, rows, threads, min_seconds=per_step)
        vals.append(v)
    value = statistics.median(vals)
    ms_per_step = N_QUERY * N_TRAIN / value * 1e3
    sample = (f"{rows} query rows x {N_TRAIN} train of the {N_QUERY}x{N_TRAIN} pair per run, exact bidirectional, "
              "runs repeated to fill each step")
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "desc-pairs/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": _config(),
        "cpu_baseline": {"value": value, "unit": "desc-pairs/s", "cores": threads, "kind": "port",
                         "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": "desc-pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    import rapidsfm_b200 as R
    from rapidsfm_b200 import synth

    ws, rank, local = _dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = R._lib.load()
    stream = torch.cuda.current_stream(dev)

    q, t, _ = synth.make_pair(N_QUERY, N_TRAIN, OVERLAP, SIGMA, seed=1 + rank)
    dq = torch.from_numpy(q).to(dev)
    dt_ = torch.from_numpy(t).to(dev)
    task = R.BFTask(dq, dt_)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    nops = 2.0 * N_QUERY * N_TRAIN * 128

    def step():
        n = 0
        R.precomp_sift_sqr_norm(task.descA, out=task.sqrA)
        n += R.last_launch_count()
        R.precomp_sift_sqr_norm(task.descB, out=task.sqrB)
        n += R.last_launch_count()
        R.bf_match_ext([task])
        n += R.last_launch_count()
        return n

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    assert R.device_error() == 0

    # ---- device-timed steps (inputs resident in HBM)
    sampler = ClockSampler(local) if rank == 0 else None
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.3)
    import ctypes
    lib.rsfm_profile_enable(1)
    step_ms, launches = [], 0
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if sampler:
        sampler.mark("t_begin")
    for i in range(args.steps):
        flush.fill_(i & 255)
        evs[i][0].record(stream)
        launches += step()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    if sampler:
        sampler.mark("t_end")
    kms = ctypes.c_float(0)
    klaunch = ctypes.c_uint32(0)
    R._lib.check(lib.rsfm_profile_collect(ctypes.byref(kms), ctypes.byref(klaunch)), "rsfm_profile_collect")
    lib.rsfm_profile_enable(0)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    if ws > 1:
        total_ms = max_over_ranks(total_ms, dev)
        torch.distributed.barrier()
    clocks = sampler.stop() if sampler else None
    ms_per_step = total_ms / args.steps
    value = ws * N_QUERY * N_TRAIN / (ms_per_step * 1e-3)
    kernel_ms = kms.value / max(1, klaunch.value)

    # ---- end to end through the public API: H2D of both descriptor sets from pinned memory,
    # match, D2H of every result array; all inside the timed region.
    hq = torch.from_numpy(q).pin_memory()
    ht = torch.from_numpy(t).pin_memory()
    outs = {k: torch.empty(v.numel(), dtype=v.dtype).pin_memory() for k, v in
            (("fwd", task.bestA), ("bwd", task.bestB), ("sec", task.secondA), ("flg", task.flagsA))}
    h2d = hq.numel() + ht.numel()
    d2h = sum(v.numel() * v.element_size() for v in outs.values())
    e2e_ms = []
    for i in range(args.steps + 1):
        flush.fill_(i & 255)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dq.copy_(hq, non_blocking=True)
        dt_.copy_(ht, non_blocking=True)
        step()
        outs["fwd"].copy_(task.bestA, non_blocking=True)
        outs["bwd"].copy_(task.bestB, non_blocking=True)
        outs["sec"].copy_(task.secondA, non_blocking=True)
        outs["flg"].copy_(task.flagsA, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        if i > 0:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_serial_step = statistics.mean(e2e_ms)

    # ---- the same, pipelined as a user would run a stream of pairs: two buffer sets on three
    # streams, so the H2D of step i+1 and the D2H of step i-1 overlap the matching of step i.
    # Every step still copies its inputs in from pinned memory and its results out.
    sets = []
    for _ in range(2):
        bq, bt = torch.empty_like(dq), torch.empty_like(dt_)
        bt_task = R.BFTask(bq, bt)
        bt_task.secondA = torch.empty_like(task.secondA)
        bt_task.flagsA = torch.empty_like(task.flagsA)
        bo = {k: torch.empty_like(v).pin_memory() for k, v in outs.items()}
        sets.append((bq, bt, bt_task, bo))
    s_h2d, s_cmp, s_d2h = (torch.cuda.Stream(dev) for _ in range(3))
    ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("h2d", "cmp", "d2h")}

    def issue(i):
        k = i % 2
        bq, bt, bt_task, bo = sets[k]
        if i >= 2:
            s_h2d.wait_event(ev["cmp"][k])  # inputs of step i-2 consumed
        with torch.cuda.stream(s_h2d):
            bq.copy_(hq, non_blocking=True)
            bt.copy_(ht, non_blocking=True)
            ev["h2d"][k].record(s_h2d)
        s_cmp.wait_event(ev["h2d"][k])
        if i >= 2:
            s_cmp.wait_event(ev["d2h"][k])  # outputs of step i-2 read back
        R.precomp_sift_sqr_norm(bq, out=bt_task.sqrA, stream=s_cmp)
        R.precomp_sift_sqr_norm(bt, out=bt_task.sqrB, stream=s_cmp)
        R.bf_match_ext([bt_task], stream=s_cmp)
        ev["cmp"][k].record(s_cmp)
        s_d2h.wait_event(ev["cmp"][k])
        with torch.cuda.stream(s_d2h):
            bo["fwd"].copy_(bt_task.bestA, non_blocking=True)
            bo["bwd"].copy_(bt_task.bestB, non_blocking=True)
            bo["sec"].copy_(bt_task.secondA, non_blocking=True)
            bo["flg"].copy_(bt_task.flagsA, non_blocking=True)
            ev["d2h"][k].record(s_d2h)

    for i in range(2):
        issue(i)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_h2d)
    s_cmp.wait_event(e0)
    s_d2h.wait_event(e0)
    for i in range(args.steps):
        issue(i)
    e1.record(s_d2h)
    torch.cuda.synchronize()
    e2e_step = e0.elapsed_time(e1) / args.steps
    e2e_last = sets[(args.steps - 1) % 2][3]  # host outputs of the last pipelined step
    # copy bandwidth of this box, each direction alone (same pinned buffers, same sizes)
    h2d_ms = _events_ms(lambda: (dq.copy_(hq, non_blocking=True), dt_.copy_(ht, non_blocking=True)), 10, stream)
    d2h_ms = _events_ms(lambda: [outs[k].copy_(v, non_blocking=True) for k, v in
                                 (("fwd", task.bestA), ("bwd", task.bestB), ("sec", task.secondA),
                                  ("flg", task.flagsA))], 10, stream)
    if ws > 1:
        e2e_step = max_over_ranks(e2e_step, dev)
        e2e_serial_step = max_over_ranks(e2e_serial_step, dev)
    e2e_value = ws * N_QUERY * N_TRAIN / (e2e_step * 1e-3)

    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return

    # ---- roofline: dense int8 tensor pipe (live MMA-only probe on this GPU)
    tops = ctypes.c_float(0)
    pms = ctypes.c_float(0)
    R._lib.check(lib.rsfm_int8_mma_peak(20000, ctypes.byref(tops), ctypes.byref(pms)), "rsfm_int8_mma_peak")
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    bf16 = None
    if os.path.exists(peaks_path):
        try:
            bf16 = json.load(open(peaks_path)).get("bf16_tflops")
        except Exception:
            bf16 = None
    achieved = nops / (kernel_ms * 1e-3) / 1e12
    peak = float(tops.value)
    roofline = {
        "bound": "tensor",
        "achieved": achieved,
        "peak": peak,
        "unit": "TOP/s",
        "frac": achieved / peak,
        # DRAM bytes per launch from an ncu capture of the 16384^2 case (dram__bytes_read.sum +
        # dram__bytes_write.sum = 4.71 MB), scaled linearly: DRAM traffic is the inputs and outputs,
        # since the B blocks each row block re-streams hit L2.
        "traffic": 4.71e6 * (N_QUERY / 16384.0),
        "traffic_note": "ncu at 16384^2, scaled by n/16384",
        "kernel": "bf_match_kernel",
        "kernel_ms": kernel_ms,
        "peak_source": "measured live: int8 tcgen05 MMA-only probe (rsfm_int8_mma_peak), dense",
        "peak_bf16_x2_of_measured": (2 * bf16) if bf16 else None,
        "ops_per_launch": nops,
    }

    # ---- CPU baseline: oracle port, all host threads, about 10 s of work on the same pair; the
    # faithful scalar loop on one core beside it (bounded row sample). The oracle's whole-pair
    # result also checks the timed pair's device outputs and the end-to-end host outputs.
    threads = os.cpu_count() or 1
    rows, (cpu_val, cpu_dt) = _cpu_sample(q, t, threads, 10.0)
    scalar_rows = 256 if args.size == 0 else max(8, min(256, N_QUERY))
    scalar_val, scalar_dt = cpu_baseline_scalar(q, t, scalar_rows)
    exact = check_exact(q, t, task.bestA.cpu(), task.bestB.cpu(), task.secondA.cpu(), task.flagsA.cpu(), threads)
    exact_e2e = check_exact(q, t, e2e_last["fwd"], e2e_last["bwd"], e2e_last["sec"], e2e_last["flg"], threads)

    extras = {}
    if not args.no_extras and ws == 1:  # single-GPU sections; scaling runs time the pair only
        extras["filtered"] = run_filtered(dev, stream, q, t)
        extras["batched"] = run_batched(dev, stream)
        extras["cascade"] = run_cascade(dev, stream, n_pairs=args.cascade_pairs)
        extras["hash"] = run_hash(dev, stream, n=1 << args.hash_log2)
        extras["ransac"] = run_ransac(dev, stream)
        extras["training"] = run_training(dev, stream)

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "desc-pairs/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": _config(),
        "e2e": {"value": e2e_value, "unit": "desc-pairs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_step,
                "mode": "pipelined: 2 buffer sets, H2D / match / D2H on 3 streams, every step copies in and out",
                "serial_ms_per_step": e2e_serial_step,
                "serial_value": ws * N_QUERY * N_TRAIN / (e2e_serial_step * 1e-3),
                "h2d_ms": h2d_ms, "h2d_GBps": h2d / (h2d_ms * 1e-3) / 1e9,
                "d2h_ms": d2h_ms, "d2h_GBps": d2h / (d2h_ms * 1e-3) / 1e9,
                "device_step_ms": ms_per_step,
                "bound": max((("host-to-device copy", h2d_ms), ("matching on the device", ms_per_step),
                              ("device-to-host copy", d2h_ms)), key=lambda x: x[1])[0],
                "exact": exact_e2e},
        "exact": exact,
        "gpu_launches": int(launches),
        "roofline": roofline,
        "cpu_baseline": {"value": cpu_val, "unit": "desc-pairs/s", "cores": threads, "kind": "port",
                         "sample": f"{rows} query rows x {N_TRAIN} train of the pair, repeated for {cpu_dt:.1f} s",
                         "cpu_model": cpu_model(),
                         "scalar": {"value": scalar_val, "unit": "desc-pairs/s", "cores": 1,
                                    "sample": f"{scalar_rows} query rows x {N_TRAIN} train, one thread, "
                                              f"scalar byte loop ({scalar_dt:.1f} s)"}},
        "clocks": clocks,
        "int8_tops_effective": nops / (ms_per_step * 1e-3) / 1e12,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def _events_ms(fn, reps, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_filtered(dev, stream, q, t, reps=10):
    """matchAndFilter, cross-check mode, one pair through the public API, wall clock per pair with
    the H2D of both descriptor sets: filters on the GPU (the count, then only the surviving
    ValidMatch records cross to the host) vs the reference's flow (both BestMatch arrays to the
    host, then the host crossCheckMatches, bruteForceMatcher.cpp:355-369, 426-442)."""
    import ctypes

    import numpy as np
    import torch

    import rapidsfm_b200 as R

    lib = R._lib.load()
    nq, nt = len(q), len(t)
    hq, ht = torch.from_numpy(q).pin_memory(), torch.from_numpy(t).pin_memory()
    dq, dt_ = torch.empty_like(hq, device=dev), torch.empty_like(ht, device=dev)
    task = R.BFTask(dq, dt_)
    cap = min(nq, nt)
    out = torch.empty((cap, 3), dtype=torch.int32, device=dev)
    cnt = torch.empty(1, dtype=torch.int32, device=dev)
    hout = torch.empty((cap, 3), dtype=torch.int32).pin_memory()
    hcnt = torch.empty(1, dtype=torch.int32).pin_memory()
    hf = torch.empty(nq, dtype=torch.int64).pin_memory()
    hb = torch.empty(nt, dtype=torch.int64).pin_memory()
    hvm = np.empty((cap, 3), dtype=np.uint32)
    sp = ctypes.c_void_p(stream.cuda_stream)

    def match():
        dq.copy_(hq, non_blocking=True)
        dt_.copy_(ht, non_blocking=True)
        R.precomp_sift_sqr_norm(dq, out=task.sqrA, stream=stream)
        R.precomp_sift_sqr_norm(dt_, out=task.sqrB, stream=stream)
        R.bf_match([task], stream=stream)

    def on_device():
        match()
        R._lib.check(lib.rsfm_cross_check_matches_device(task.bestA.data_ptr(), nq, task.bestB.data_ptr(), nt,
                                                         out.data_ptr(), cnt.data_ptr(), sp), "filter")
        hcnt.copy_(cnt, non_blocking=True)
        stream.synchronize()
        n = int(hcnt[0])
        hout[:n].copy_(out[:n], non_blocking=True)
        stream.synchronize()
        return n, 4 + 12 * n

    def on_host():
        match()
        hf.copy_(task.bestA, non_blocking=True)
        hb.copy_(task.bestB, non_blocking=True)
        stream.synchronize()
        n = lib.rsfm_cross_check_matches(hf.data_ptr(), nq, hb.data_ptr(), nt, hvm.ctypes.data)
        return n, 8 * (nq + nt)

    res = {}
    for name, fn in (("device_filter", on_device), ("host_filter", on_host)):
        for _ in range(3):
            fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            n, d2h = fn()
        ms = (time.perf_counter() - t0) * 1e3 / reps
        res[name] = {"ms_per_pair": ms, "matches": int(n), "d2h_bytes": int(d2h)}
    assert res["device_filter"]["matches"] == res["host_filter"]["matches"]
    res["pair"] = f"{nq}x{nt}"
    return res


def run_batched(dev, stream, seed=2):
    """Config 2: 512 uneven pairs (sizes U[2000,16000], overlap U[0.1,0.7], noise U[4,12]) as one
    autotuned graph plan vs. one rsfm_bf_match_ext call per pair. Inputs (about 1.2 GB) exceed L2."""
    import torch
    import rapidsfm_b200 as R
    from rapidsfm_b200 import synth
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    tasks, pairs = [], 0
    for _ in range(512):
        na, nb = int(rng.integers(2000, 16001)), int(rng.integers(2000, 16001))
        q, t, _ = synth.make_pair_torch(na, nb, float(rng.uniform(0.1, 0.7)), float(rng.uniform(4, 12)), g, dev)
        tasks.append(R.BFTask(q, t))
        pairs += na * nb
    t0 = time.perf_counter()
    opts, _ = R.autotune_plan(tasks, reps=2)
    tune_s = time.perf_counter() - t0
    plan = R.BFPlan(tasks, options=opts)
    plan_ms = _events_ms(lambda: plan.launch(stream), 5, stream)
    per_ms = _events_ms(lambda: [R.bf_match_ext([t], stream=stream) for t in tasks], 2, stream)
    plan.close()
    return {"workload": "512 pairs, N,M ~ U[2000,16000]", "desc_pairs": pairs,
            "plan_ms": plan_ms, "plan_desc_pairs_per_s": pairs / (plan_ms * 1e-3),
            "per_pair_ms": per_ms, "per_pair_desc_pairs_per_s": pairs / (per_ms * 1e-3),
            "speedup_vs_per_pair": per_ms / plan_ms,
            "options": {"rowTiles": opts.rowTiles, "colBlocks": opts.colBlocks,
                        "epilogueGroups": opts.epilogueGroups, "schedule": opts.schedule},
            "autotune_s": tune_s, "int8_tops": 256.0 * pairs / (plan_ms * 1e-3) / 1e12}


def run_cascade(dev, stream, n_pairs=1000, n=8192, seed=3):
    """Configs 3 and 4: n_pairs pairs of n descriptors (40% overlap, noise 8); ranked cascade
    matching (T tables x 8 bits, 128-bit Hamming ranking, top-10 exact re-rank, ratio 0.8) with
    random projections vs. the learned hash, all pairs in one launch each. The brute-force
    matches are the brute-force best matches that pass the ratio test and the cross-check.
    Recall = share of the brute-force matches that the hash matcher finds; precision = share of
    the hash matcher's reported matches (its ratio test passes; for findBestMatch, its two
    directions cross-check) that are brute-force matches."""
    import torch
    import rapidsfm_b200 as R
    from rapidsfm_b200 import cashash as ch
    from rapidsfm_b200 import learned_hash as lh
    from rapidsfm_b200 import synth
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    imgs = [synth.make_pair_torch(n, n, 0.4, 8.0, g, dev)[:2] for _ in range(n_pairs)]
    tasks = [R.BFTask(q, t) for q, t in imgs]
    plan = R.BFPlan(tasks)
    bf_ms = _events_ms(lambda: plan.launch(stream), 2, stream)
    plan.close()
    truth = [((t.flagsA & 3) == 3, t.bestA & 0xFFFFFFFF) for t in tasks]
    pairs = n_pairs * n * n
    out = {"workload": f"{n_pairs} pairs x {n} descriptors, 40% overlap, noise 8", "desc_pairs": pairs,
           "brute_force_plan_ms": bf_ms}
    hashers = {"plain": ch.CasHash(ch.gaussian_weights(1))}
    wpath = lh.default_params_path()
    if os.path.exists(wpath):
        hashers["learned"] = lh.LearnedHash(np.load(wpath))
    for name, h in hashers.items():
        if name == "plain":
            for q, t in imgs:
                h.fit(q)
                h.fit(t)
        # registration of all images (hash, norms, buckets, records) with one library call
        t0 = time.perf_counter()
        flat = ch.register_ranked_images(h, [x for pair in imgs for x in pair], stream=stream)
        torch.cuda.synchronize()
        hash_s = time.perf_counter() - t0
        # train images' records in each table's bucket-list order (table records): a candidate is
        # then one load at its list position; the same images without them read a bucket entry,
        # then the record (same results, checked below)
        t0 = time.perf_counter()
        for t in flat[1::2]:
            t.pack_table_records(stream=stream)
        torch.cuda.synchronize()
        trec_s = time.perf_counter() - t0
        ranked = list(zip(flat[0::2], flat[1::2]))
        bare = []
        for t in flat[1::2]:
            b = copy.copy(t)
            b.table_records = None
            bare.append(b)
        ranked_bare = list(zip(flat[0::2], bare))
        rows = {}
        for tables in (2, 3, 4, 6, 8):
            bb = ch.RankedBatch(ranked_bare, tables, 10)
            ms_bare = _events_ms(lambda: bb.launch(stream), 3, stream)
            batch = ch.RankedBatch(ranked, tables, 10)
            ms = _events_ms(lambda: batch.launch(stream), 3, stream)
            equal = all(torch.equal(x[0], y[0]) and torch.equal(x[1], y[1]) and torch.equal(x[2], y[2])
                       for x, y in zip(batch.results, bb.results))
            bb.close()
            hit = torch.zeros((), dtype=torch.int64, device=dev)
            tot = torch.zeros((), dtype=torch.int64, device=dev)
            rep = torch.zeros((), dtype=torch.int64, device=dev)
            tp = torch.zeros((), dtype=torch.int64, device=dev)
            for (ok, gt), (best, _, flg, _) in zip(truth, batch.results):
                same = (best & 0xFFFFFFFF) == gt
                hit += (same & ok).sum()
                tot += ok.sum()
                # reported matches: the hash matcher's own ratio test passes
                r = (flg & 1) == 1
                rep += r.sum()
                tp += (r & same & ok).sum()
            rows[str(tables)] = {"match_ms": ms, "match_ms_thread_per_query": ms_bare,
                                 "results_equal_thread_per_query": equal, "recall": int(hit) / max(1, int(tot)),
                                 "precision": int(tp) / max(1, int(rep)), "reported": int(rep),
                                 "desc_pairs_per_s": pairs / (ms * 1e-3)}
            batch.close()
        ok98 = [int(k) for k, v in rows.items() if v["recall"] >= 0.98]
        out[name] = {"tables": rows, "hash_and_buckets_host_s": hash_s, "table_records_host_s": trec_s,
                     "fewest_tables_at_98pct_recall": min(ok98) if ok98 else None}
        if name == "plain":
            # reference mode (cashash::findBestMatch): all 8 schemes, exact L2 over every descriptor
            # pair sharing a bucket, per-scheme bucket lists; one call per pair
            fbm = lambda: [ch.find_best_match([qi], ti, stream=stream) for qi, ti in ranked]
            ms_calls = _events_ms(fbm, 2, stream)
            # all pairs in one call (rsfm_cashash_find_best_match_pairs: builds its work list, one
            # host synchronization per call) and as a batch built once (rsfm_cashash_fbm_batch_*:
            # each launch = result init + the matching kernel, no synchronization)
            fbp = lambda: ch.find_best_match_pairs(ranked, stream=stream)
            ms_call = _events_ms(fbp, 3, stream)
            fbb = ch.FindBestMatchBatch(ranked, stream=stream)
            ms = _events_ms(lambda: fbb.launch(stream), 3, stream)
            res = fbb.results
            hit = torch.zeros((), dtype=torch.int64, device=dev)
            tot = torch.zeros((), dtype=torch.int64, device=dev)
            rep = torch.zeros((), dtype=torch.int64, device=dev)
            tp = torch.zeros((), dtype=torch.int64, device=dev)
            for (ok, gt), (bq, bt) in zip(truth, res):
                jq = bq & 0xFFFFFFFF
                same = jq == gt
                hit += (same & ok).sum()
                tot += ok.sum()
                # reported matches: cross-checked in the two directions (the reference matcher's
                # use of findBestMatch results, bruteForceMatch.cpp:23-40)
                valid = jq < bt.numel()
                back = (bt[jq.clamp(max=bt.numel() - 1)] & 0xFFFFFFFF) == torch.arange(bq.numel(), device=dev)
                r = valid & back
                rep += r.sum()
                tp += (r & same & ok).sum()
            fbb.close()
            out["find_best_match_8_schemes"] = {"ms": ms, "recall": int(hit) / max(1, int(tot)),
                                                "precision": int(tp) / max(1, int(rep)), "reported": int(rep),
                                                "one_call_all_pairs_ms": ms_call,
                                                "desc_pairs_per_s": pairs / (ms * 1e-3),
                                                "one_call_per_pair_ms": ms_calls}
    # registration blobs (the reference's preCompForMatch layout, cascade-hash flags: norms, bias
    # from the running accumulator, keys with fused histogram, bounds, bucket lists), image by image
    from rapidsfm_b200 import precomp
    reg = precomp.Registrar(use_sqr_norm=True, use_cas_hash=True, device=dev)
    sample = [x for pair in imgs[:100] for x in pair]
    for k, d in enumerate(sample[:4]):
        reg.register(("warm-up", k), d, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for k, d in enumerate(sample):
        reg.register(k, d, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    out["registration_blob"] = {"images": len(sample), "descriptors_per_image": n,
                                "ms_per_image": ms / len(sample), "wall_ms_per_image": 1e3 * wall / len(sample),
                                "desc_per_s": len(sample) * n / (ms * 1e-3)}
    if "learned" in out:
        p6 = out["plain"]["tables"]["6"]
        ok = [v for v in out["learned"]["tables"].values() if v["recall"] >= p6["recall"]]
        out["learned_speedup_at_plain_recall"] = (p6["match_ms"] / min(v["match_ms"] for v in ok)) if ok else None

        def at98(name):
            t = out[name]["fewest_tables_at_98pct_recall"]
            return out[name]["tables"][str(t)]["match_ms"] if t else None

        a, b = at98("plain"), at98("learned")
        out["learned_speedup_at_98pct_recall"] = a / b if a and b else None
        out["plain_speedup_vs_brute_force_at_98pct_recall"] = out["brute_force_plan_ms"] / a if a else None
        # the fastest plain cascade-hash path at >= 98 % recall: ranked tables or findBestMatch
        fbm = out.get("find_best_match_8_schemes")
        if fbm and fbm["recall"] >= 0.98:
            a = min(a, fbm["ms"]) if a else fbm["ms"]
        out["fastest_plain_at_98pct_recall_ms"] = a
        out["learned_speedup_vs_fastest_plain_at_98pct_recall"] = a / b if a and b else None
    return out


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except Exception:
        return {}


def run_hash(dev, stream, n=1 << 24):
    """Hashing throughput on n descriptors (2 GiB, far above L2): cascade hash (192 channels,
    fused histogram; algorithmic bytes n*(128+8+16)), descriptor accumulation (n*128 bytes) and the
    learned hash (131072 bf16 FLOP per descriptor), against the measured HBM and bf16 peaks."""
    import torch
    from rapidsfm_b200 import cashash as ch
    from rapidsfm_b200 import learned_hash as lh
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    desc = torch.randint(0, 256, (n, 128), dtype=torch.uint8, device=dev, generator=g)
    cas = ch.CasHash(ch.gaussian_weights(4))
    cas.fit(desc[: 1 << 20])
    keys = torch.empty((n, 8), dtype=torch.uint8, device=dev)
    codes = torch.empty((n, 4), dtype=torch.int32, device=dev)
    hist = torch.empty((8, 256), dtype=torch.int32, device=dev)
    lib = R_lib()
    p = ch._p

    def hash_call():
        lib.rsfm_cashash_compute_hash(p(cas.w), p(cas.bias), 192, p(desc), n, p(keys), p(codes), p(hist),
                                      ctypes.c_void_p(stream.cuda_stream))

    def acc_call():
        lib.rsfm_cashash_accumulate_desc(p(cas.acc), 1, p(desc), n, ctypes.c_void_p(stream.cuda_stream))

    peaks = _peaks()
    hbm = peaks.get("hbm_gbs")
    bf16 = peaks.get("bf16_tflops")
    out = {"n_desc": n}
    ms = _events_ms(hash_call, 5, stream)
    gbs = n * (128 + 8 + 16) / (ms * 1e-3) / 1e9
    out["cashash_hash"] = {"ms": ms, "GB/s": gbs, "frac_of_measured_hbm": gbs / hbm if hbm else None,
                           "channels": 192}

    def hash64_call():  # computeHashForBucketOnly: the 64 key channels, what the matcher registers
        lib.rsfm_cashash_compute_hash(p(cas.w), p(cas.bias), 64, p(desc), n, p(keys), None, p(hist),
                                      ctypes.c_void_p(stream.cuda_stream))

    ms = _events_ms(hash64_call, 5, stream)
    gbs = n * (128 + 8) / (ms * 1e-3) / 1e9
    out["cashash_hash_keys_only"] = {"ms": ms, "GB/s": gbs, "frac_of_measured_hbm": gbs / hbm if hbm else None,
                                     "channels": 64}
    ms = _events_ms(acc_call, 5, stream)
    gbs = n * 128 / (ms * 1e-3) / 1e9
    out["cashash_accumulate"] = {"ms": ms, "GB/s": gbs, "frac_of_measured_hbm": gbs / hbm if hbm else None}
    wpath = lh.default_params_path()
    if os.path.exists(wpath):
        h = lh.LearnedHash(np.load(wpath))
        ms = _events_ms(lambda: h.hash(desc, keys=keys, codes=codes, stream=stream), 5, stream)
        tf = n * 131072.0 / (ms * 1e-3) / 1e12
        gbs = n * (128 + 8 + 16) / (ms * 1e-3) / 1e9
        out["learned_hash"] = {"ms": ms, "TFLOP/s": tf, "frac_of_measured_bf16": tf / bf16 if bf16 else None,
                               "GB/s": gbs, "frac_of_measured_hbm": gbs / hbm if hbm else None}
    return out


TRAIN_FLOP_PER_ROW = 5 * 2 * 128 * 256  # five contractions of 128 x 256 per gathered row (3 rows per triplet)


def run_training(dev, stream, batch=4096, steps=300, seed=7):
    """Learned-hash trainer throughput: batch-4096 triplet steps (gather, forward, triplet loss,
    backward, Adam; the five contractions on the tensor cores) over synthetic SIFT-like pairs with
    known correspondences; triplet indices drawn on the device every step, as the training loop
    does. Reports ms per step, the projected time of the 20k-step training run and the
    contractions' TFLOP/s against the measured bf16 peak."""
    import torch
    from rapidsfm_b200 import learned_hash as lh
    from rapidsfm_b200 import synth
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    n = 8192
    qs, ts, A, P = [], [], [], []
    for k in range(8):
        q, t, truth = synth.make_pair_torch(n, n, 0.4, 8.0, g, dev)
        pos = torch.nonzero(truth >= 0).flatten()
        qs.append(q)
        ts.append(t)
        A.append(truth[pos] + k * n)
        P.append(pos + k * n)
    Q, T, A, P = torch.cat(qs), torch.cat(ts), torch.cat(A), torch.cat(P)
    tr = lh.Trainer(lh.init_params(seed), batch, lr=1e-3, margin=48.0)

    def one():
        sel = torch.randint(0, len(A), (batch,), device=dev, generator=g)
        ip = P[sel].int()
        inn = ((ip // n) * n + torch.randint(0, n, (batch,), device=dev, generator=g)).int()
        tr.step(Q, A[sel].int(), T, ip, T, inn)

    # as the training loop runs it: a few eager steps, then one step (sampling included) replayed
    # from a CUDA graph; also the eager step for comparison
    with torch.cuda.stream(stream):
        ms_eager = _events_ms(one, 50, stream)
        graph = lh.StepGraph(one, generators=(g,))
        ms = _events_ms(graph.replay, steps, stream)
        first = float(tr.loss.item())
        for _ in range(50):
            graph.replay()
        last = float(tr.loss.item())
    del graph
    tr.close()
    flop = TRAIN_FLOP_PER_ROW * 3 * batch
    tf = flop / (ms * 1e-3) / 1e12
    bf16 = _peaks().get("bf16_tflops")
    return {"batch": batch, "ms_per_step": ms, "ms_per_step_eager": ms_eager, "steps_per_s": 1e3 / ms,
            "projected_20k_steps_s": 20000 * ms / 1e3,
            "contraction_flop_per_step": flop, "TFLOP/s": tf, "frac_of_measured_bf16": tf / bf16 if bf16 else None,
            "loss_first_last": [first, last], "timed_steps": steps}


def run_full_training(dev):
    """The learned hash's full training run as the package performs it (rapidsfm_b200.learned_hash
    train_from_brute_force: brute-force correspondences of 200 seeded pairs of 8192, then 20k
    steps of batch 4096), wall time of each phase."""
    import torch
    from rapidsfm_b200 import learned_hash as lh
    t0 = time.perf_counter()
    times = {}
    params = lh.train_from_brute_force(log=lambda m: times.setdefault("log", []).append(m), timings=times)
    torch.cuda.synchronize()
    times["total_s"] = time.perf_counter() - t0
    return params, times


def run_ransac(dev, stream, n_pairs=1000, n=4000, seed=6, cpu_pairs=8):
    """RANSAC match filter (the step after matching) on n_pairs image pairs of n matches each
    (1600x1200, 60 % inliers, 16 cell columns, 256 tests, tryOtherAffines as in the reference's
    default config): all pairs in one batched device call vs one call per pair; the CPU oracle
    (one thread) on a sample of pairs beside it. Work unit: inlier tests (one affine applied to one
    match), counted from the cell bounds."""
    import torch
    from oracle import oracle as orc  # CPU comparison leg only
    from rapidsfm_b200 import ransac, synth
    rng = np.random.default_rng(seed)
    tasks, host, tests = [], [], 0
    for k in range(n_pairs):
        pairs, _ = synth.make_ransac_matches(n, inlier_frac=0.6, seed=int(rng.integers(1 << 30)))
        sp, bounds, _, cols, rows, cw = ransac.bin_matches(1600, 1200, pairs)
        thr = float(np.float32(cw) * np.float32(0.15))
        votes, aff = ransac.device_buffers(n, cols, rows, device=dev)
        tasks.append(dict(votes=votes, affines=aff, matches=torch.from_numpy(sp).to(dev),
                          bounds=torch.from_numpy(bounds.view(np.int32)).to(dev), cols=cols, rows=rows, threshold=thr))
        if k < cpu_pairs:
            host.append((sp, bounds, cols, rows, thr))
        padded = np.pad(np.diff(bounds).astype(np.int64).reshape(rows, cols), 1)
        hood = sum(padded[dy:dy + rows, dx:dx + cols] for dy in range(3) for dx in range(3)).ravel()
        tests += int((hood[hood >= 9] * 256).sum() + hood.sum() * cols * rows + hood.sum())
    batch_ms = _events_ms(lambda: ransac.ransac_match_filter_batch(tasks, try_other=True, seed=1, stream=stream), 5,
                          stream)
    single_ms = _events_ms(lambda: [ransac.ransac_match_filter(t["votes"], t["affines"], t["matches"], t["bounds"],
                                                               t["cols"], t["rows"], 256, t["threshold"], True, 1,
                                                               stream) for t in tasks[:100]], 3, stream) * n_pairs / 100
    t0 = time.perf_counter()
    for sp, bounds, cols, rows, thr in host:
        orc.ransac_votes(sp, bounds, cols, rows, 256, thr, True, 1)
    cpu_s = (time.perf_counter() - t0) / len(host)
    return {"pairs": n_pairs, "matches_per_pair": n, "batched_ms": batch_ms,
            "pairs_per_s": n_pairs / (batch_ms * 1e-3), "one_call_per_pair_ms": single_ms,
            "inlier_tests_per_s": tests / (batch_ms * 1e-3),
            "cpu_oracle_1_thread_pairs_per_s": 1.0 / cpu_s, "cpu_sample_pairs": len(host)}


def R_lib():
    from rapidsfm_b200 import _lib
    return _lib.load()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=0, help="descriptors per side (smaller profiling cases)")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and cascade-hash sections")
    ap.add_argument("--cascade-pairs", type=int, default=1000)
    ap.add_argument("--only-hash", action="store_true", help="run the hashing-throughput section alone (profiling)")
    ap.add_argument("--only-cascade", action="store_true", help="run the cascade-hash section alone (profiling)")
    ap.add_argument("--only-ransac", action="store_true", help="run the RANSAC-filter section alone (profiling)")
    ap.add_argument("--ransac-pairs", type=int, default=1000)
    ap.add_argument("--hash-log2", type=int, default=24, help="log2 of the descriptors in the hashing section")
    ap.add_argument("--only-train", action="store_true", help="run the trainer-throughput section alone")
    ap.add_argument("--full-training", default="",
                    help="run the learned hash's whole training (200 pairs, 20k steps), time it and save the "
                         "parameter block to this path")
    args = ap.parse_args()
    if args.only_train or args.full_training:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        out = {"training": run_training(dev, torch.cuda.current_stream(dev))}
        if args.full_training:
            params, times = run_full_training(dev)
            np.save(args.full_training, params)
            out["full_training"] = times
        print(json.dumps(out), flush=True)
        return
    if args.only_ransac:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"ransac": run_ransac(dev, torch.cuda.current_stream(dev), n_pairs=args.ransac_pairs)}),
              flush=True)
        return
    if args.only_cascade:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"cascade": run_cascade(dev, torch.cuda.current_stream(dev), n_pairs=args.cascade_pairs)}),
              flush=True)
        return
    if args.only_hash:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"hash": run_hash(dev, torch.cuda.current_stream(dev), n=1 << args.hash_log2)}), flush=True)
        return
    if args.size:
        globals().update(N_QUERY=args.size, N_TRAIN=args.size, WORKLOAD=f"bf_pair_{args.size}x{args.size}")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
