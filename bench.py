#!/usr/bin/env python3
"""Benchmark: bit-exact Goldilocks coset LDE on B200.

Workload (one step): coset LDE of 128 columns x 2^22 Goldilocks words,
uniform in [0, p), bit-reversed evaluations in, blowup 2 (two cosets of
128 x 2^22 out, 8 GiB), bit-reversed output -- inverse NTT, coset shift by
g = 7, forward NTT.  Inputs (4 GiB) and outputs are far larger than L2, so
no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours       the fused LDE (bc_lde_fused) through the C ABI; also reports the
           plain composition (bc_lde_plain), per-step p50/p99, the dominant
           kernel's roofline and a CPU baseline (oracle, host cores).
reference  the reference's own CUDA kernels (native/ntt.cu, compiled for
           sm_100a into oracle/_ref/libref_ntt.so) driven exactly as its
           callers drive them: one inverse batch_ntt then one forward
           batch_ntt per coset.
One JSON line on stdout (rank 0).  For N > 1 (torchrun) every rank runs the
same per-GPU workload (weak scaling, no collective on the data path); the
time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "era-boojum-cuda_b200"))

P = 0xFFFFFFFF00000001
METRIC = "bit-exact Goldilocks LDE Melem/s: batched vs plain, % HBM roofline; p99 ms"
LOG_N, COLS, LOG_BLOWUP = 22, 128, 1
L2_BYTES = 126 * 2**20  # B200 L2
SPEC_HBM_GBS = 8000.0  # B200 HBM3e specification (DGX figure), for the spec fraction beside the measured one


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def l2_note() -> str:
    """How the timed LDE relates to the 126 MB L2 (inputs and outputs of the configured workload)."""
    n_in = 8 * COLS * (1 << LOG_N)
    n_out = n_in << LOG_BLOWUP
    fmt = lambda b: f"{b / 2**30:g} GiB" if b >= 2**30 else f"{b / 2**20:g} MiB"  # noqa: E731
    if n_in > L2_BYTES:
        return f"inputs {fmt(n_in)} and outputs {fmt(n_out)}, larger than L2; no flush"
    return f"inputs {fmt(n_in)} and outputs {fmt(n_out)}; inputs fit in L2 (a small case, not the bench workload)"


def measured_traffic(log_n: int, log_blowup: int, cols: int):
    """DRAM bytes of one top-window launch from the committed ncu summary, scaled to `cols` columns, and the
    ALU / FMA pipe utilisation (% of peak) of that capture: (bytes, alu_pct, fma_pct), Nones if absent."""
    path = os.path.join(ROOT, "profiles", f"lde_top_kernel_traffic_logn{log_n}_blowup{1 << log_blowup}.txt")
    try:
        for line in open(path):
            if line.startswith("kernel="):
                kv = dict(tok.split("=", 1) for tok in line.split())
                if int(kv["log_n"]) == log_n and int(kv["log_blowup"]) == log_blowup:
                    byts = round((int(kv["dram_read"]) + int(kv["dram_write"])) * cols / int(kv["cols"]))
                    alu, fma = kv.get("alu_pipe_pct"), kv.get("fma_pipe_pct")
                    return byts, float(alu) if alu else None, float(fma) if fma else None
    except OSError:
        pass
    return None, None, None


class ClockSampler:
    """SM clock / throttle-reason samples during the timed region, read in-process through NVML.

    (A polling nvidia-smi subprocess was seen to stall the GPU for hundreds of ms.)"""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self.error = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception as e:  # no NVML: report it instead of clocks
            self.nv = None
            self.error = str(e)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h) if hasattr(
                    nv, "nvmlDeviceGetCurrentClocksEventReasons") else nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.samples.append((float(sm), int(r)))
            except Exception as e:
                self.error = str(e)
                return
            self._stop.wait(0.05)

    def __enter__(self):
        if self.nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"no samples: {self.error}"]}
        sm = sorted(s for s, _ in self.samples)
        reasons = sorted({k for _, r in self.samples for k, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.max_mhz, "reasons": reasons, "samples": len(sm),
                "source": "NVML"}


def dist_setup(gpus: int):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier_max(value: float, world: int) -> float:
    """Max of a per-rank value over all ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world: int, steps: int, units_per_rank_step: int, max_total_ms: float) -> float:
    """Whole-job throughput in M units/s: every rank processes its own units (weak scaling), the time is
    the max over ranks of the timed region."""
    return world * steps * units_per_rank_step / (max_total_ms / 1e3) / 1e6


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def uniform_words(count: int, seed: int, device: str = "cuda"):
    """`count` Goldilocks words uniform in [0, p), generated on the device (seeded), as int64 bit patterns.

    A word is two independent uniform 32-bit halves; the words >= p (high half 2^32 - 1 and low half non-zero,
    about one in 2^32) are drawn again until none is left, so every value in [0, p) is equally likely."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)

    def draw(k):
        hi = torch.randint(0, 2**32, (k,), device=device, dtype=torch.int64, generator=g)
        lo = torch.randint(0, 2**32, (k,), device=device, dtype=torch.int64, generator=g)
        return hi, lo

    out = torch.empty(count, device=device, dtype=torch.int64)
    chunk = 1 << 26
    for c0 in range(0, count, chunk):
        k = min(chunk, count - c0)
        hi, lo = draw(k)
        bad = ((hi == 2**32 - 1) & (lo != 0)).nonzero().flatten()
        while bad.numel():
            h2, l2 = draw(bad.numel())
            hi[bad], lo[bad] = h2, l2
            bad = bad[(h2 == 2**32 - 1) & (l2 != 0)]
        # the high half as a signed 32-bit value keeps the product inside int64
        out[c0:c0 + k] = torch.where(hi >= 2**31, hi - 2**32, hi) * 2**32 + lo
    return out


def make_inputs(seed: int):
    """128 x 2^22 words uniform in [0, p) generated on the device (seeded)."""
    return uniform_words(COLS << LOG_N, seed)


def time_steps(fn, steps: int, warmup: int, world: int, stream):
    """W untimed steps, then K steps between barriers; returns (total ms max over ranks, per-step ms)."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(stream)
    for i in range(steps):
        fn()
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    per = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
    total = evs[0].elapsed_time(evs[-1])
    barrier(world)
    return barrier_max(total, world), per


def plan_windows(log_n: int, log_blowup: int):
    """Window bits of the pass plan the fused LDE uses (top window first), from the loaded plan table; None
    when the table has no entry (the library's built-in plan)."""
    import bc_ntt

    for line in bc_ntt.plan_table_export().splitlines():
        f = line.split()
        if len(f) >= 3 and int(f[0]) == log_n and int(f[1]) == log_blowup:
            return [int(f[3 + 2 * i]) for i in range(int(f[2]))]
    return None


def lde_kernel_butterflies(windows, log_n: int, cols: int, log_blowup: int):
    """Radix-2 butterflies of each kernel of the fused LDE, in launch order: the inverse passes below the top
    window (bottom-up), the top-window kernel (inverse stages once, forward stages for every coset), the forward
    passes below it (every coset)."""
    half, B = (1 << log_n) // 2 * cols, 1 << log_blowup
    below = windows[1:]
    return ([k * half for k in reversed(below)] + [windows[0] * (1 + B) * half] + [k * B * half for k in below])


def butterfly_peak(target_ms: float = 10.0, reps: int = 5):
    """Butterflies per second of the transform kernels' round arithmetic alone, from registers, in every resident
    thread slot (bc_butterfly_peak): the 32-bit integer issue roofline.  Best of `reps` short launches (about
    `target_ms` each, 50 ms apart: a long run of this loop reaches the board's power cap and lowers the SM clock,
    which the transform kernels, with their memory phases, do not), CUDA events on the current stream.
    Returns (G butterflies/s, launch ms, SM clock samples around the launches)."""
    import ctypes

    import torch

    import bc_ntt

    L = bc_ntt.lib()
    words = ctypes.c_size_t(0)
    assert L.bc_butterfly_peak_words(ctypes.byref(words)) == 0
    out = torch.empty(words.value, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    bfly = ctypes.c_uint64(0)

    def launch(iters):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rc = L.bc_butterfly_peak(out.data_ptr(), words.value, iters, stream.cuda_stream, ctypes.byref(bfly))
        assert rc == 0, rc
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    iters = 64
    ms = launch(iters)
    ms = launch(iters)
    iters = max(1, int(iters * target_ms / max(ms, 1e-3)))
    best = None
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(reps):
            time.sleep(0.05)
            ms = launch(iters)
            rate = bfly.value / (ms / 1e3) / 1e9
            best = (rate, ms) if best is None or rate > best[0] else best
    del out
    return best[0], best[1], clk.summary()


def lde_matches_fused(ev, out, log_n: int, cols: int, log_blowup: int, chunk_words: int = 1 << 28) -> bool:
    """True when `out`, the dense coset-major LDE of `ev` (device tensors), equals bc_lde_fused's result bit for
    bit.  The reference result is computed again column chunk by column chunk into a scratch buffer of at most
    `chunk_words` words, so any job size is checked in bounded memory."""
    import torch

    import bc_ntt

    L = bc_ntt.lib()
    n, B = 1 << log_n, 1 << log_blowup
    chunk = max(1, min(cols, chunk_words // (B * n)))
    tmp = torch.empty(B * chunk * n, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    view = out.view(B, cols, n)
    for c0 in range(0, cols, chunk):
        k = min(chunk, cols - c0)
        rc = L.bc_lde_fused(ev.data_ptr() + 8 * c0 * n, tmp.data_ptr(), log_n, k, n, n, k * n, log_blowup, s)
        assert rc == 0, rc
        if not torch.equal(view[:, c0:c0 + k], tmp[:B * k * n].view(B, k, n)):
            return False
    return True


def pct(xs, q):
    s = sorted(xs)
    return s[min(len(s) - 1, int(round(q / 100.0 * (len(s) - 1))))]


def cpu_baseline(threads: int, budget_s: float = 12.0):
    """Oracle LDE (C restatement, all host threads) on a bounded sample of whole columns."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    n = 1 << LOG_N
    rng = np.random.default_rng(42)
    cols = threads
    x = rng.integers(0, P, size=cols * n, dtype=np.uint64)
    t0 = time.perf_counter()
    oracle.lde(x, LOG_N, cols, n, LOG_BLOWUP, threads=threads)
    dt = time.perf_counter() - t0
    reps = max(1, int(budget_s / max(dt, 1e-3)) - 1)
    t0 = time.perf_counter()
    for _ in range(reps):
        oracle.lde(x, LOG_N, cols, n, LOG_BLOWUP, threads=threads)
    dt = (time.perf_counter() - t0) / reps
    out_elems = (1 << LOG_BLOWUP) * n * cols
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            model = next((ln.split(":", 1)[1].strip() for ln in f if ln.startswith("model name")), model)
    except OSError:
        pass
    return {"value": out_elems / dt / 1e6, "unit": "Melem/s", "cores": threads, "kind": "port",
            "nproc": os.cpu_count(), "cpu_model": model,
            "sample": f"{cols} of {COLS} columns (2^{LOG_N}, blowup {1 << LOG_BLOWUP}) x {reps} reps, "
                      f"{dt:.2f} s each; oracle/gl_oracle.c, one column per thread"}


def run_small_ntt_section(call, reps: int = 200, log_n: int = 16, cols: int = 16):
    """Plain forward NTT (natural in, bit-reversed out, no coset) of 16 columns x 2^16: a latency-bound call.
    Device time of each call (CUDA events around it) over `reps` calls, and `reps` calls issued back to back
    under one event pair; `call(in_ptr, out_ptr, log_n, cols, stream)`.  The 8 MiB of columns stay in L2, as
    they do for a caller that issues this call repeatedly."""
    import torch

    n = 1 << log_n
    stream = torch.cuda.current_stream()
    x = uniform_words(cols * n, 16)
    y = torch.empty_like(x)
    for _ in range(20):
        call(x.data_ptr(), y.data_ptr(), log_n, cols, stream.cuda_stream)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for a, b in evs:
        a.record(stream)
        call(x.data_ptr(), y.data_ptr(), log_n, cols, stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
    per_us = [a.elapsed_time(b) * 1e3 for a, b in evs]
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        call(x.data_ptr(), y.data_ptr(), log_n, cols, stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    b2b_us = a.elapsed_time(b) * 1e3 / reps
    del x, y
    return {"workload": f"forward NTT {cols} cols x 2^{log_n}, natural -> bit-reversed", "reps": reps,
            "p50_us": round(pct(per_us, 50), 2), "p99_us": round(pct(per_us, 99), 2),
            "back_to_back_us": round(b2b_us, 2), "melem_per_s": round(cols * n / b2b_us, 1),
            "l2": "8 MiB of columns, L2-resident across calls"}


def copy_floor_ms(h_in, d_in, d_out, h_out, stream, reps: int = 3) -> float:
    """The e2e leg's host<->device copies alone: the whole input host->device and the whole output
    device->host, issued at once on two streams (full-duplex PCIe), no transform; the best of `reps`."""
    import torch

    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = None
    for i in range(reps + 1):
        torch.cuda.synchronize()
        a.record(stream)
        s_in.wait_stream(stream)
        s_out.wait_stream(stream)
        with torch.cuda.stream(s_in):
            d_in.copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s_out):
            h_out.copy_(d_out, non_blocking=True)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)
        b.record(stream)
        torch.cuda.synchronize()
        if i > 0:
            best = a.elapsed_time(b) if best is None else min(best, a.elapsed_time(b))
    return best


def run_ours(args, rank, world):
    import ctypes

    import torch

    import bc_ntt

    n = 1 << LOG_N
    B = 1 << LOG_BLOWUP
    L = bc_ntt.lib()
    bc_ntt.Context.create(12, 12)
    tuned = bc_ntt.load_tuned_plans() if not args.no_tuned_plans else False
    stream = torch.cuda.current_stream()
    s_handle = stream.cuda_stream
    x = make_inputs(1234 + rank)
    out = torch.empty(B * COLS * n, device="cuda", dtype=torch.int64)
    xp, op = x.data_ptr(), out.data_ptr()

    def fused():  # noqa: E306
        rc = L.bc_lde_fused(xp, op, LOG_N, COLS, n, n, COLS * n, LOG_BLOWUP, s_handle)
        assert rc == 0, rc

    def plain():
        rc = L.bc_lde_plain(xp, op, LOG_N, COLS, n, n, COLS * n, LOG_BLOWUP, s_handle)
        assert rc == 0, rc

    # result of one fused step for the bit-exactness spot check against the plain path
    fused()
    torch.cuda.synchronize()
    ref_sum = out.clone()
    plain()
    torch.cuda.synchronize()
    bit_exact_vs_plain = bool(torch.equal(ref_sum, out))
    del ref_sum

    # the integer roofline first, on a GPU that has not yet run at full power for long
    peak_bfly, peak_ms, peak_clocks = butterfly_peak()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        total_ms, per = time_steps(fused, args.steps, args.warmup, world, stream)
    plain_ms, plain_per = time_steps(plain, max(3, args.steps // 2), 1, world, stream)

    out_elems = B * n * COLS
    value = whole_job_value(world, args.steps, out_elems, total_ms)
    ms_per_step = total_ms / args.steps

    # dominant kernel: per-kernel durations from events recorded between the fused LDE's launches
    nk = ctypes.c_uint32(0)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(8)]
    kern_ms = None
    for e in evs:
        e.record(stream)  # torch creates the CUDA event on first record
    torch.cuda.synchronize()
    ev_handles = (ctypes.c_void_p * 8)(*[e.cuda_event for e in evs])
    if all(ev_handles):
        reps = 3
        acc = None
        for _ in range(reps):
            rc = L.bc_lde_fused_profiled(xp, op, LOG_N, COLS, n, n, COLS * n, LOG_BLOWUP, s_handle,
                                         ctypes.cast(ev_handles, ctypes.c_void_p), 8, ctypes.byref(nk))
            assert rc == 0
            torch.cuda.synchronize()
            d = [evs[i].elapsed_time(evs[i + 1]) for i in range(nk.value)]
            acc = d if acc is None else [a + b for a, b in zip(acc, d)]
        kern_ms = [a / reps for a in acc]

    peak, peak_kind = measured_peaks()
    # bytes each kernel of the fused plan must move: inverse passes below the top window read+write the
    # columns; the top-window kernel reads them once and writes every coset; the forward passes below the
    # top window read+write every coset
    col_bytes = 8 * n * COLS
    npass = (nk.value + 1) // 2 if nk.value else 1
    kernels = ([(f"lde inverse pass {i} (b2n)", 2 * col_bytes) for i in range(npass - 1)]
               + [("lde_top_kernel (inverse top window, scale, forward top window, all cosets)",
                   (1 + B) * col_bytes)]
               + [(f"lde forward pass {i} (n2b, all cosets)", 2 * B * col_bytes) for i in range(npass - 1)])
    roofline = None
    traffic, alu_pct, fma_pct = measured_traffic(LOG_N, LOG_BLOWUP, COLS)
    windows = plan_windows(LOG_N, LOG_BLOWUP)
    kbfly = lde_kernel_butterflies(windows, LOG_N, COLS, LOG_BLOWUP) if windows else None
    if kern_ms and len(kern_ms) == len(kernels):
        dom = max(range(len(kern_ms)), key=lambda i: kern_ms[i])
        name, byts = kernels[dom]
        achieved = byts / (kern_ms[dom] / 1e3) / 1e9
        top = "lde_top_kernel" in name
        # The HBM roofline of the kernel's algorithmic bytes (achieved / peak / frac) is reported as the contract
        # asks, but it does not bound these kernels: (1 + B) (n / 2) log n butterflies of 64-bit modular arithmetic
        # on 32-bit integer pipes do.  `limiter` is that roofline: butterflies per second of the kernel against
        # the same round arithmetic run from registers (bc_butterfly_peak, measured in this run).
        roofline = {"bound": "int32 issue", "kernel": name, "achieved": round(achieved, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                    "hbm_frac_note": "achieved/peak/frac: HBM roofline of the algorithmic bytes; see limiter",
                    "spec_frac": round(achieved / SPEC_HBM_GBS, 4),
                    "traffic": traffic if top else None,
                    "traffic_unit": "bytes per launch (ncu dram read+write, scaled from the profiled case)",
                    "kernel_ms": [round(v, 3) for v in kern_ms],
                    "step_algorithmic_frac": round(8 * n * COLS * (1 + B) / (ms_per_step / 1e3) / 1e9 / peak, 4)}
        if kbfly and len(kbfly) == len(kern_ms):
            rates = [b / (t / 1e3) / 1e9 for b, t in zip(kbfly, kern_ms)]
            step_rate = sum(kbfly) / (ms_per_step / 1e3) / 1e9
            roofline["limiter"] = {
                "bound": "int32 issue", "unit": "G butterflies/s", "kernel": name,
                "achieved": round(rates[dom], 1), "peak": round(peak_bfly, 1),
                "frac": round(rates[dom] / peak_bfly, 4),
                "per_kernel_achieved": [round(r, 1) for r in rates],
                "step_achieved": round(step_rate, 1), "step_frac": round(step_rate / peak_bfly, 4),
                "butterflies_per_step": sum(kbfly), "plan_windows": windows,
                "peak_source": f"bc_butterfly_peak: the kernels' radix-16 round arithmetic from registers, every "
                               f"resident thread slot, best of 5 launches of {peak_ms:.1f} ms, this run",
                "peak_clocks": peak_clocks,
                "alu_pipe_pct": alu_pct, "fma_pipe_pct": fma_pct,
                "pipe_source": "ncu of the top-window kernel and of the round loop, "
                               "profiles/int32_roofline_butterfly_peak_and_lde_kernels_8cols_logn22_blowup2.md"}

    # end to end through the C ABI with host buffers: bc_lde_host takes pinned host input and writes pinned
    # host output every step, overlapping chunked copy-in / transform / copy-out on three streams
    hx = torch.empty(COLS * n, dtype=torch.int64, pin_memory=True)
    hx.copy_(x)
    hout = torch.empty(B * COLS * n, dtype=torch.int64, pin_memory=True)
    chunk_cols = max(1, min(COLS, 8))
    ws = torch.empty(3 * chunk_cols * n * (1 + B), dtype=torch.int64, device="cuda")

    def e2e_step():
        rc = L.bc_lde_host(hx.data_ptr(), hout.data_ptr(), LOG_N, COLS, n, n, COLS * n, LOG_BLOWUP, ws.data_ptr(),
                           ws.numel() * 8, chunk_cols, s_handle)
        assert rc == 0, rc

    e2e_steps = max(2, min(args.steps, 5))
    e2e_ms, _ = time_steps(e2e_step, e2e_steps, 1, world, stream)
    e2e_value = world * e2e_steps * out_elems / (e2e_ms / 1e3) / 1e6
    # the result must be the device LDE's, bit for bit (checked on the last step's host output)
    fused()
    torch.cuda.synchronize()
    e2e_exact = bool(torch.equal(hout, out.cpu())) if COLS * n <= (1 << 30) else None
    floor_ms = copy_floor_ms(hx, x, out, hout, stream)

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "Melem/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64 (Goldilocks)", "data": "synthetic",
        "config": {"workload": f"coset LDE {COLS} cols x 2^{LOG_N}, blowup {B}, bit-reversed in/out",
                   "log_n": LOG_N, "columns": COLS, "blowup": B, "path": "bc_lde_fused",
                   "plans": "autotuned (era-boojum-cuda_b200/plans_b200.txt)" if tuned else "built-in",
                   "l2": l2_note(), "parallelism": f"replicas x{world}"},
        "p50_ms": round(pct(per, 50), 4), "p99_ms": round(pct(per, 99), 4),
        "plain": {"value": round(world * len(plain_per) * out_elems / (plain_ms / 1e3) / 1e6, 1),
                  "ms_per_step": round(plain_ms / len(plain_per), 4), "path": "bc_lde_plain",
                  "bit_exact_vs_fused": bit_exact_vs_plain},
        "roofline": roofline,
        "clocks": clk.summary(),
        "e2e": {"value": round(e2e_value, 1), "unit": "Melem/s", "h2d_bytes_per_step": 8 * COLS * n,
                "d2h_bytes_per_step": 8 * B * COLS * n, "ms_per_step": round(e2e_ms / e2e_steps, 3),
                "path": f"bc_lde_host: pinned host in/out, {chunk_cols}-column chunks, copies overlapped",
                "bit_exact_vs_device": e2e_exact, "copy_floor_ms": round(floor_ms, 3),
                "frac_of_copy_floor": round(floor_ms / (e2e_ms / e2e_steps), 4)},
        "gpu_launches": args.steps * (len(kern_ms) if kern_ms else 3),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(os.cpu_count() or 1)
    del x, out, hx, hout, ws
    torch.cuda.empty_cache()
    if world == 1:
        def small_call(a, b, log_n, cols, s):
            rc = L.bc_batch_ntt_internal(a, b, log_n, cols, 1 << log_n, 1 << log_n, False, False, 0, 0, s)
            assert rc == 0, rc

        line["small_ntt"] = run_small_ntt_section(small_call)
    torch.cuda.empty_cache()
    if world == 1 and not args.no_batch:
        line["batch"] = run_batch_section()
        line["batch_small_jobs"] = run_small_batch_section()
    if world == 1 and not args.no_large:
        line["large"] = run_large_section()
    if world == 1 and not args.no_serve:
        line["serve"] = run_serve_section()
        line["serve_device"] = run_serve_device_section()
    if world == 1 and not args.no_ops:
        line["ops"] = run_ops_section(ops_ours(), log_n=args.ops_log_n)
    return line


def _uneven_tensors(specs):
    import torch

    tens = []
    for sp in specs:
        ev = uniform_words(sp.in_words, sp.seed)
        tens.append((ev, torch.empty(sp.out_words, dtype=torch.int64, device="cuda"), sp.log_n, sp.cols,
                     sp.log_blowup))
    return tens


def run_batch_section(reps: int = 3):
    """96 seeded uneven LDE jobs: one persistent launch vs one call per job (fused, plain)."""
    import torch

    import bc_ntt
    import workloads

    specs = workloads.uneven_batch(n_jobs=96, seed=42)
    tens = _uneven_tensors(specs)
    plan = bc_ntt.LdeBatch(tens)
    stream = torch.cuda.current_stream()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    out_elems = sum(sp.out_words for sp in specs)
    t_batch = timed(plan.run)
    status = plan.status()
    # every output of every job, bit for bit against the same job alone through bc_lde_fused
    exact_persistent = sum(lde_matches_fused(*t) for t in tens)
    # hybrid: jobs whose kernels span >= 4 waves of CTAs run as their own kernels in the same graph
    hybrid = bc_ntt.LdeBatch(tens, standalone_min_ctas=4 * 2 * torch.cuda.get_device_properties(0).multi_processor_count)
    for t in tens:
        t[1].zero_()
    t_hybrid = timed(hybrid.run)
    status |= hybrid.status()
    hybrid.close()
    exact_hybrid = sum(lde_matches_fused(*t) for t in tens)
    t_fused = timed(lambda: [bc_ntt.lde(*t, fused=True) for t in tens])
    t_plain = timed(lambda: [bc_ntt.lde(*t, fused=False) for t in tens])
    info = plan.info()
    plan.close()
    # the jobs the reference's kernels can run (log_n + log2 B <= 24): the same paths, for the reference arm's
    # per-job composition on the same subset
    sub = [t for t, sp in zip(tens, specs) if reference_can_run(sp)]
    sub_plan = bc_ntt.LdeBatch(sub)
    t_sub_batch = timed(sub_plan.run)
    status |= sub_plan.status()
    sub_plan.close()
    t_sub_fused = timed(lambda: [bc_ntt.lde(*t, fused=True) for t in sub])
    t_sub_plain = timed(lambda: [bc_ntt.lde(*t, fused=False) for t in sub])
    sub_elems = sum(sp.out_words for sp in specs if reference_can_run(sp))
    del sub
    del tens
    torch.cuda.empty_cache()
    mel = lambda ms: round(out_elems / (ms / 1e3) / 1e6, 1)  # noqa: E731
    return {"workload": "96 jobs, log_n U{12..22}, cols log-U[1,256], blowup U{2,4,8}, seed 42",
            "bit_exact_all_96": exact_persistent == len(specs) and exact_hybrid == len(specs),
            "jobs_exact": {"persistent": exact_persistent, "hybrid": exact_hybrid, "of": len(specs),
                           "against": "each job alone through bc_lde_fused, every output word"},
            "total_out_gelem": round(out_elems / 1e9, 2),
            "persistent_one_launch": {"ms": round(t_batch, 2), "value": mel(t_batch), "status": status,
                                      "records": info["records"], "items": info["items"], "grid": info["grid"]},
            "hybrid_one_graph": {"ms": round(t_hybrid, 2), "value": mel(t_hybrid),
                                 "rule": "jobs with >= 4 waves of CTAs per kernel as their own kernels"},
            "per_job_fused": {"ms": round(t_fused, 2), "value": mel(t_fused)},
            "per_job_plain": {"ms": round(t_plain, 2), "value": mel(t_plain)},
            "persistent_vs_plain": round(t_plain / t_batch, 3), "hybrid_vs_plain": round(t_plain / t_hybrid, 3),
            "fused_vs_plain": round(t_plain / t_fused, 3), "unit": "Melem/s",
            "reference_subset": {"jobs": sum(reference_can_run(sp) for sp in specs), "rule": "log_n + log2 B <= 24",
                                 "out_gelem": round(sub_elems / 1e9, 3),
                                 "persistent_ms": round(t_sub_batch, 2), "per_job_fused_ms": round(t_sub_fused, 2),
                                 "per_job_plain_ms": round(t_sub_plain, 2),
                                 "note": "the reference arm times its own per-job composition on these jobs "
                                         "(batch_per_job_reference.per_job_reference_ms); vs_reference_per_job = "
                                         "that time / ours"}}


def reference_can_run(spec) -> bool:
    """The reference's kernels cover transforms with log_n + log_extension_degree <= 24 (src/context.rs:12)."""
    return spec.log_n + spec.log_blowup <= 24


def run_reference_batch_section(ref, reps: int = 3):
    """The 96-job uneven workload as the reference's callers run it, one job at a time: per job one inverse
    batch_ntt, then one forward batch_ntt per coset (src/ntt.rs:179-290; log_n < 16 goes through its per-stage
    launches), on the jobs its kernels cover (log_n + log2 B <= 24)."""
    import torch

    import workloads

    specs = [sp for sp in workloads.uneven_batch(n_jobs=96, seed=42) if reference_can_run(sp)]
    tens = _uneven_tensors(specs)
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream

    def job(ev, out, log_n, cols, log_b):
        n, B = 1 << log_n, 1 << log_b
        coef = out.data_ptr() + 8 * (B - 1) * cols * n
        ref.batch_ntt(ev.data_ptr(), coef, log_n, cols, n, n, True, True, 0, 0, s)
        for k in range(B):
            ref.batch_ntt(coef, out.data_ptr() + 8 * k * cols * n, log_n, cols, n, n, False, False, log_b, k, s)

    def all_jobs():
        for t in tens:
            job(*t)

    all_jobs()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        all_jobs()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    out_elems = sum(sp.out_words for sp in specs)
    del tens
    torch.cuda.empty_cache()
    return {"workload": "the 96-job uneven batch (seed 42), jobs with log_n + log2 B <= 24", "jobs": len(specs),
            "out_gelem": round(out_elems / 1e9, 3), "per_job_reference_ms": round(ms, 2),
            "value": round(out_elems / (ms / 1e3) / 1e6, 1), "unit": "Melem/s"}


def run_small_batch_section(reps: int = 5):
    """Many small uneven jobs (log_n 10..16, 1..8 columns): where one launch per job is launch-bound."""
    import torch

    import bc_ntt
    import workloads

    specs = workloads.uneven_batch(n_jobs=256, seed=11, log_n_range=(10, 16), cols_range=(1, 8))
    tens = _uneven_tensors(specs)
    plan = bc_ntt.LdeBatch(tens)
    stream = torch.cuda.current_stream()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    out_elems = sum(sp.out_words for sp in specs)
    t_batch = timed(plan.run)
    status = plan.status()
    first = [t[1].clone() for t in tens]
    t_fused = timed(lambda: [bc_ntt.lde(*t, fused=True) for t in tens])
    exact = all(torch.equal(a, t[1]) for a, t in zip(first, tens))
    t_plain = timed(lambda: [bc_ntt.lde(*t, fused=False) for t in tens])
    plan.close()
    del tens, first
    torch.cuda.empty_cache()
    mel = lambda ms: round(out_elems / (ms / 1e3) / 1e6, 1)  # noqa: E731
    return {"workload": "256 jobs, log_n U{10..16}, cols log-U[1,8], blowup U{2,4,8}, seed 11",
            "persistent_one_launch": {"ms": round(t_batch, 3), "value": mel(t_batch), "status": status},
            "per_job_fused": {"ms": round(t_fused, 3), "value": mel(t_fused)},
            "per_job_plain": {"ms": round(t_plain, 3), "value": mel(t_plain)},
            "persistent_vs_plain": round(t_plain / t_batch, 2), "persistent_vs_fused": round(t_fused / t_batch, 2),
            "bit_exact_persistent_vs_per_job": bool(exact), "unit": "Melem/s"}


def run_large_section(reps: int = 5):
    """64 columns x 2^23 at blowup 4 (16 GiB out): fused vs the unfused plain composition."""
    import torch

    import bc_ntt

    log_n, cols, log_b = 23, 64, 2
    n, B = 1 << log_n, 1 << log_b
    x = uniform_words(cols * n, 77)
    out = torch.empty(B * cols * n, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fused):
        bc_ntt.lde(x, out, log_n, cols, log_b, fused=fused)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            bc_ntt.lde(x, out, log_n, cols, log_b, fused=fused)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    t_f = timed(True)
    ref = out.clone()
    t_p = timed(False)
    exact = bool(torch.equal(ref, out))
    del x, out, ref
    torch.cuda.empty_cache()
    peak, _ = measured_peaks()
    alg = 8 * n * cols * (1 + B)
    return {"workload": "coset LDE 64 cols x 2^23, blowup 4 (16 GiB out)",
            "fused_ms": round(t_f, 3), "plain_ms": round(t_p, 3), "fused_vs_plain": round(t_p / t_f, 3),
            "fused_value": round(B * n * cols / (t_f / 1e3) / 1e6, 1), "unit": "Melem/s",
            "fused_hbm_frac": round(alg / (t_f / 1e3) / 1e9 / peak, 4),
            "plain_hbm_frac": round(alg / (t_p / 1e3) / 1e9 / peak, 4), "bit_exact_fused_vs_plain": exact}


def run_ops_section(ops, reps: int = 5, note: str | None = None, log_n: int = 28):
    """The ops beside the NTT (include/bc_ops.h; src/ops_complex.rs) on HBM-sized inputs.

    `ops` maps an op name to a callable (src_ptr, dst_ptr, aux, stream) -> None: this library's entry points
    in the ours arm, the reference's own kernels in the reference arm, on the same workloads (`aux`: pointers of
    the smaller buffers).  Every op is bound by HBM traffic: 16 bytes per element for the bit reversal and the
    omega shift (read + write), 8 for the powers (write only), 16 per extension coefficient written by the
    barycentric precompute, 8 per value read by the barycentric evaluation (64 polynomials x 2^22 rows);
    achieved = those bytes / event-timed duration, frac of the measured copy peak.
    """
    import torch

    peak, peak_kind = measured_peaks()
    n_vec = 1 << log_n                    # 2 GiB of u64 at the default 2^28, larger than L2
    log_rows, cols = 22, n_vec >> 22      # bit reversal / batch evaluation: cols x 2^22 rows
    n_coef = 1 << min(24, log_n - 4)      # barycentric coefficients
    a = torch.randint(-(2**63), 2**63 - 1, (n_vec,), device="cuda", dtype=torch.int64,
                      generator=torch.Generator(device="cuda").manual_seed(5))
    b = torch.empty_like(a)
    small = {"x": torch.tensor([12345678901, 98765432109], dtype=torch.int64, device="cuda"),
             "cf": torch.zeros(2, dtype=torch.int64, device="cuda"),
             "coef": torch.zeros(2 * max(n_coef, 1 << log_rows), dtype=torch.int64, device="cuda"),
             # the reference's partial matrix: 32 * ceil(2^22 / 192) rows x cols x 2 words
             "partial": torch.zeros(2 * cols * 32 * (((1 << log_rows) + 191) // 192), dtype=torch.int64,
                                    device="cuda"),
             "evals": torch.zeros(128, dtype=torch.int64, device="cuda")}
    aux = {k: v.data_ptr() for k, v in small.items()}
    aux["partial_words"] = small["partial"].numel()
    aux.update(n=n_vec, rows=1 << log_rows, log_rows=log_rows, cols=cols, n_coef=n_coef)
    stream = torch.cuda.current_stream()
    work = {  # name -> (elements, bytes per element, workload)
        "bit_reverse": (cols << log_rows, 16, f"{cols} cols x 2^{log_rows}, out of place"),
        "bit_reverse_in_place": (cols << log_rows, 16, f"{cols} cols x 2^{log_rows}, in place"),
        "omega_shift": (n_vec, 16, f"2^{log_n} elements, log_degree 24, shift 3"),
        "get_powers_of_w": (n_vec, 8, f"2^{log_n} elements, log_degree 24"),
        "get_powers_of_g": (n_vec, 8, f"2^{log_n} elements, log_degree 24"),
        "get_powers_by_val_bf": (n_vec, 8, f"2^{log_n} elements, base 42"),
        "barycentric_precompute_at_ext": (n_coef, 16, f"2^{min(24, log_n - 4)} coefficients at an extension point, "
                                                       "bit-reversed"),
        "batch_eval_base_at_base": (n_vec, 8, f"{cols} polynomials x 2^{log_rows} rows at a base point"),
        "batch_eval_base_at_ext": (n_vec, 8, f"{cols} polynomials x 2^{log_rows} rows at an extension point"),
    }
    res = {}
    for name, fn in ops.items():
        elems, bpe, workload = work[name]
        fn(a.data_ptr(), b.data_ptr(), aux, stream.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn(a.data_ptr(), b.data_ptr(), aux, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = elems * bpe / (ms / 1e3) / 1e9
        res[name] = {"workload": workload, "ms": round(ms, 4), "gelem_per_s": round(elems / (ms / 1e3) / 1e9, 2),
                     "achieved_gbs": round(gbs, 1), "hbm_frac": round(gbs / peak, 4)}
    del a, b, small
    torch.cuda.empty_cache()
    res["peak_gbs"] = peak
    res["peak_kind"] = peak_kind
    if note:
        res["note"] = note
    return res


def ops_ours():
    """This library's ops, as run_ops_section callables (sizes from aux)."""
    import bc_ntt

    L = bc_ntt.lib()

    def ck(rc):
        assert rc == 0, rc

    return {
        "bit_reverse": lambda a, b, x, s: ck(L.bc_bit_reverse(a, x["rows"], b, x["rows"], x["log_rows"], x["cols"], s)),
        "bit_reverse_in_place": lambda a, b, x, s: ck(L.bc_bit_reverse_in_place(a, x["rows"], x["log_rows"], x["cols"],
                                                                                s)),
        "omega_shift": lambda a, b, x, s: ck(L.bc_omega_shift(a, 24, 0, False, 3, b, x["n"], s)),
        "get_powers_of_w": lambda a, b, x, s: ck(L.bc_get_powers_of_w(24, 0, False, False, b, x["n"], s)),
        "get_powers_of_g": lambda a, b, x, s: ck(L.bc_get_powers_of_g(24, 0, False, False, b, x["n"], s)),
        "get_powers_by_val_bf": lambda a, b, x, s: ck(L.bc_get_powers_by_val_bf(42, 0, False, b, x["n"], s)),
        "barycentric_precompute_at_ext": lambda a, b, x, s: ck(L.bc_precompute_lagrange_coeffs_at_ext(
            x["x"], x["cf"], 7, x["coef"], x["n_coef"], True, s)),
        "batch_eval_base_at_base": lambda a, b, x, s: ck(L.bc_batch_eval(
            0, a, x["rows"], x["cols"], x["coef"], x["partial"], x["partial_words"], None, 0, x["evals"], s)),
        "batch_eval_base_at_ext": lambda a, b, x, s: ck(L.bc_batch_eval(
            1, a, x["rows"], x["cols"], x["coef"], x["partial"], x["partial_words"], None, 0, x["evals"], s)),
    }


def ops_reference(ref):
    """The reference's own ops kernels (oracle.RefKernels), as run_ops_section callables.  Its batch_eval
    is timed by its partial-reduce kernel alone: the column sums that follow are a CUB call on its Rust side."""
    return {
        "bit_reverse": lambda a, b, x, s: ref.bit_reverse(a, x["rows"], b, x["rows"], x["log_rows"], x["cols"], s),
        "bit_reverse_in_place": lambda a, b, x, s: ref.bit_reverse(a, x["rows"], a, x["rows"], x["log_rows"],
                                                                   x["cols"], s),
        "omega_shift": lambda a, b, x, s: ref.omega_shift(a, 24, 0, False, 3, b, x["n"], s),
        "get_powers_of_w": lambda a, b, x, s: ref.get_powers_of(24, 0, False, False, False, b, x["n"], s),
        "get_powers_of_g": lambda a, b, x, s: ref.get_powers_of(24, 0, False, False, True, b, x["n"], s),
        "get_powers_by_val_bf": lambda a, b, x, s: ref.get_powers_by_val(42, 0, False, b, x["n"], s),
        "barycentric_precompute_at_ext": lambda a, b, x, s: ref.barycentric_precompute(
            True, x["x"], x["cf"], 7, x["coef"], x["n_coef"], True, s),
        "batch_eval_base_at_base": lambda a, b, x, s: ref.batch_eval_partial(0, a, x["rows"], x["cols"], x["coef"],
                                                                          x["partial"], s),
        "batch_eval_base_at_ext": lambda a, b, x, s: ref.batch_eval_partial(1, a, x["rows"], x["cols"], x["coef"],
                                                                         x["partial"], s),
    }


def run_serve_section(n_requests: int = 24, rates=(10.0, 20.0), budget_gib: int = 40, slots: int = 4):
    """Poisson LDE requests through the continuous-batching server vs the same requests served one at a time.

    Every request has its own pinned host input and output region (carved from two pinned pools), and after every
    server run each request's output is checked, bit for bit, against the same request computed alone on the
    device through bc_lde_fused.
    latency: requests arrive at each rate in `rates` (the seeded Poisson arrivals scaled to that rate); p50/p99 of
             completion - arrival, beside the FCFS one-at-a-time plain path fed the same arrivals (its queueing
             computed from measured per-request service times).
    capacity: all requests queued at once; output Melem/s of the server vs the one-at-a-time plain path.
    """
    import torch

    import bc_ntt
    import workloads

    reqs = workloads.serving_stream(n_requests=n_requests, rate_per_s=rates[0], seed=7)
    in_off, out_off, a, b = [], [], 0, 0
    for r in reqs:
        in_off.append(a)
        out_off.append(b)
        a += r.in_words
        b += r.out_words
    out_elems = b
    t_pin = time.perf_counter()
    hin = torch.empty(a, dtype=torch.int64, pin_memory=True)
    hout = torch.empty(b, dtype=torch.int64, pin_memory=True)
    pin_s = time.perf_counter() - t_pin
    # inputs uniform in [0, p) (each request its own seed); the expected outputs stay on the device
    expected = []
    for r, o in zip(reqs, in_off):
        ev = uniform_words(r.in_words, r.seed)
        hin[o:o + r.in_words].copy_(ev)
        exp = torch.empty(r.out_words, dtype=torch.int64, device="cuda")
        bc_ntt.lde(ev, exp, r.log_n, r.cols, r.log_blowup, fused=True)
        expected.append(exp)
        del ev
    torch.cuda.synchronize()

    def exact_requests() -> int:
        """Requests whose host output region equals their expected output, word for word."""
        good = 0
        for r, o, exp in zip(reqs, out_off, expected):
            good += int(torch.equal(hout[o:o + r.out_words].to("cuda", non_blocking=True), exp))
        return good

    # one at a time through the plain path: copy in, bc_lde_plain, copy out; service time of each request
    max_in = max(r.in_words for r in reqs)
    max_out = max(r.out_words for r in reqs)
    dev_in = torch.empty(max_in, dtype=torch.int64, device="cuda")
    dev_out = torch.empty(max_out, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(reqs) + 1)]
    hout.zero_()
    torch.cuda.synchronize()
    evs[0].record(stream)
    for i, r in enumerate(reqs):
        dev_in[:r.in_words].copy_(hin[in_off[i]:in_off[i] + r.in_words], non_blocking=True)
        bc_ntt.lde(dev_in, dev_out, r.log_n, r.cols, r.log_blowup, fused=False)
        hout[out_off[i]:out_off[i] + r.out_words].copy_(dev_out[:r.out_words], non_blocking=True)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    service = [evs[i].elapsed_time(evs[i + 1]) for i in range(len(reqs))]
    serial_s = sum(service) / 1e3
    exact = {"serial_plain": exact_requests()}
    del dev_in, dev_out
    torch.cuda.empty_cache()

    def serve(arrivals):
        hout.zero_()
        srv = bc_ntt.LdeServer(memory_budget_bytes=budget_gib << 30, slots=slots)
        t0 = time.perf_counter()
        ids = []
        for i, (r, at) in enumerate(zip(reqs, arrivals)):
            d = t0 + at - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(hin[in_off[i]:in_off[i] + r.in_words], hout[out_off[i]:out_off[i] + r.out_words],
                                  r.log_n, r.cols, r.log_blowup))
        for i in ids:
            srv.wait(i, timeout_ms=600000)
        st = srv.stats()
        srv.close()
        return st

    latency = []
    for rate in rates:
        arrivals = [r.arrival_s * rates[0] / rate for r in reqs]
        st = serve(arrivals)
        exact[f"rate_{rate:g}"] = exact_requests()
        # FCFS single-server latencies of the plain path under the same arrivals
        t_free, lat_serial = 0.0, []
        for at, sv in zip(arrivals, service):
            start = max(at * 1e3, t_free)
            t_free = start + sv
            lat_serial.append(t_free - at * 1e3)
        latency.append({"rate_per_s": rate, "p50_ms": round(st["p50_ms"], 2), "p99_ms": round(st["p99_ms"], 2),
                        "max_ms": round(st["max_ms"], 2), "completed": int(st["completed"]),
                        "serial_plain_same_arrivals_p50_ms": round(pct(lat_serial, 50), 2),
                        "serial_plain_same_arrivals_p99_ms": round(pct(lat_serial, 99), 2)})
    st_cap = serve([0.0] * len(reqs))
    exact["capacity"] = exact_requests()
    # the same requests device-resident (inputs and outputs in HBM, no PCIe): all queued at once
    dev_in = [hin[o:o + r.in_words].to("cuda") for r, o in zip(reqs, in_off)]
    dev_out = [torch.empty(r.out_words, dtype=torch.int64, device="cuda") for r in reqs]
    device_mode = {}
    for label, max_batch in (("coalesced", 1 << 22), ("per_request", 0)):
        for t in dev_out:
            t.zero_()
        st_d, dst = serve_device(reqs, dev_in, dev_out, [0.0] * len(reqs), max_batch, budget_bytes=1 << 30)
        device_mode[label] = {"value": round(st_d["out_melem_per_s"], 1), "span_s": round(st_d["span_s"], 4),
                              **dst, "exact": sum(int(torch.equal(o, e)) for o, e in zip(dev_out, expected))}
    del hin, hout, expected, dev_in, dev_out
    torch.cuda.empty_cache()
    return {"workload": f"{n_requests} requests, log_n U{{14..22}}, cols log-U[8,512], blowup U{{2,4}}, seed 7, "
                        f"per-request pinned host buffers, {budget_gib} GiB budget, {slots} slots",
            "unit": "Melem/s", "total_out_gelem": round(out_elems / 1e9, 3), "pin_s": round(pin_s, 2),
            "bit_exact": all(v == len(reqs) for v in exact.values()),
            "requests_exact": dict(exact, of=len(reqs), against="each request alone through bc_lde_fused"),
            "latency": latency,
            "capacity": {"server_value": round(st_cap["out_melem_per_s"], 1),
                         "serial_plain_value": round(out_elems / serial_s / 1e6, 1),
                         "speedup": round(st_cap["out_melem_per_s"] / (out_elems / serial_s / 1e6), 3),
                         "server_span_s": round(st_cap["span_s"], 3), "serial_plain_s": round(serial_s, 3)},
            "device_resident_capacity": dict(device_mode, note="the same requests with inputs and outputs in device "
                                             "memory (bc_lde_server_submit_device), all queued at once")}


def serve_device(reqs, dev_in, dev_out, arrivals, max_batch_elems: int, budget_bytes: int = 1 << 30):
    """Submits device-resident requests to a server at the given arrival times (seconds, paced by spinning on the
    host clock), waits for all; returns (server stats, device-batching stats)."""
    import bc_ntt

    srv = bc_ntt.LdeServer(memory_budget_bytes=budget_bytes, slots=1)
    srv.set_device_batching(max_batch_elems)
    t0 = time.perf_counter()
    ids = []
    for r, a, o, at in zip(reqs, dev_in, dev_out, arrivals):
        while time.perf_counter() - t0 < at:
            pass
        ids.append(srv.submit_device(a, o, r.log_n, r.cols, r.log_blowup))
    for i in ids:
        srv.wait(i, timeout_ms=600000)
    st, dst = srv.stats(), srv.device_stats()
    srv.close()
    return st, dst


def run_serve_device_section(n_requests: int = 300, rates=(5000.0, 20000.0)):
    """Small LDE requests whose columns already sit in device memory (a prover's own earlier kernels produced
    them): log_n U{10..16}, columns log-U[1,16], blowup U{2,4}, seeded Poisson arrivals.  The server coalesces
    the device requests pending together into one persistent batch launch; against the same server running every
    request as its own fused LDE, and against one fused call per request issued back to back on one stream (device
    time).  Every request's output is checked against the same request alone after every run."""
    import torch

    import bc_ntt
    import workloads

    reqs = workloads.serving_stream(n_requests=n_requests, rate_per_s=rates[0], seed=9, log_n_range=(10, 16),
                                    cols_range=(1, 16))
    dev_in = [uniform_words(r.in_words, r.seed) for r in reqs]
    dev_out = [torch.empty(r.out_words, dtype=torch.int64, device="cuda") for r in reqs]
    expected = []
    for r, a in zip(reqs, dev_in):
        e = torch.empty(r.out_words, dtype=torch.int64, device="cuda")
        bc_ntt.lde(a, e, r.log_n, r.cols, r.log_blowup, fused=True)
        expected.append(e)
    out_elems = sum(r.out_words for r in reqs)
    stream = torch.cuda.current_stream()
    # one fused call per request back to back on one stream: device time of each and in total
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(reqs) + 1)]
    torch.cuda.synchronize()
    evs[0].record(stream)
    for i, (r, a, o) in enumerate(zip(reqs, dev_in, dev_out)):
        bc_ntt.lde(a, o, r.log_n, r.cols, r.log_blowup, fused=True)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    service = [evs[i].elapsed_time(evs[i + 1]) for i in range(len(reqs))]
    serial_ms = evs[0].elapsed_time(evs[-1])

    def exact() -> int:
        return sum(int(torch.equal(o, e)) for o, e in zip(dev_out, expected))

    # first use of every kernel shape and of the server path (lazy module loading, attribute caches), untimed
    for max_batch in (1 << 22, 0):
        serve_device(reqs[:32], dev_in[:32], dev_out[:32], [0.0] * 32, max_batch)
    res = {"workload": f"{n_requests} device-resident requests, log_n U{{10..16}}, cols log-U[1,16], blowup U{{2,4}}, "
                       "seed 9", "unit": "Melem/s", "total_out_melem": round(out_elems / 1e6, 2),
           "serial_fused_calls": {"value": round(out_elems / (serial_ms / 1e3) / 1e6, 1), "ms": round(serial_ms, 3),
                                  "exact": exact()}}
    for label, max_batch in (("coalesced", 1 << 22), ("per_request", 0)):
        mode = {}
        for t in dev_out:
            t.zero_()
        st, dst = serve_device(reqs, dev_in, dev_out, [0.0] * len(reqs), max_batch)
        mode["capacity"] = {"value": round(st["out_melem_per_s"], 1), "span_ms": round(st["span_s"] * 1e3, 3),
                            **dst, "exact": exact()}
        for rate in rates:
            arrivals = [r.arrival_s * rates[0] / rate for r in reqs]
            for t in dev_out:
                t.zero_()
            st, dst = serve_device(reqs, dev_in, dev_out, arrivals, max_batch)
            # FCFS one-at-a-time fused calls under the same arrivals, from their measured service times
            t_free, lat = 0.0, []
            for at, sv in zip(arrivals, service):
                start = max(at * 1e3, t_free)
                t_free = start + sv
                lat.append(t_free - at * 1e3)
            mode[f"rate_{rate:g}"] = {"p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                                      **dst, "exact": exact(),
                                      "serial_fused_same_arrivals_p50_ms": round(pct(lat, 50), 3),
                                      "serial_fused_same_arrivals_p99_ms": round(pct(lat, 99), 3)}
        res[label] = mode
    runs = [res["serial_fused_calls"]["exact"]] + [m[k]["exact"] for m in (res["coalesced"], res["per_request"])
                                                    for k in m]
    res["bit_exact"] = all(v == len(reqs) for v in runs)
    res["coalesced_vs_per_request_capacity"] = round(res["coalesced"]["capacity"]["value"] /
                                                     max(res["per_request"]["capacity"]["value"], 1e-9), 3)
    del dev_in, dev_out, expected
    torch.cuda.empty_cache()
    return res


def run_reference(args, rank, world):
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not os.path.exists(oracle.REF_LIB):
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_ntt.so not built (needs the reference sources)"}
    n = 1 << LOG_N
    B = 1 << LOG_BLOWUP
    ref = oracle.RefKernels()
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream
    x = make_inputs(1234 + rank)
    out = torch.empty(B * COLS * n, device="cuda", dtype=torch.int64)
    coef = out[(B - 1) * COLS * n:]
    xp, op, cp = x.data_ptr(), out.data_ptr(), coef.data_ptr()

    def step(src=None):
        ref.batch_ntt(src or xp, cp, LOG_N, COLS, n, n, True, True, 0, 0, s)
        for k in range(B):
            ref.batch_ntt(cp, op + 8 * k * COLS * n, LOG_N, COLS, n, n, False, False, LOG_BLOWUP, k, s)

    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        total_ms, per = time_steps(step, args.steps, args.warmup, world, stream)
    out_elems = B * n * COLS
    value = whole_job_value(world, args.steps, out_elems, total_ms)
    hx = torch.empty(COLS * n, dtype=torch.int64, pin_memory=True)
    hx.copy_(x)
    hout = torch.empty(B * COLS * n, dtype=torch.int64, pin_memory=True)
    dx = torch.empty_like(x)

    def e2e_step():
        dx.copy_(hx, non_blocking=True)
        step(dx.data_ptr())
        hout.copy_(out, non_blocking=True)

    e2e_steps = max(2, min(args.steps, 5))
    e2e_ms, _ = time_steps(e2e_step, e2e_steps, 1, world, stream)
    del dx, hx, hout, x, out, coef
    torch.cuda.empty_cache()
    small = run_small_ntt_section(
        lambda a, b, log_n, cols, s: ref.batch_ntt(a, b, log_n, cols, 1 << log_n, 1 << log_n, False, False, 0, 0, s)) \
        if world == 1 else None
    ops = run_ops_section(ops_reference(ref), log_n=args.ops_log_n,
                          note="batch_eval_*: the reference's partial-reduce kernel only; "
                          "the CUB column sums that its Rust side runs after it are not timed") \
        if world == 1 and not args.no_ops else None
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "Melem/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks)", "data": "synthetic", "impl": "reference",
        "reference_kind": ("the reference's own CUDA kernels (native/ntt.cu) compiled for sm_100a, driven like "
                           "src/ntt.rs batch_ntt_internal: 1 inverse + 1 forward call per coset; the reference "
                           "has no CPU implementation of this path (boojum's CPU NTT is not vendored)"),
        "config": {"workload": f"coset LDE {COLS} cols x 2^{LOG_N}, blowup {B}, bit-reversed in/out",
                   "log_n": LOG_N, "columns": COLS, "blowup": B, "path": "reference kernels",
                   "l2": l2_note(), "parallelism": f"replicas x{world}"},
        "p50_ms": round(pct(per, 50), 4), "p99_ms": round(pct(per, 99), 4), "clocks": clk.summary(),
        "e2e": {"value": round(world * e2e_steps * out_elems / (e2e_ms / 1e3) / 1e6, 1), "unit": "Melem/s",
                "h2d_bytes_per_step": 8 * COLS * n, "d2h_bytes_per_step": 8 * B * COLS * n,
                "ms_per_step": round(e2e_ms / e2e_steps, 3)},
    }
    if small is not None:
        line["small_ntt"] = small
    if world == 1 and not args.no_batch:
        line["batch_per_job_reference"] = run_reference_batch_section(ref)
    if ops is not None:
        line["ops"] = ops
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the uneven-batch section")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving section")
    ap.add_argument("--no-large", action="store_true", help="skip the 64 x 2^23 blowup-4 section")
    ap.add_argument("--no-ops", action="store_true", help="skip the bit-reversal / powers / omega-shift section")
    ap.add_argument("--ops-log-n", type=int, default=28, help="elements of the ops section's buffers (log2, >= 23)")
    ap.add_argument("--no-tuned-plans", action="store_true", help="ignore the autotuned plan file")
    ap.add_argument("--log-n", type=int, default=22, help="column length 2^log_n (default 22)")
    ap.add_argument("--cols", type=int, default=128, help="columns (default 128)")
    ap.add_argument("--log-blowup", type=int, default=1, help="log2 of the blowup (default 1)")
    args = ap.parse_args()
    global LOG_N, COLS, LOG_BLOWUP
    LOG_N, COLS, LOG_BLOWUP = args.log_n, args.cols, args.log_blowup
    rank, world, _ = dist_setup(args.gpus)
    line = run_ours(args, rank, world) if args.impl == "ours" else run_reference(args, rank, world)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
