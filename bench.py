"""Benchmark of ssblasGemmBatchedEx on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--mode ozaki|plain|bf16x3]
    python bench.py --impl reference ...      (the reference's own CPU implementation)

Default workload: FP64 batched GEMM, 32 instances of 1024^3, op(A)=N, op(B)=T, ld 1032,
entries sign * U[1,2) * 2^U{-8..8}, alpha 1, beta 0 -- timed in the Ozaki int8-slice emulated
form (value) and in the plain DMMA form (config.modes.plain), each with its max normalised error
against the FP64-exact oracle. A step is one ssblasGemmBatchedEx call over the whole batch.

value : FP64-equivalent TFLOP/s (2*m*n*k*batch per step, summed over ranks) with the operands
        resident in HBM (host arrays of device pointers, asynchronous calls back to back, CUDA
        events on the library stream). The operands (805 MB) exceed the 126 MB L2, so no flush is
        needed.
e2e   : the same metric through the reference-style call (host arrays of host pointers in pinned
        memory); every step copies A and B to the device and C back inside the timed region and
        returns after C is on the host. e2e.pageable: the same with every instance in its own
        pageable allocation, as the reference's example allocates them.
config.secondary (rank 0, default workload only): the other benchmark configurations, each timed
        for a few seconds with CUDA events -- int8 512 x 512^3 TN (bit-exact count, HBM fraction),
        fp32 4096 x 64^3 TT in the plain and 3xBF16 forms (errors, HBM fractions), fp32 64 x 128^3
        NN, and the grouped 10,000-instance call against one plain launch per instance.
Multi-GPU (torchrun): every rank runs the full workload on its own GPU (weak scaling, batch
instances are independent -- there is no collective on the data path); the time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as ct
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from ssblasex_b200 import workloads as W  # noqa: E402

METRIC = "Batched GEMM TFLOP/s & %roofline: plain vs emulated form at equal FP64 error"
CPU_SAMPLE = {"f64_batch32_1024": 2, "i8_batch512_512": 4, "fp32_batch64_128": 64, "fp32_batch4096_64": 512,
              "i8_batch8_4096": 1, "f64_batch2_256_8192": 1, "i8_batch64_512_nn": 4}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="f64_batch32_1024", choices=list(W.WORKLOADS) + ["grouped_10000"])
    ap.add_argument("--mode", default="auto", choices=["auto", "ozaki", "plain", "bf16x3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--batch", type=int, default=None,
                    help="fewer instances than the named workload (profiling runs only)")
    return ap.parse_args()


# ------------------------------------------------------------------------------- clocks -----
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []          # (host time, csv line)
        self.window = None       # (t0, t1) host times of the timed region

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)      # let the sampler start before the timed region
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t0: float, t1: float):
        """Host times bracketing the timed region; samples within 50 ms of it are kept."""
        self.window = (t0 - 0.05, t1 + 0.05)

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sms, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if self.window and not (self.window[0] <= ts <= self.window[1]):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sms)}


# ------------------------------------------------------------------------------- helpers ----
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", d["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


# Figures of the dominant kernel from one ncu capture each (profiles/ holds the summaries):
#   traffic: dram__bytes_read.sum + dram__bytes_write.sum per launch. The 32-instance launch is
#   too large to capture under ncu, so an 8-instance launch of the same kernel was captured
#   (153 MB) and scaled by the instances it processes.
#   imma_pipe: sm__pipe_tensor_cycles_active share of the int8 (imma) tensor pipe in that capture;
#   it reads below `frac` because the int8 peak used for `frac` is derived (2 x measured bf16).
NCU = {("f64_batch32_1024", "ozaki"): {"traffic": 153.1e6 * 4, "imma_pipe_frac": 0.685,
                                       "profile": "profiles/ozaki_gemm_f64_batch8_1024_full.md"}}


def cpu_threads():
    n = os.cpu_count() or 1
    return n if n not in (2, 3, 4, 6) else 1


def sample_problem(p: W.Problem, count: int) -> W.Problem:
    import dataclasses
    return dataclasses.replace(p, batch=count, A=p.A[:count], B=p.B[:count], C=p.C[:count].copy())


def reference_timing(p: W.Problem, steps: int, warmup: int, sample: int):
    """The reference library (compiled from its own sources into oracle/_ref) on `sample`
    instances per step, with all host threads. Returns (seconds per step list, kind)."""
    from oracle import oracle as O
    q = sample_problem(p, sample)
    if O.reference_available():
        run, kind = (lambda: O.reference_gemm(q, C=q.C)), "reference"
    else:
        run, kind = (lambda: O.restated_gemm(q, C=q.C)), "port"
    for _ in range(warmup):
        run()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        st, _ = run()
        ts.append(time.perf_counter() - t0)
        assert st == 0
    return ts, kind


def openblas_loop_timing(p: W.Problem, sample: int, reps: int = 3):
    """The reference example's per-instance OpenBLAS loop (example/include/naive_gemm.hpp:195-226)
    through numpy's bundled OpenBLAS, on `sample` instances; best of reps."""
    if p.row == "i8":
        return None
    q = sample_problem(p, sample)
    A = [np.ascontiguousarray(q.op_a(b)) for b in range(sample)]
    B = [np.ascontiguousarray(q.op_b(b)) for b in range(sample)]
    best = float("inf")
    for _ in range(reps + 1):
        t0 = time.perf_counter()
        for b in range(sample):
            out = q.alpha * (A[b] @ B[b])
            if q.beta != 0:
                out += q.beta * q.c_view(q.C, b)
        best = min(best, time.perf_counter() - t0)
    return best


def mode_id(S, mode: str) -> int:
    return {"ozaki": S.SSBLAS_MATH_FP64_OZAKI, "plain": S.SSBLAS_MATH_PLAIN,
            "bf16x3": S.SSBLAS_MATH_FP32_BF16X3}[mode]


class Leg:
    """One workload on one GPU: device copies, the reference-convention call with host arrays of
    device pointers, CUDA-event timing on the library stream, and the error check."""

    def __init__(self, S, p: W.Problem, device: str, stream):
        from ssblasex_b200 import runner
        self.S, self.p, self.stream = S, p, stream
        self.dp = runner.DeviceProblem(p, device=device)
        self.al = np.array([p.alpha], dtype=p.scale_dtype)
        self.be = np.array([p.beta], dtype=p.scale_dtype)
        # host arrays of device pointers: the library sees the instances' spacing without a device
        # read-back, so equally spaced batches take the tensor-map paths directly
        self.Ah, self.Bh, self.Ch = self.dp.host_arrays()

    def call(self):
        p = self.p
        ta, tb, tc = p.types
        return self.S.lib().ssblasGemmBatchedEx(p.transa, p.transb, p.m, p.n, p.k, self.al.ctypes.data, self.Ah, ta,
                                                p.lda, self.Bh, tb, p.ldb, self.be.ctypes.data, self.Ch, tc,
                                                p.ldc, p.batch, 0, 0)

    def timed(self, math_mode, steps, warmup, profile=False, clk=None, barrier=None, queued=False):
        """CUDA-event time per step on the library stream. queued: a spin kernel (about 80 us per
        step) goes on the stream first, so every call is enqueued before the GPU reaches it and the
        events time the kernels back to back; otherwise a call whose host work outlasts its kernels
        leaves the stream idle and the time per step is the host's."""
        import torch
        S = self.S
        S.set_math_mode(math_mode)
        S.set_sync_mode(False)
        for _ in range(warmup):
            assert self.call() == 0
        torch.cuda.synchronize()
        if barrier:
            barrier()
        torch.cuda.synchronize()
        S.set_profiling(profile)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.time()
        with torch.cuda.stream(self.stream):
            if queued:
                torch.cuda._sleep(int(steps * 80e-6 * 2.0e9))
            e0.record(self.stream)
            for _ in range(steps):
                st = self.call()
                assert st == 0, st
            e1.record(self.stream)
        torch.cuda.synchronize()
        if clk is not None:
            clk.mark(t0, time.time())
        ms = e0.elapsed_time(e1) / steps
        prof = S.get_profile() if profile else {}
        S.set_profiling(False)
        info = S.last_run_info()
        S.set_sync_mode(True)
        return ms, prof, info

    def error(self, math_mode, instances=None, rows=None):
        """Max normalised error against the FP64-exact oracle (fp rows), or mismatches against the
        exact int64 result (int8 row), on sampled instances and rows."""
        from ssblasex_b200 import runner
        from oracle import oracle as O
        p = self.p
        self.S.set_math_mode(math_mode)
        self.dp.reset_c()
        st, C = runner.call(p, mode="device_array", dp=self.dp)
        assert st == 0
        if p.row == "i8":
            bad = 0
            rr = np.arange(p.m) if p.m * p.n * p.k <= 2 ** 28 else np.arange(0, p.m, max(1, p.m // 16))
            for b in (instances or (0, p.batch - 1)):
                want = (p.op_a(b)[rr].astype(np.int64) @ p.op_b(b).astype(np.int64) * int(p.alpha)
                        + int(p.beta) * p.c_view(p.C, b)[rr].astype(np.int64))
                want = ((want + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
                bad += int(np.sum(p.c_view(C, b)[rr] != want))
            return float(bad)
        inst = instances if instances is not None else sorted({0, p.batch // 2, p.batch - 1})
        rr = rows if rows is not None else range(0, p.m, max(1, p.m // 16))
        return O.normalized_error(p, C, instances=inst, rows=rr)


def dominant(prof: dict, steps: int):
    """(kernel name, ms per launch, launches per step) of the kernel with the largest event time."""
    if not prof:
        return "?", 1.0, 1.0
    name, (n, ms) = max(prof.items(), key=lambda kv: kv[1][1])
    return name, ms / max(n, 1), n / steps


def hbm_roof(bytes_per_launch: float, ms: float, pk: dict) -> dict:
    gbs = bytes_per_launch / (ms * 1e-3) / 1e9
    return {"achieved": gbs, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": gbs / pk["hbm_gbs"]}


# ------------------------------------------------------------------------------- arms -------
def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
    p = W.workload(args.workload)
    sample = CPU_SAMPLE[args.workload]
    ts, kind = reference_timing(p, args.steps, args.warmup, sample)
    flops = 2.0 * p.m * p.n * p.k * sample
    t = float(np.mean(ts))
    val = flops / t / 1e12
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": p.row, "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "sample_instances_per_step": sample},
            "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
                             "kind": kind,
                             "sample": f"{sample} of {p.batch} instances of {p.m}x{p.n}x{p.k} per step"},
            "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def grouped_leg(S, count: int, steps: int, warmup: int, stream):
    """10,000 uneven GEMMs (m, n, k log-uniform in [8, 512]; half fp64 in the Ozaki mode, half
    fp32 in the 3xBF16 mode) through one ssblasGemmGroupedBatchedEx call per step (pre-pass and
    persistent GEMM launches replayed from a CUDA graph), against the same instances as one plain
    ssblasGemmBatchedEx launch each (asynchronous, back to back). Both on the library stream,
    timed with CUDA events."""
    import torch
    from ssblasex_b200 import runner
    probs = W.grouped_problems(count=count)
    flops = sum(2.0 * p.m * p.n * p.k for p in probs)
    gd = runner.GroupedDevice(probs)

    def timed(fn, n, w):
        for _ in range(w):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, (time.perf_counter() - t0) * 1e3 / n

    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI | S.SSBLAS_MATH_FP32_BF16X3)
    S.set_sync_mode(False)
    ms_g, wall_g = timed(lambda: gd.call(device_arrays=True), steps, warmup)
    launches = S.last_run_info()["kernel_launches"]
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    calls = []
    for p, (a, b, c) in zip(probs, gd.tensors):
        arrs = [(ct.c_void_p * 1)(t.data_ptr()) for t in (a, b, c)]
        al, be = np.array([p.alpha], p.scale_dtype), np.array([p.beta], p.scale_dtype)
        calls.append((p, arrs, al, be))

    def loop():
        for p, arrs, al, be in calls:
            S.lib().ssblasGemmBatchedEx(p.transa, p.transb, p.m, p.n, p.k, al.ctypes.data, arrs[0], p.types[0],
                                        p.lda, arrs[1], p.types[1], p.ldb, be.ctypes.data, arrs[2], p.types[2],
                                        p.ldc, 1, 0, 0)
    ms_l, wall_l = timed(loop, max(1, steps // 5), 1)
    # the same grouped call in plain mode (fp64 tiles on DMMA, fp32 tiles on FFMA): the same
    # arithmetic as the loop above, one call
    ms_gp, wall_gp = timed(lambda: gd.call(device_arrays=True), steps, warmup)
    launches_p = S.last_run_info()["kernel_launches"]
    S.set_sync_mode(True)
    return {"workload": f"grouped_{count}", "instances": count, "flops": flops,
            "tflops": flops / (ms_g * 1e-3) / 1e12,
            "grouped": {"ms_device": ms_g, "ms_wall": wall_g, "launches": launches},
            "plain_loop": {"ms_device": ms_l, "ms_wall": wall_l, "launches": count},
            "speedup_vs_plain_loop": ms_l / ms_g, "speedup_vs_plain_loop_wall": wall_l / wall_g,
            "grouped_plain": {"ms_device": ms_gp, "ms_wall": wall_gp, "launches": launches_p,
                              "speedup_vs_plain_loop": ms_l / ms_gp}}


def run_grouped(args):
    import torch
    import ssblasex_b200 as S
    stream = torch.cuda.Stream()
    S.set_stream(stream.cuda_stream)
    g = grouped_leg(S, args.batch or 10000, args.steps, args.warmup, stream)
    line = {"metric": METRIC, "value": g["tflops"], "unit": "TFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": g["grouped"]["ms_device"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "i8+bf16",
            "data": "synthetic (seeded)", "config": g}
    print(json.dumps(line), flush=True)
    return 0


def secondary_legs(S, device: str, stream, pk: dict) -> dict:
    """The other benchmark configurations, a few seconds each (rank 0 of the default run)."""
    out = {}
    # int8 -> int32, 512 x 512^3, TN, beta = 1: HBM-bound (arithmetic intensity ~102 op/B)
    p = W.workload("i8_batch512_512")
    leg = Leg(S, p, device, stream)
    bad = leg.error(S.SSBLAS_MATH_PLAIN, instances=(0, 255, 511))
    ms, prof, info = leg.timed(S.SSBLAS_MATH_PLAIN, 10, 3, profile=True)
    name, kms, per = dominant(prof, 10)
    out["i8_batch512_512"] = {
        "ms_per_step": ms, "tops": 2.0 * p.m * p.n * p.k * p.batch / (ms * 1e-3) / 1e12,
        "mismatches": bad, "checked": "3 instances, every row", "path": info["path"],
        "roofline": {"bound": "hbm", "kernel": name, **hbm_roof(p.algorithmic_bytes() / per, kms, pk)},
        "int8_tensor_frac": 2.0 * p.m * p.n * p.k * p.batch / per / (kms * 1e-3) / 1e12 / (2.0 * pk["bf16_tflops"])}
    del leg
    # fp32 4096 x 64^3 TT with outliers: plain FFMA and 3xBF16
    p = W.workload("fp32_batch4096_64")
    leg = Leg(S, p, device, stream)
    modes = {}
    inst = list(range(0, p.batch, 64))
    for md in ("plain", "bf16x3"):
        err = leg.error(mode_id(S, md), instances=inst)
        ms, prof, info = leg.timed(mode_id(S, md), 20, 3, profile=True)
        name, kms, per = dominant(prof, 20)
        modes[md] = {"ms_per_step": ms, "tflops": p.flops() / (ms * 1e-3) / 1e12,
                     "max_normalized_error": err, "path": info["path"],
                     "step_hbm_frac": p.algorithmic_bytes() / (ms * 1e-3) / 1e9 / pk["hbm_gbs"],
                     "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()},
                     "roofline": {"bound": "hbm", "kernel": name, **hbm_roof(p.algorithmic_bytes() / per, kms, pk)}}
    out["fp32_batch4096_64"] = modes
    del leg
    # fp32 64 x 128^3 NN
    p = W.workload("fp32_batch64_128")
    leg = Leg(S, p, device, stream)
    err = leg.error(S.SSBLAS_MATH_PLAIN, instances=range(p.batch), rows=range(p.m))
    ms, prof, info = leg.timed(S.SSBLAS_MATH_PLAIN, 50, 5, profile=True)
    name, kms, per = dominant(prof, 50)
    # the same 50 calls enqueued behind a spin kernel: the device time of the kernels alone
    qms, qprof, _ = leg.timed(S.SSBLAS_MATH_PLAIN, 50, 5, profile=True, queued=True)
    _, qkms, _ = dominant(qprof, 50)
    out["fp32_batch64_128"] = {"ms_per_step": ms, "tflops": p.flops() / (ms * 1e-3) / 1e12,
                               "max_normalized_error": err, "path": info["path"], "kernel": name,
                               "kernel_ms": kms, "hbm_bound_ms": p.algorithmic_bytes() / (pk["hbm_gbs"] * 1e9) * 1e3,
                               "queued": {"ms_per_step": qms, "kernel_ms": qkms,
                                          "note": "calls enqueued behind a spin kernel; kernel_ms is the "
                                                  "kernel's device time with no host gap before it"}}
    del leg
    # grouped 10,000
    out["grouped_10000"] = grouped_leg(S, 10000, 5, 2, stream)
    return out


def pageable_e2e(S, p: W.Problem, math: int, steps: int):
    """The reference caller's layout: every instance of A, B and C in its own pageable (not
    page-locked) host allocation, host arrays of host pointers, synchronous call."""
    As = [np.array(p.A[b]) for b in range(p.batch)]
    Bs = [np.array(p.B[b]) for b in range(p.batch)]
    Cs = [np.array(p.C[b]) for b in range(p.batch)]
    mk = lambda xs: (ct.c_void_p * p.batch)(*[x.ctypes.data for x in xs])
    Ap, Bp, Cp = mk(As), mk(Bs), mk(Cs)
    al = np.array([p.alpha], dtype=p.scale_dtype)
    be = np.array([p.beta], dtype=p.scale_dtype)
    ta, tb, tc = p.types
    S.set_math_mode(math)
    S.set_sync_mode(True)

    def call():
        return S.lib().ssblasGemmBatchedEx(p.transa, p.transb, p.m, p.n, p.k, al.ctypes.data, Ap, ta, p.lda, Bp, tb,
                                           p.ldb, be.ctypes.data, Cp, tc, p.ldc, p.batch, 0, 0)
    assert call() == 0
    t0 = time.perf_counter()
    for _ in range(steps):
        assert call() == 0
    return (time.perf_counter() - t0) / steps


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "grouped_10000":
        return run_grouped(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import ssblasex_b200 as S
    from ssblasex_b200 import runner

    device = f"cuda:{local}"
    p = W.workload(args.workload, batch=args.batch)
    mode = args.mode
    if mode == "auto":
        mode = {"f64": "ozaki", "f32": "plain", "i8": "plain"}[p.row]
    math = mode_id(S, mode)
    stream = torch.cuda.Stream()
    S.set_stream(stream.cuda_stream)
    leg = Leg(S, p, device, stream)
    barrier = dist.barrier if world > 1 else None

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    results = {}
    modes = [mode] + (["plain"] if mode != "plain" else [])
    for md in modes:
        mm = mode_id(S, md)
        err = leg.error(mm)
        with ClockSampler(local) as clk:
            ms, _, info = leg.timed(mm, args.steps, args.warmup, clk=clk, barrier=barrier)
        ms = max_over_ranks(ms)
        np_ = max(3, args.steps // 2)
        _, prof, _ = leg.timed(mm, np_, 1, profile=True, barrier=barrier)
        results[md] = dict(ms=ms, err=err, info=info, prof=prof, prof_steps=np_, clocks=clk.summary())

    head = results[mode]
    flops = p.flops() * world
    value = flops / (head["ms"] * 1e-3) / 1e12

    # roofline of the dominant kernel of the headline mode
    pk = peaks()
    dom_name, per_launch_ms, launches_per_step = dominant(head["prof"], head["prof_steps"])
    ncu = NCU.get((args.workload, mode), {}) if p.batch == W.WORKLOADS.get(args.workload, {}).get("batch") else {}
    if mode == "ozaki":
        # int8 tensor work of the slice-pair products per launch
        slices = head["info"]["slices"]
        pairs = slices * (slices + 1) // 2
        ops = 2.0 * p.m * p.n * p.k * p.batch * pairs / launches_per_step
        int8_peak = 2.0 * pk["bf16_tflops"]
        achieved = ops / (per_launch_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS (int8)",
                "frac": achieved / int8_peak, "traffic": ncu.get("traffic"), "kernel": dom_name,
                "peak_source": f"2 x bf16_tflops ({pk['source']}): dense int8 rate is twice bf16 on B200",
                "imma_pipe_frac_ncu": ncu.get("imma_pipe_frac"), "ncu_profile": ncu.get("profile")}
        # the slicing pre-pass is HBM-bound: its algorithmic bytes are the fp64 operands read once
        # and the int8 slices written once
        sl = head["prof"].get("ozaki_slice")
        if sl:
            sl_bytes = (8.0 * (p.m + p.n) * p.k + slices * (p.m + p.n) * p.k) * p.batch
            sl_ms = sl[1] / sl[0]
            roof["pre_pass"] = {"kernel": "ozaki_slice", "bound": "hbm", "ms_per_launch": sl_ms,
                                **hbm_roof(sl_bytes, sl_ms, pk)}
    elif p.row == "i8":
        # the bound is whichever of the int8 tensor rate and HBM gives the longer time
        bytes_ = p.algorithmic_bytes() / launches_per_step
        ops = 2.0 * p.m * p.n * p.k * p.batch / launches_per_step
        int8_peak = 2.0 * pk["bf16_tflops"]
        if ops / (int8_peak * 1e12) > bytes_ / (pk["hbm_gbs"] * 1e9):
            achieved = ops / (per_launch_ms * 1e-3) / 1e12
            roof = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS (int8)",
                    "frac": achieved / int8_peak, "traffic": None, "kernel": dom_name,
                    "peak_source": f"2 x bf16_tflops ({pk['source']}): dense int8 rate is twice bf16 on B200"}
        else:
            roof = {"bound": "hbm", "traffic": None, "kernel": dom_name, "peak_source": pk["source"],
                    **hbm_roof(bytes_, per_launch_ms, pk)}
    else:
        fl = p.flops() / launches_per_step
        achieved = fl / (per_launch_ms * 1e-3) / 1e12
        fp_peak = {"f64": 40.0, "f32": 80.0}[p.row]
        roof = {"bound": "fp64_pipe" if p.row == "f64" else "fp32_pipe", "achieved": achieved, "peak": fp_peak,
                "unit": "TFLOP/s", "frac": achieved / fp_peak, "traffic": None, "kernel": dom_name,
                "peak_source": "nominal B200 SIMT peak (no measured figure for this pipe)"}

    # end to end through the reference-style call with host buffers
    e2e = None
    if not args.no_e2e:
        S.set_math_mode(math)
        S.set_sync_mode(True)
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
        hA, hB, hC = pin(p.A), pin(p.B), pin(p.C.copy())
        hp = W.Problem(**{**p.__dict__, "A": hA, "B": hB})
        for _ in range(2):
            st, _ = runner.call(hp, mode="host_matrices", host_C=hC)
            assert st == 0
        e2e_steps = max(2, min(args.steps, 5))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            st, _ = runner.call(hp, mode="host_matrices", host_C=hC)
        t_e2e = max_over_ranks((time.perf_counter() - t0) / e2e_steps)
        del hA, hB, hC, hp
        h2d = p.A.nbytes + p.B.nbytes + (p.C.nbytes if p.beta != 0 else 0)
        d2h = p.m * p.n * np.dtype(p.c_dtype).itemsize * p.batch
        t_pg = max_over_ranks(pageable_e2e(S, p, math, 2))
        e2e = {"value": flops / t_e2e / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": t_e2e * 1e3,
               "note": "host arrays of host pointers (pinned), copies and synchronous return inside the timed region",
               "pageable": {"value": flops / t_pg / 1e12, "unit": "TFLOP/s", "ms_per_step": t_pg * 1e3,
                            "note": "every instance in its own pageable allocation, as the reference's "
                                    "example allocates them"}}

    secondary = None
    if rank == 0 and not args.no_secondary and args.workload == "f64_batch32_1024" and args.batch is None:
        del leg
        torch.cuda.empty_cache()
        secondary = secondary_legs(S, device, stream, pk)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
        sample = CPU_SAMPLE[args.workload]
        ts, kind = reference_timing(p, 3, 1, sample)
        fl = 2.0 * p.m * p.n * p.k * sample
        cpu = {"value": fl / min(ts) / 1e12, "unit": "TFLOP/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
               "kind": kind, "sample": f"{sample} of {p.batch} instances per timing, best of 3",
               "label": "reference built from its own sources, x86 emulation of its SVE kernels (host has no SVE)"}
        tb_ = openblas_loop_timing(p, sample)
        if tb_:
            cpu["openblas_loop"] = {"value": fl / tb_ / 1e12, "unit": "TFLOP/s",
                                    "label": "example's per-instance OpenBLAS loop (numpy OpenBLAS), host has no SVE"}

    if rank == 0:
        extra = {md: {"tflops": flops / (r["ms"] * 1e-3) / 1e12, "ms_per_step": r["ms"],
                      "max_normalized_error" if p.row != "i8" else "mismatches": r["err"],
                      "path": r["info"]["path"], "slices": r["info"]["slices"],
                      "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in r["prof"].items()}}
                 for md, r in results.items()}
        if mode == "ozaki":
            dtype = f"f64 (Ozaki int8 slices, S={head['info']['slices']})"
            extra["ozaki_over_plain"] = results["plain"]["ms"] / head["ms"]
        else:
            dtype = p.row
        line = {"metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded)",
                "config": {"workload": args.workload, "batch": p.batch, "m": p.m, "n": p.n, "k": p.k,
                           "transa": "NT"[p.transa], "transb": "NT"[p.transb], "ld": [p.lda, p.ldb, p.ldc],
                           "mode": mode, "emulates": p.row, "parallelism": f"batch-replica x{world}",
                           "l2": "operands larger than L2, no flush", "modes": extra, "secondary": secondary},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": int(head["info"]["kernel_launches"] * args.steps),
                "clocks": head["clocks"]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
