"""Benchmark of ssblasGemmBatchedEx on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--mode ozaki|plain]
    python bench.py --impl reference ...      (the reference's own CPU implementation)

Default workload: FP64 batched GEMM, 32 instances of 1024^3, op(A)=N, op(B)=T, ld 1032,
entries sign * U[1,2) * 2^U{-8..8}, alpha 1, beta 0 -- timed in the Ozaki int8-slice emulated
form (value) and in the plain DFMA form (config.plain), each with its max normalised error
against the FP64-exact oracle. A step is one ssblasGemmBatchedEx call over the whole batch.

value : FP64-equivalent TFLOP/s (2*m*n*k*batch per step, summed over ranks) with the operands
        resident in HBM (device pointer arrays, asynchronous calls back to back, CUDA events on
        the library stream). The operands (805 MB) exceed the 126 MB L2, so no flush is needed.
e2e   : the same metric through the reference-style call (host arrays of host pointers in
        pinned memory); every step copies A and B to the device and C back inside the timed
        region and returns after C is on the host.
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


# DRAM traffic per launch of the dominant kernel (dram__bytes_read.sum + dram__bytes_write.sum from
# one ncu capture). The 32-instance launch is too large to capture under ncu, so an 8-instance
# launch of the same kernel was captured (153 MB) and scaled by the instances it processes.
NCU_TRAFFIC = {("f64_batch32_1024", "ozaki"): 153.1e6 * 4}


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


# ------------------------------------------------------------------------------- arms -------
def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
    p = W.workload(args.workload)
    sample = {"f64_batch32_1024": 2, "i8_batch512_512": 4, "fp32_batch64_128": 64,
              "fp32_batch4096_64": 512, "i8_batch8_4096": 1, "f64_batch2_256_8192": 1,
              "i8_batch64_512_nn": 4}[args.workload]
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


def run_grouped(args):
    """10,000 uneven GEMMs (m, n, k log-uniform in [8, 512]; half fp64 in the Ozaki mode, half
    fp32 in the 3xBF16 mode) through one ssblasGemmGroupedBatchedEx call per step (pre-pass and
    persistent GEMM launches replayed from a CUDA graph), against the same instances as one plain
    ssblasGemmBatchedEx launch each (asynchronous, back to back)."""
    import torch
    import ssblasex_b200 as S
    from ssblasex_b200 import runner
    count = args.batch or 10000
    probs = W.grouped_problems(count=count)
    flops = sum(2.0 * p.m * p.n * p.k for p in probs)
    gd = runner.GroupedDevice(probs)
    stream = torch.cuda.Stream()
    S.set_stream(stream.cuda_stream)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, (time.perf_counter() - t0) * 1e3 / steps

    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI | S.SSBLAS_MATH_FP32_BF16X3)
    S.set_sync_mode(False)
    ms_g, wall_g = timed(lambda: gd.call(device_arrays=True), args.steps, args.warmup)
    launches = S.last_run_info()["kernel_launches"]
    # one plain launch per instance
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
    ms_l, wall_l = timed(loop, max(1, args.steps // 5), 1)
    S.set_sync_mode(True)
    line = {"metric": METRIC, "value": flops / (ms_g * 1e-3) / 1e12, "unit": "TFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_g, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i8+bf16", "data": "synthetic (seeded)",
            "config": {"workload": f"grouped_{count}", "instances": count, "flops": flops,
                       "grouped": {"ms_device": ms_g, "ms_wall": wall_g, "launches": launches},
                       "plain_loop": {"ms_device": ms_l, "ms_wall": wall_l, "launches": count},
                       "speedup_vs_plain_loop_wall": wall_l / wall_g}}
    print(json.dumps(line), flush=True)
    return 0


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
    from oracle import oracle as O

    p = W.workload(args.workload, batch=args.batch)
    mode = args.mode
    if mode == "auto":
        mode = {"f64": "ozaki", "f32": "plain", "i8": "plain"}[p.row]
    math = {"ozaki": S.SSBLAS_MATH_FP64_OZAKI, "plain": S.SSBLAS_MATH_PLAIN,
            "bf16x3": S.SSBLAS_MATH_FP32_BF16X3}[mode]

    dp = runner.DeviceProblem(p, device=f"cuda:{local}")
    stream = torch.cuda.Stream()
    S.set_stream(stream.cuda_stream)
    al = np.array([p.alpha], dtype=p.scale_dtype)
    be = np.array([p.beta], dtype=p.scale_dtype)
    # host arrays of device pointers: the library sees the instances' spacing without a device
    # read-back, so equally spaced batches take the tensor-map paths directly
    Ah, Bh, Ch = dp.host_arrays()
    ta, tb, tc = p.types

    def call():
        return S.lib().ssblasGemmBatchedEx(p.transa, p.transb, p.m, p.n, p.k, al.ctypes.data, Ah, ta,
                                           p.lda, Bh, tb, p.ldb, be.ctypes.data, Ch, tc,
                                           p.ldc, p.batch, 0, 0)

    def timed(math_mode, steps, warmup, profile=False, clk=None):
        S.set_math_mode(math_mode)
        S.set_sync_mode(False)
        for _ in range(warmup):
            assert call() == 0
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        S.set_profiling(profile)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.time()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(steps):
                st = call()
                assert st == 0, st
            e1.record(stream)
        torch.cuda.synchronize()
        if clk is not None:
            clk.mark(t0, time.time())
        ms = e0.elapsed_time(e1) / steps
        prof = S.get_profile() if profile else {}
        S.set_profiling(False)
        info = S.last_run_info()
        S.set_sync_mode(True)
        if world > 1:
            t = torch.tensor([ms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, prof, info

    def error_of(math_mode):
        S.set_math_mode(math_mode)
        dp.reset_c()
        st, C = runner.call(p, mode="device_array", dp=dp)
        assert st == 0
        if p.row == "i8":
            # integer rows are exact: check two instances bit for bit (16 rows of each when the
            # instances are large)
            bad = 0
            rows = np.arange(p.m) if p.m * p.n * p.k <= 2 ** 28 else np.arange(0, p.m, max(1, p.m // 16))
            for b in (0, p.batch - 1):
                want = (p.op_a(b)[rows].astype(np.int64) @ p.op_b(b).astype(np.int64) * int(p.alpha)
                        + int(p.beta) * p.c_view(p.C, b)[rows].astype(np.int64))
                want = ((want + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
                bad += int(np.sum(p.c_view(C, b)[rows] != want))
            return float(bad)
        inst = sorted({0, p.batch // 2, p.batch - 1})
        rows = range(0, p.m, max(1, p.m // 16))
        return O.normalized_error(p, C, instances=inst, rows=rows)

    results = {}
    modes = [mode] + (["plain"] if mode != "plain" else [])
    for md in modes:
        mm = {"ozaki": S.SSBLAS_MATH_FP64_OZAKI, "plain": S.SSBLAS_MATH_PLAIN, "bf16x3": S.SSBLAS_MATH_FP32_BF16X3}[md]
        err = error_of(mm)
        with ClockSampler(local) as clk:
            ms, _, info = timed(mm, args.steps, args.warmup, clk=clk)
        _, prof, _ = timed(mm, max(3, args.steps // 2), 1, profile=True)
        results[md] = dict(ms=ms, err=err, info=info, prof=prof, clocks=clk.summary())

    head = results[mode]
    flops = p.flops() * world
    value = flops / (head["ms"] * 1e-3) / 1e12

    # roofline of the dominant kernel of the headline mode
    pk = peaks()
    dom_name, (dom_n, dom_ms) = max(head["prof"].items(), key=lambda kv: kv[1][1]) if head["prof"] else ("?", (1, 1.0))
    per_launch_ms = dom_ms / max(dom_n, 1)
    launches_per_step = dom_n / max(3, args.steps // 2)
    if mode == "ozaki":
        # int8 tensor work of the slice-pair products per launch
        pairs = head["info"]["slices"] * (head["info"]["slices"] + 1) // 2
        ops = 2.0 * p.m * p.n * p.k * p.batch * pairs / launches_per_step
        int8_peak = 2.0 * pk["bf16_tflops"]
        achieved = ops / (per_launch_ms * 1e-3) / 1e12
        traffic = NCU_TRAFFIC.get((args.workload, mode)) if p.batch == 32 else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS (int8)",
                "frac": achieved / int8_peak, "traffic": traffic, "kernel": dom_name,
                "peak_source": f"2 x bf16_tflops ({pk['source']}): dense int8 rate is twice bf16 on B200"}
        # the slicing pre-pass is HBM-bound: its algorithmic bytes are the fp64 operands read once
        # and the int8 slices written once
        sl = head["prof"].get("ozaki_slice")
        if sl:
            sl_bytes = (8.0 * (p.m + p.n) * p.k + head["info"]["slices"] * (p.m + p.n) * p.k) * p.batch
            sl_ms = sl[1] / sl[0]
            roof["pre_pass"] = {"kernel": "ozaki_slice", "bound": "hbm", "unit": "GB/s",
                                "achieved": sl_bytes / (sl_ms * 1e-3) / 1e9, "peak": pk["hbm_gbs"],
                                "frac": sl_bytes / (sl_ms * 1e-3) / 1e9 / pk["hbm_gbs"],
                                "ms_per_launch": sl_ms}
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
            achieved = bytes_ / (per_launch_ms * 1e-3) / 1e9
            roof = {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / pk["hbm_gbs"], "traffic": None, "kernel": dom_name,
                    "peak_source": pk["source"]}
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
        for _ in range(2):
            st, _ = runner.call(W.Problem(**{**p.__dict__, "A": hA, "B": hB}), mode="host_matrices", host_C=hC)
            assert st == 0
        e2e_steps = max(2, min(args.steps, 5))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            st, _ = runner.call(W.Problem(**{**p.__dict__, "A": hA, "B": hB}), mode="host_matrices", host_C=hC)
        t_e2e = (time.perf_counter() - t0) / e2e_steps
        if world > 1:
            t = torch.tensor([t_e2e], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        ab = np.dtype(p.ab_dtype).itemsize
        h2d = p.A.nbytes + p.B.nbytes + (p.C.nbytes if p.beta != 0 else 0)
        d2h = p.m * p.n * np.dtype(p.c_dtype).itemsize * p.batch
        e2e = {"value": flops / t_e2e / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": t_e2e * 1e3,
               "note": "host arrays of host pointers (pinned), copies and synchronous return inside the timed region"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
        sample = {"f64_batch32_1024": 2, "i8_batch512_512": 4, "fp32_batch64_128": 64, "fp32_batch4096_64": 512,
                  "i8_batch8_4096": 1, "f64_batch2_256_8192": 1, "i8_batch64_512_nn": 4}[args.workload]
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
        line = {"metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "i8" if mode == "ozaki" else p.row, "data": "synthetic (seeded)",
                "config": {"workload": args.workload, "batch": p.batch, "m": p.m, "n": p.n, "k": p.k,
                           "transa": "NT"[p.transa], "transb": "NT"[p.transb], "ld": [p.lda, p.ldb, p.ldc],
                           "mode": mode, "emulates": p.row, "parallelism": f"batch-replica x{world}",
                           "l2": "operands larger than L2, no flush", "modes": extra},
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
