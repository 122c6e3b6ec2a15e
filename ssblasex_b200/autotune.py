"""Autotuner: times every configuration of each tensor-core kernel family on representative
problems and writes the winners, per power-of-two size bucket, to the library's tuning table
(ssblasex_b200/tune/ssblas_tune.json, read by csrc/tune.cpp).

    python -m ssblasex_b200.autotune [--out PATH] [--quick]

Each candidate is checked against the default configuration's result before it can win (bit for
bit on the integer and Ozaki paths, whose arithmetic does not depend on the tiling).
"""
from __future__ import annotations

import argparse
import json
import pathlib
import time

import numpy as np

from . import PATH_IDS, get_profile, lib, set_kernel_config, set_math_mode, set_profiling, set_sync_mode
from . import SSBLAS_MATH_FP32_BF16X3, SSBLAS_MATH_FP64_OZAKI, SSBLAS_MATH_PLAIN
from . import runner, workloads as W

OUT = pathlib.Path(__file__).resolve().parent / "tune" / "ssblas_tune.json"

# path -> (math mode, configurations, kernel name, problems)
FAMILIES = {
    "ozaki_tcgen05": (SSBLAS_MATH_FP64_OZAKI, [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11], "ozaki_gemm", [
        dict(row="f64", transa=0, transb=1, m=1024, n=1024, k=1024, batch=32, alpha=1.0, beta=0.0,
             lda=1032, ldb=1032, ldc=1032, dist="expspread"),
        dict(row="f64", transa=0, transb=0, m=512, n=512, k=512, batch=64, alpha=1.0, beta=0.0,
             dist="expspread"),
        dict(row="f64", transa=1, transb=0, m=256, n=256, k=2048, batch=32, alpha=1.0, beta=0.0,
             dist="expspread"),
    ]),
    # slicing pre-pass of the Ozaki path: two passes (1: digits per 32 x 128 chunk; 7: digits by
    # persistent CTAs over 16 x 512 slabs) or one pass with thread-block clusters of 32 x 256 (2),
    # 16 x 512 (3) or 8 x 1024 (4) per 512-thread CTA, or 16 x 256 per 256-thread CTA, two CTAs
    # per SM (5) -- the cluster size is ceil(k / that K)
    "ozaki_slicer": (SSBLAS_MATH_FP64_OZAKI, [1, 2, 3, 4, 5, 7], "(all)", [
        dict(row="f64", transa=0, transb=1, m=1024, n=1024, k=1024, batch=32, alpha=1.0, beta=0.0,
             lda=1032, ldb=1032, ldc=1032, dist="expspread"),
        dict(row="f64", transa=1, transb=0, m=256, n=256, k=2048, batch=32, alpha=1.0, beta=0.0,
             dist="expspread"),
    ]),
    # split-K factor (K pieces per output tile) of the Ozaki GEMM, on shapes with few tiles
    "splitk_ozaki": (SSBLAS_MATH_FP64_OZAKI, [1, 2, 4, 8, 16], "(all)", [
        dict(row="f64", transa=1, transb=0, m=256, n=256, k=8192, batch=2, alpha=1.0, beta=0.0,
             dist="expspread"),
        dict(row="f64", transa=0, transb=1, m=512, n=512, k=4096, batch=1, alpha=1.0, beta=0.0,
             dist="expspread"),
    ]),
    "splitk_i8": (SSBLAS_MATH_PLAIN, [1, 2, 4, 8, 16], "i8_gemm", [
        dict(row="i8", transa=1, transb=0, m=512, n=512, k=16384, batch=1, alpha=1, beta=0,
             lda=16384, ldb=16384, ldc=512),
        dict(row="i8", transa=1, transb=0, m=1024, n=1024, k=8192, batch=2, alpha=1, beta=0,
             lda=8192, ldb=8192, ldc=1024),
    ]),
    "i8_tcgen05": (SSBLAS_MATH_PLAIN, [0, 1], "i8_gemm", [
        dict(row="i8", transa=1, transb=0, m=512, n=512, k=512, batch=512, alpha=1, beta=1,
             lda=512, ldb=512, ldc=512),
        dict(row="i8", transa=1, transb=0, m=256, n=256, k=1024, batch=512, alpha=1, beta=0,
             lda=1024, ldb=1024, ldc=256),
    ]),
    "dmma": (SSBLAS_MATH_PLAIN, [0, 1, 3, 4], "dmma_gemm", [
        dict(row="f64", transa=0, transb=1, m=1024, n=1024, k=1024, batch=32, alpha=1.0, beta=0.0,
             lda=1032, ldb=1032, ldc=1032, dist="expspread"),
        dict(row="f64", transa=1, transb=0, m=128, n=128, k=128, batch=256, alpha=1.0, beta=0.5),
    ]),
    "simt": (SSBLAS_MATH_PLAIN, [0, 1, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13], "(all)", [
        dict(row="f32", transa=0, transb=0, m=128, n=128, k=128, batch=64, alpha=1.0, beta=0.5),
        dict(row="f32", transa=1, transb=1, m=64, n=64, k=64, batch=4096, alpha=0.75, beta=0.25,
             dist="outliers"),
    ]),
    "bf16x3_tcgen05": (SSBLAS_MATH_FP32_BF16X3, [0, 1, 2], "(all)", [
        dict(row="f32", transa=1, transb=1, m=64, n=64, k=64, batch=4096, alpha=0.75, beta=0.25,
             dist="outliers"),
        dict(row="f32", transa=0, transb=0, m=256, n=256, k=256, batch=256, alpha=1.0, beta=0.0),
    ]),
}


def bucket(m, n, k, batch):
    c = lambda x: max(0, int(np.ceil(np.log2(max(x, 1)))))
    return f"m{c(m)}n{c(n)}k{c(k)}b{c(batch)}"


def time_kernel(p, dp, kernel, reps):
    import torch
    al = np.array([p.alpha], p.scale_dtype)
    be = np.array([p.beta], p.scale_dtype)
    Ah, Bh, Ch = dp.host_arrays()
    ta, tb, tc = p.types
    call = lambda: lib().ssblasGemmBatchedEx(p.transa, p.transb, p.m, p.n, p.k, al.ctypes.data, Ah, ta, p.lda,
                                             Bh, tb, p.ldb, be.ctypes.data, Ch, tc, p.ldc, p.batch, 0, 0)
    set_sync_mode(False)
    for _ in range(2):
        assert call() == 0
    torch.cuda.synchronize()
    set_profiling(True)
    # a spin kernel ahead of the calls keeps them all enqueued before the GPU starts them, so the
    # per-launch events time kernels, not the host's per-call work between them
    torch.cuda._sleep(int(reps * 80e-6 * 2.0e9))
    for _ in range(reps):
        assert call() == 0
    prof = get_profile()
    set_profiling(False)
    set_sync_mode(True)
    if kernel in prof:
        n, ms = prof[kernel]
        return ms / max(n, 1)
    # configurations of one family may run different kernels: time the whole call
    return sum(ms for _, ms in prof.values()) / reps


# grouped calls: the Ozaki tile shape per instance size bucket (0: 128 x 64 tiles, one
# accumulator; 1: 128 x 32 tiles, two), timed on groups of equal-size instances (m, n, k)
GROUPED_OZAKI_BUCKETS = [(64, 64, 64), (128, 128, 128), (256, 256, 256), (512, 512, 512), (64, 64, 512),
                         (256, 256, 64), (512, 64, 512), (128, 128, 512), (256, 256, 512)]


def time_grouped(gd, reps):
    import torch
    set_sync_mode(False)
    for _ in range(3):                     # plan, capture, first replay
        assert gd.call(device_arrays=True) == 0
    torch.cuda.synchronize()
    set_profiling(True)
    torch.cuda._sleep(int(reps * 80e-6 * 2.0e9))
    for _ in range(reps):
        assert gd.call(device_arrays=True) == 0
    prof = get_profile()
    set_profiling(False)
    set_sync_mode(True)
    return sum(ms for _, ms in prof.values()) / reps


def tune_grouped_ozaki(entries, report, quick):
    from . import release_workspace
    set_math_mode(SSBLAS_MATH_FP64_OZAKI)
    for m, n, k in GROUPED_OZAKI_BUCKETS[: 2 if quick else None]:
        count = max(8, min(600, (1 << 27) // (m * n * k)))
        probs = [W.make_problem("f64", i % 2, (i // 2) % 2, m, n, k, 1, 1.0, 0.0, seed=300 + i, dist="expspread",
                                name=f"t{i}") for i in range(count)]
        gd = runner.GroupedDevice(probs)
        times, ref = {}, None
        for cfg in (0, 1):
            set_kernel_config("grouped_ozaki_tile", cfg)
            gd.reset_c()
            assert gd.call(device_arrays=True) == 0
            res = np.concatenate([c.ravel() for c in gd.results()])
            if ref is None:
                ref = res
            elif not np.array_equal(res.view(np.uint64), ref.view(np.uint64)):
                continue
            times[cfg] = time_grouped(gd, 5)
        set_kernel_config("grouped_ozaki_tile", -1)
        release_workspace()               # drop the cached grouped plan
        best = min(times, key=times.get)
        b = bucket(m, n, k, 1)
        entries.append({"path": PATH_IDS["grouped_ozaki_tile"], "bucket": b, "config": best})
        report.append({"family": "grouped_ozaki_tile", "bucket": b, "instances": count, "ms": times, "best": best})
        print(json.dumps(report[-1]), flush=True)
    set_math_mode(SSBLAS_MATH_PLAIN)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(OUT))
    ap.add_argument("--quick", action="store_true")
    args = ap.parse_args()
    entries, report = [], []
    for family, (mode, configs, kernel, probs) in FAMILIES.items():
        set_math_mode(mode)
        for kw in probs[: 1 if args.quick else None]:
            p = W.make_problem(seed=7, **kw)
            dp = runner.DeviceProblem(p)
            ref = None
            times = {}
            for cfg in configs:
                set_kernel_config(family, cfg)
                dp.reset_c()
                st, C = runner.call(p, mode="host_array", dp=dp)
                assert st == 0
                if ref is None:
                    ref = C
                elif p.row == "f32":
                    if not np.allclose(C, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max()):
                        continue
                elif not np.array_equal(C.view(np.uint8), ref.view(np.uint8)):
                    continue          # a configuration that disagrees never wins
                times[cfg] = time_kernel(p, dp, kernel, 5)
            set_kernel_config(family, -1)
            best = min(times, key=times.get)
            b = bucket(p.m, p.n, p.k, p.batch)
            entries.append({"path": PATH_IDS[family], "bucket": b, "config": best})
            report.append({"family": family, "bucket": b, "ms": times, "best": best})
            print(json.dumps(report[-1]), flush=True)
    tune_grouped_ozaki(entries, report, args.quick)
    set_math_mode(SSBLAS_MATH_PLAIN)
    out = pathlib.Path(args.out)
    out.parent.mkdir(parents=True, exist_ok=True)
    lines = [json.dumps(e) for e in entries]
    out.write_text("{\"version\": 1, \"generated\": \"%s\", \"entries\": [\n%s\n]}\n"
                   % (time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), ",\n".join(lines)))
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
