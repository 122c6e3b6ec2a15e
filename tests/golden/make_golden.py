"""Generate the golden fixtures in this directory from the reference library itself.

The reference (hirokitokura/ssblasEx) is compiled from its own sources by oracle/Makefile into
oracle/_ref/libssblas_ref.so (x86 build; see oracle/ref_x86_build.cpp). This script runs it on
small seeded problems and stores inputs, outputs and status codes in golden_cases.npz.

    OMP_NUM_THREADS=8 python tests/golden/make_golden.py

The fixtures are committed; tests read them and never need the reference tree.
"""
from __future__ import annotations

import os
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from ssblasex_b200 import workloads as W  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent / "golden_cases.npz"

ALPHAS = {"f32": [1.0, 0.75, 2.0, 0.0], "f64": [1.0, 0.75, 2.0, 0.0], "i8": [1, 2, -3, 0]}
BETAS = {"f32": [0.0, 1.0, -3.0, 0.5], "f64": [0.0, 1.0, -3.0, 0.5], "i8": [0, 1, -3, 2]}


def cases():
    seed = 100
    # odd and tail shapes over all four N/T combinations, with ld > stored rows
    shapes = [(37, 29, 45), (1, 1, 1), (8, 1, 8), (65, 33, 64), (33, 17, 129)]
    for row in ("f32", "f64", "i8"):
        for si, (m, n, k) in enumerate(shapes):
            for ta in (W.OP_N, W.OP_T):
                for tb in (W.OP_N, W.OP_T):
                    seed += 1
                    pad = 3 + (seed % 5)
                    ar, _ = W.stored_shape(ta, m, k)
                    br, _ = W.stored_shape(tb, k, n)
                    al = ALPHAS[row][(si + ta) % 4]
                    be = BETAS[row][(si + tb + ta) % 4]
                    yield dict(row=row, transa=ta, transb=tb, m=m, n=n, k=k, batch=2 if si < 3 else 1, alpha=al,
                               beta=be, lda=ar + pad, ldb=br + (pad if si % 2 else 0),
                               ldc=m + (pad if si % 2 == 0 else 0), seed=seed)
    # K crossing the reference's 512-wide K blocks (two and three blocks)
    for row in ("f32", "f64", "i8"):
        for (ta, tb), (m, n, k) in zip([(0, 0), (1, 0), (0, 1), (1, 1)],
                                       [(20, 12, 1030), (9, 14, 513), (16, 5, 1024), (7, 9, 600)]):
            seed += 1
            yield dict(row=row, transa=ta, transb=tb, m=m, n=n, k=k, batch=1,
                       alpha=ALPHAS[row][1], beta=BETAS[row][3], seed=seed)
    # int8 wrap-around: alpha and C large enough that int32 arithmetic overflows
    seed += 1
    yield dict(row="i8", transa=0, transb=1, m=19, n=23, k=300, batch=2, alpha=1 << 20,
               beta=1 << 12, seed=seed)
    # the exponent-spread fp64 distribution of the 32 x 1024^3 workload, small
    seed += 1
    yield dict(row="f64", transa=0, transb=1, m=40, n=36, k=200, batch=2, alpha=1.0, beta=0.0,
               lda=48, ldb=40, ldc=48, seed=seed, dist="expspread")
    # the 1%-outlier fp32 distribution of the 4096 x 64^3 workload, small
    seed += 1
    yield dict(row="f32", transa=1, transb=1, m=64, n=64, k=64, batch=1, alpha=0.75, beta=0.25,
               seed=seed, dist="outliers")


def status_cases():
    """Degenerate calls whose status and effect on C are pinned on the reference."""
    base = dict(row="f32", transa=0, transb=0, m=5, n=4, k=3, batch=2, alpha=1.0, beta=0.5, seed=9)
    yield "m0", base, dict(m=0)
    yield "n0", base, dict(n=0)
    yield "batch0", base, dict(batch=0)
    yield "k0", base, dict(k=0)
    yield "opC_f32", base, dict(transa=2)
    yield "opC_f64", dict(base, row="f64"), dict(transb=2)
    yield "bad_types", base, dict(types=(W.R_32F, W.R_64F, W.R_32F))
    yield "r16f", base, dict(types=(W.R_16F, W.R_16F, W.R_16F))
    yield "k0_i8", dict(base, row="i8", alpha=1, beta=2), dict(k=0)
    yield "m0_i8", dict(base, row="i8", alpha=1, beta=2), dict(m=0)


# The benchmark configurations at their full shapes: the reference runs on the instances listed
# (all of the 64 x 128^3 workload, a slice of the larger ones); the fixture keeps its output on
# sampled rows of those instances plus the column sums over all rows (int64 for the int8 row, so
# those compare exactly). The inputs are not stored: tests regenerate them from the workload's seed
# (tests/test_oracle_golden.py checks that the regenerated inputs are the ones the reference saw).
CONFIG_FIXTURES = [
    ("fp32_batch64_128", list(range(64)), list(range(0, 128, 9))),
    ("f64_batch32_1024", [0, 1], list(range(5, 1024, 67))),
    ("i8_batch512_512", [0, 1], list(range(3, 512, 37))),
    ("fp32_batch4096_64", list(range(0, 4096, 256)), list(range(64))),
]
CONFIG_OUT = pathlib.Path(__file__).resolve().parent / "config_cases.npz"


def config_fixtures():
    out = {}
    for name, inst, rows in CONFIG_FIXTURES:
        full = W.workload(name)
        q = W.Problem(**{**full.__dict__, "batch": len(inst), "A": full.A[inst], "B": full.B[inst],
                         "C": full.C[inst].copy()})
        st, C = O.reference_gemm(q)
        assert st == 0, (name, st)
        views = [q.c_view(C, b) for b in range(q.batch)]
        out[name + "_inst"] = np.array(inst, np.int64)
        out[name + "_rows"] = np.array(rows, np.int64)
        out[name + "_C"] = np.stack([v[rows, :] for v in views])
        acc = np.int64 if q.row == "i8" else np.float64
        out[name + "_colsum"] = np.stack([v.astype(acc).sum(axis=0) for v in views])
        print(f"  {name}: {len(inst)} instances")
    np.savez_compressed(CONFIG_OUT, **out)
    print(f"wrote {CONFIG_OUT} ({CONFIG_OUT.stat().st_size / 1e6:.2f} MB)")


def main():
    if os.environ.get("OMP_NUM_THREADS", "").strip() in {"2", "3", "4", "6"}:
        raise SystemExit("OMP_NUM_THREADS in {2,3,4,6} crashes the reference")
    config_fixtures()
    out = {}
    meta = []
    for i, kw in enumerate(cases()):
        p = W.make_problem(**kw)
        st, C = O.reference_gemm(p)
        assert st == 0, (kw, st)
        tag = f"c{i:03d}"
        out[tag + "_A"], out[tag + "_B"], out[tag + "_C0"], out[tag + "_C"] = p.A, p.B, p.C, C
        meta.append([i, ["f32", "f64", "i8"].index(p.row), p.transa, p.transb, p.m, p.n, p.k,
                     p.lda, p.ldb, p.ldc, p.batch, float(p.alpha), float(p.beta), st])
    out["meta"] = np.array(meta, dtype=np.float64)
    smeta = []
    for j, (name, kw, over) in enumerate(status_cases()):
        p = W.make_problem(**kw)
        st, C = O.reference_gemm(p, **over)
        tag = f"s{j:03d}"
        out[tag + "_name"] = np.array(name)
        out[tag + "_A"], out[tag + "_B"], out[tag + "_C0"], out[tag + "_C"] = p.A, p.B, p.C, C
        ov = [over.get(key, -99) for key in ("m", "n", "k", "batch", "transa", "transb")]
        types = over.get("types", p.types)
        smeta.append([j, ["f32", "f64", "i8"].index(p.row), p.transa, p.transb, p.m, p.n, p.k,
                      p.lda, p.ldb, p.ldc, p.batch, float(p.alpha), float(p.beta), st,
                      *ov, *types])
    out["status_meta"] = np.array(smeta, dtype=np.float64)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e6:.2f} MB, {len(meta)} cases, {len(smeta)} status cases)")


if __name__ == "__main__":
    main()


def dump_text(lib_path: str) -> str:
    """stdout of one call of `lib_path`'s ssblasGemmBatchedEx with SSBLAS_GEMMBATCHEDEX_DEBUG set
    (the call itself is degenerate: batchCount 0, so nothing is computed)."""
    import subprocess
    code = (
        "import ctypes as ct\n"
        f"L = ct.CDLL({lib_path!r})\n"
        "vp, l, i = ct.c_void_p, ct.c_long, ct.c_int\n"
        "L.ssblasGemmBatchedEx.argtypes = [i, i, l, l, l, vp, vp, i, l, vp, i, l, vp, vp, i, l, l, i, i]\n"
        "a = ct.c_double(1.0)\n"
        "arr = (vp * 1)()\n"
        "for args in [(1, 0, 7, 5, 3, 5, 10, 3, 12, 5, 7, 0, 0), (2, 9, 0, 1, 2, 0, 1, 4, 3, 0, 0, 1, 1),"
        " (0, 1, 64, 128, 256, 4, 70, 4, 256, 4, 80, 2, 2)]:\n"
        "    ta, tb, m, n, k, at, lda, bt, ldb, ct_, ldc, comp, algo = args\n"
        "    L.ssblasGemmBatchedEx(ta, tb, m, n, k, ct.addressof(a), arr, at, lda, arr, bt, ldb,"
        " ct.addressof(a), arr, ct_, ldc, 0, comp, algo)\n")
    env = dict(os.environ, SSBLAS_GEMMBATCHEDEX_DEBUG="1", OMP_NUM_THREADS="1")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env)
    return r.stdout


if __name__ == "__main__" and os.environ.get("SSBLAS_GOLDEN_DUMP", "1") == "1":
    txt = dump_text(str(ROOT / "oracle" / "_ref" / "libssblas_ref.so"))
    (OUT.parent / "debug_dump.txt").write_text(txt)
    print(f"wrote debug_dump.txt ({len(txt.splitlines())} lines)")
