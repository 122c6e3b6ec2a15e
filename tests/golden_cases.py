"""Reads the golden fixtures (tests/golden/golden_cases.npz, made by tests/golden/make_golden.py
from the reference library itself) back into workloads.Problem objects."""
import numpy as np

from ssblasex_b200 import workloads as W

ROWS = ["f32", "f64", "i8"]


def load_cases(g):
    for r in g["meta"]:
        i = int(r[0])
        row = ROWS[int(r[1])]
        tag = f"c{i:03d}"
        st = W.ROW_TYPES[row][4]
        p = W.Problem(row, int(r[2]), int(r[3]), int(r[4]), int(r[5]), int(r[6]), int(r[7]),
                      int(r[8]), int(r[9]), int(r[10]), st(r[11]).item(), st(r[12]).item(),
                      g[tag + "_A"], g[tag + "_B"], g[tag + "_C0"], name=tag)
        yield p, g[tag + "_C"], int(r[13])


def load_status_cases(g):
    keys = ("m", "n", "k", "batch", "transa", "transb")
    for r in g["status_meta"]:
        j = int(r[0])
        row = ROWS[int(r[1])]
        tag = f"s{j:03d}"
        st = W.ROW_TYPES[row][4]
        p = W.Problem(row, int(r[2]), int(r[3]), int(r[4]), int(r[5]), int(r[6]), int(r[7]),
                      int(r[8]), int(r[9]), int(r[10]), st(r[11]).item(), st(r[12]).item(),
                      g[tag + "_A"], g[tag + "_B"], g[tag + "_C0"], name=str(g[tag + "_name"]))
        over = {k: int(v) for k, v in zip(keys, r[14:20]) if int(v) != -99}
        types = tuple(int(t) for t in r[20:23])
        if types != tuple(p.types):
            over["types"] = types
        yield p, over, g[tag + "_C"], int(r[13])


def fp_tolerance(p):
    """4 * k * u, normalised by |alpha| |op(A)| |op(B)| + |beta| |C| (u = unit roundoff)."""
    u = {"f32": 2.0 ** -24, "f64": 2.0 ** -53}[p.row]
    return 4.0 * max(p.k, 1) * u


CONFIGS = ["fp32_batch64_128", "f64_batch32_1024", "i8_batch512_512", "fp32_batch4096_64"]


def load_config_case(cfg, name):
    """(problem over the fixture's instances, sampled rows, the reference's output on those rows
    [instance, row, column], its column sums over all rows [instance, column]) of one benchmark
    configuration from tests/golden/config_cases.npz; the inputs are regenerated from the
    workload's seed."""
    full = W.workload(name)
    inst = cfg[name + "_inst"]
    p = W.Problem(**{**full.__dict__, "batch": len(inst), "A": full.A[inst], "B": full.B[inst],
                     "C": full.C[inst].copy(), "name": name})
    return p, cfg[name + "_rows"], cfg[name + "_C"], cfg[name + "_colsum"]


def check_against_config_fixture(p, C, rows, ref_rows, ref_colsum, exact_fn, tol):
    """C (all of p's instances) against the reference's sampled rows and column sums: int8 equal,
    fp within `tol` normalised by |alpha||op(A)||op(B)| + |beta||C| (column sums within the sum of
    the per-entry tolerances of their column, bounded through the row norms)."""
    import numpy as np
    for b in range(p.batch):
        got = p.c_view(C, b)
        if p.row == "i8":
            np.testing.assert_array_equal(got[rows, :], ref_rows[b], err_msg=f"{p.name} instance {b}")
            np.testing.assert_array_equal(got.astype(np.int64).sum(axis=0), ref_colsum[b])
            continue
        ex, nrm = exact_fn(p, b, rows)
        diff = np.abs(got[rows, :].astype(np.float64) - ref_rows[b].astype(np.float64))
        assert np.max(diff / nrm) <= tol, (p.name, b, float(np.max(diff / nrm)))
        # every row enters the column sums: |sum_i (C - C_ref)(i, j)| <= tol * sum_i norm(i, j), and
        # sum_i norm(i, j) = |alpha| sum_k (sum_i |op(A)_ik|) |op(B)_kj| + |beta| sum_i |C0(i, j)|
        a = np.abs(p.op_a(b).astype(np.float64))
        bb = np.abs(p.op_b(b).astype(np.float64))
        c0 = np.abs(p.c_view(p.C, b).astype(np.float64))
        col_norm = abs(p.alpha) * (a.sum(axis=0) @ bb) + abs(p.beta) * c0.sum(axis=0)
        d = np.abs(got.astype(np.float64).sum(axis=0) - ref_colsum[b])
        assert np.all(d <= tol * col_norm + 1e-300), (p.name, b)
