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
