"""Error bounds the tests check results against (test helpers, no GPU).

ozaki_bound: the a-priori bound of the Ozaki FP64 emulation stated in include/ssblasBatch.h,
    |C - C*| <= |alpha| k 2^(e_i + f_j) (S + 1) 2^(2 - 8S) + (S + 1) u (|alpha| |op(A)||op(B)| + |beta C|)
where 2^e_i (2^f_j) is the smallest power of two above max_k |op(A)_ik| (max_k |op(B)_kj|).
"""
import numpy as np

U64 = 2.0 ** -53


def pow2_above(x: np.ndarray, axis: int) -> np.ndarray:
    """2^e with max |x| < 2^e along `axis` (1.0 for an all-zero line)."""
    mx = np.max(np.abs(x), axis=axis)
    e = np.frexp(mx)[1]
    return np.where(mx > 0, np.ldexp(1.0, e), 1.0)


def term_bound(S: int) -> float:
    return (S + 1) * 2.0 ** (2 - 8 * S)


def ozaki_bound(p, b: int, rows, S: int, norm: np.ndarray) -> np.ndarray:
    """Per-entry bound for instance b on `rows` (norm: |alpha||op(A)||op(B)| + |beta||C0| of those
    entries, as the FP64-exact oracle returns it)."""
    ea = pow2_above(p.op_a(b)[np.asarray(rows)], axis=1)        # rows of op(A)
    fb = pow2_above(p.op_b(b), axis=0)                          # columns of op(B)
    scale = abs(p.alpha) * p.k * np.outer(ea, fb)
    return scale * term_bound(S) + (S + 1) * U64 * norm


def check_ozaki(p, C: np.ndarray, S: int, instances, rows, exact_fn) -> float:
    """Asserts the stated bound on the sampled entries; returns the largest ratio error / bound."""
    worst = 0.0
    rows = np.asarray(rows)
    for b in instances:
        ex, nrm = exact_fn(p, b, rows)
        got = p.c_view(C, b)[rows, :].astype(np.float64)
        bound = ozaki_bound(p, b, rows, S, nrm)
        err = np.abs(got - ex)
        assert np.all(np.isfinite(got)), "non-finite output"
        assert np.all(err <= bound), (b, float(np.max(err / bound)))
        worst = max(worst, float(np.max(err / bound)))
    return worst
