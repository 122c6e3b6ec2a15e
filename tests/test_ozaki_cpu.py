"""CPU checks of the Ozaki emulation's host-side rules (no GPU): the 32-bit row-maximum key the
slicing kernels reduce gives the exponent of the true row maximum, and the CPU restatement of the
emulation (the bit-exact target of the GPU tests) stays within its error bound and follows the
Inf/NaN rule."""
import numpy as np
import pytest

from oracle import oracle as O

NONFINITE = 4096


def true_exponent(x: np.ndarray) -> int:
    """e with max|x| < 2^e (0 for an all-zero row), or the non-finite sentinel."""
    if not np.all(np.isfinite(x)):
        return NONFINITE
    m = np.max(np.abs(x)) if x.size else 0.0
    return int(np.frexp(m)[1]) if m > 0 else 0


def key_exponent(x: np.ndarray) -> int:
    """The slicing kernels' rule: key = max high word of |x| << 32 when that is nonzero, else the
    maximum low word; the exponent is taken from the key read back as a double."""
    u = x.view(np.uint64)
    hi = ((u >> np.uint64(32)) & np.uint64(0x7FFFFFFF)).astype(np.uint64)
    lo = (u & np.uint64(0xFFFFFFFF)).astype(np.uint64)
    mh = int(hi.max()) if x.size else 0
    key = (mh << 32) if mh else (int(lo.max()) if x.size else 0)
    if key >= 0x7FF0000000000000:
        return NONFINITE
    m = np.array([key], np.uint64).view(np.float64)[0]
    return int(np.frexp(m)[1]) if m > 0 else 0


def _rows(rng, n=600, k=97):
    """Rows spanning every case the key distinguishes."""
    tiny = 2.0 ** -1074
    rows = []
    for i in range(n):
        kind = i % 8
        if kind == 0:
            r = rng.standard_normal(k) * 2.0 ** rng.integers(-60, 60)
        elif kind == 1:
            r = rng.integers(-2 ** 31, 2 ** 31, k) * tiny          # below 2^-1042: high words zero
        elif kind == 2:
            r = rng.integers(-2 ** 51, 2 ** 51, k) * tiny          # subnormals above 2^-1042
        elif kind == 3:
            r = rng.integers(-2 ** 20, 2 ** 20, k) * tiny
            r[rng.integers(k)] = rng.standard_normal() * 2.0 ** -1000
        elif kind == 4:
            r = np.zeros(k)
            r[rng.integers(k)] = -0.0
        elif kind == 5:
            r = rng.standard_normal(k)
            r[rng.integers(k)] = [np.inf, -np.inf, np.nan][i % 3]
        elif kind == 6:
            # values that differ only in their low words: the key keeps the high word, which
            # fixes the exponent
            base = 2.0 ** int(rng.integers(-1000, 1000))
            r = base * (1.0 + rng.integers(0, 2 ** 20, k) * 2.0 ** -52) * rng.choice([-1.0, 1.0], k)
        else:
            r = np.full(k, 2.0 ** int(rng.integers(-1074, 1023)))  # exact powers of two
        rows.append(np.ascontiguousarray(r, dtype=np.float64))
    return rows


def test_row_key_gives_the_true_exponent():
    rng = np.random.default_rng(42)
    for r in _rows(rng):
        assert key_exponent(r) == true_exponent(r), r[:4]


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_ozaki_restatement_error_bound(ta, tb):
    """S = 7 (28 slice-pair products): max normalised error below the 4 k u bound that the GPU
    tests apply to plain FP64, on exponent-spread inputs."""
    from ssblasex_b200 import workloads as W
    p = W.make_problem("f64", ta, tb, 37, 29, 211, 2, 1.25, -0.5, seed=ta + 2 * tb, dist="expspread")
    st, C = O.ozaki_f64(p, 7)
    assert st == 0
    assert O.normalized_error(p, C) <= 4 * p.k * 2.0 ** -53


def test_ozaki_restatement_nonfinite_rule():
    """A row of op(A) or column of op(B) holding an Inf or a NaN turns exactly the C(i, j) it
    touches into the quiet NaN 0x7ff8000000000000; every other entry stays finite."""
    from ssblasex_b200 import workloads as W
    p = W.make_problem("f64", 0, 0, 20, 15, 33, 1, 1.0, 0.0, seed=5, dist="expspread")
    p.op_a(0)[4, 7] = np.inf
    p.op_b(0)[3, 9] = np.nan
    st, C = O.ozaki_f64(p, 7)
    assert st == 0
    got = p.c_view(C, 0)
    nan = np.zeros((p.m, p.n), bool)
    nan[4, :] = True
    nan[:, 9] = True
    np.testing.assert_array_equal(np.isnan(got), nan)
    assert np.all(got[nan].view(np.uint64) == np.uint64(0x7FF8000000000000))


def test_exponent_reduction_with_zero_sentinel():
    """The clusters-of-one slicing path reduces per-thread exponents instead of keys: a thread
    whose values are all zero contributes a sentinel below every exponent, and the maximum over
    the threads is the exponent of the whole row (0 for a zero row)."""
    rng = np.random.default_rng(7)
    sentinel = -0x40000000
    for r in _rows(rng, n=160, k=96):
        parts = np.split(np.concatenate([r, np.zeros(32)]), 8)   # zero fill past k, as in a slab
        es = [key_exponent(q) if np.any(q.view(np.uint64) & np.uint64(0x7FFFFFFFFFFFFFFF)) else sentinel
              for q in parts]
        e = max(es)
        assert (0 if e == sentinel else e) == true_exponent(r)


@pytest.mark.parametrize("S", [3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("dist", ["expspread", "expspread30", "uniform", "outliers"])
def test_ozaki_restatement_meets_the_stated_bound(S, dist):
    """The a-priori bound of include/ssblasBatch.h holds entry by entry for every slice count, on
    rows whose entries span up to 2^+-30 (where the small entries keep few of their bits) and on
    the other input distributions; the GPU result equals this restatement bit for bit."""
    from ssblasex_b200 import workloads as W
    from bounds import check_ozaki
    for ta, tb in [(0, 1), (1, 0)]:
        p = W.make_problem("f64", ta, tb, 23, 19, 157, 2, -1.5, 0.25, seed=S * 10 + ta, dist=dist)
        st, C = O.ozaki_f64(p, S)
        assert st == 0
        check_ozaki(p, C, S, range(p.batch), np.arange(p.m), O.exact_f64)


def test_ozaki_bound_is_tight_enough_to_choose_the_slices():
    """Rows of a single power of two against full-mantissa columns: the dropped pairs and the
    rounding then sit near their worst case, and the measured error approaches the bound's first
    term (the bound is not vacuous)."""
    from ssblasex_b200 import workloads as W
    from bounds import term_bound
    p = W.make_problem("f64", 0, 0, 16, 16, 64, 1, 1.0, 0.0, seed=3, dist="uniform")
    p.op_a(0)[:] = np.where(np.random.default_rng(1).random((16, 64)) < 0.5, -1.0, 1.0) * (1 - 2.0 ** -30)
    st, C = O.ozaki_f64(p, 3)
    ex, _ = O.exact_f64(p, 0)
    err = np.max(np.abs(p.c_view(C, 0) - ex))
    assert err > 1e-3 * p.k * term_bound(3)


def test_slice_count_follows_the_tolerance():
    """The automatic count is the smallest S in 3..8 with (S + 1) 2^(2 - 8S) <= tolerance; the
    default tolerance 2^-51 gives 7. Refused: negative or NaN tolerances, and ones below the
    8-slice bound."""
    import ssblasex_b200 as S
    from bounds import term_bound
    try:
        assert S.set_ozaki_slices(0) == 0
        assert S.set_ozaki_tolerance(0) == 0 and S.get_ozaki_slices() == 7
        for tol in [2.0 ** -20, 2.0 ** -30, 2.0 ** -40, 2.0 ** -45, 2.0 ** -51, 2.0 ** -55, 2.0 ** -58.5, 1.0]:
            assert S.set_ozaki_tolerance(tol) == 0
            want = next((s for s in range(3, 8) if term_bound(s) <= tol), 8)
            assert S.get_ozaki_slices() == want, (tol, want)
        assert S.set_ozaki_tolerance(2.0 ** -20) == 0 and S.get_ozaki_slices() == 3
        assert S.set_ozaki_tolerance(term_bound(7)) == 0 and S.get_ozaki_slices() == 7
        assert S.set_ozaki_tolerance(term_bound(7) * 0.999) == 0 and S.get_ozaki_slices() == 8
        for bad in [-1.0, float("nan"), term_bound(8) / 2]:
            assert S.set_ozaki_tolerance(bad) == S.SSBLAS_STATUS_INVALID_VALUE
        assert S.set_ozaki_slices(5) == 0 and S.get_ozaki_slices() == 5   # a fixed count wins
    finally:
        S.set_ozaki_slices(0)
        S.set_ozaki_tolerance(0)
