"""ssblasGemmGroupedBatchedEx on a B200: uneven instances of every kind in one call, each checked
against its CPU restatement (Ozaki bit-exact, int8 bit-exact, BF16x3 and plain fp within their
bounds), first as a fresh plan and then as a replayed CUDA graph."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mixed(count=60, seed=9):
    from ssblasex_b200 import workloads as W
    probs = W.grouped_problems(count=count, seed=seed, lo=1, hi=300)
    rng = np.random.default_rng(seed)
    # a few int8 instances and non-zero beta to cover every epilogue
    for i in range(0, count, 7):
        p = probs[i]
        probs[i] = W.make_problem("i8", p.transa, p.transb, p.m, p.n, p.k, 1, 2, -1, seed=seed + i)
    for i in range(3, count, 11):
        p = probs[i]
        probs[i] = W.make_problem(p.row, p.transa, p.transb, p.m, p.n, p.k, 1, 0.5, 1.5, seed=seed + 1000 + i)
    return probs


def _check(p, C, mode):
    if p.row == "i8":
        np.testing.assert_array_equal(C, O.restated_gemm(p)[1], err_msg=p.name)
    elif p.row == "f64" and mode & 1:
        np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, 7)[1].view(np.uint64), err_msg=p.name)
    elif p.row == "f32" and mode & 2:
        emu = O.bf16x3_f32(p, 0)
        ex, nrm = O.exact_f64(p, 0)
        got = p.c_view(C, 0).astype(np.float64)
        assert np.max(np.abs(got - emu) / nrm) <= 4 * p.k * 2.0 ** -24, p.name
    else:
        u = 2.0 ** -24 if p.row == "f32" else 2.0 ** -53
        assert O.normalized_error(p, C) <= 4 * p.k * u, p.name


@pytest.mark.parametrize("mode", [0, 3])
@pytest.mark.parametrize("device_arrays", [True, False])
def test_grouped_mixed_kinds(mode, device_arrays):
    import ssblasex_b200 as S
    from ssblasex_b200 import runner
    S.set_math_mode(mode)
    try:
        probs = _mixed()
        gd = runner.GroupedDevice(probs)
        for rep in range(3):            # plan, capture, replay
            gd.reset_c()
            assert gd.call(device_arrays=device_arrays) == 0
            res = gd.results()
            for p, C in zip(probs, res):
                _check(p, C, mode)
        assert S.last_run_info()["path"] == "grouped"
    finally:
        S.set_math_mode(0)


def test_grouped_status_conventions():
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    probs = [W.make_problem("f32", 0, 0, 5, 4, 3, 1, 1.0, 0.0, seed=1) for _ in range(3)]
    gd = runner.GroupedDevice(probs)
    gd.m[1] = 0
    assert gd.call() == S.SSBLAS_STATUS_INTERNAL_ERROR
    gd.m[1] = 5
    gd.ta[2] = 2
    assert gd.call() == S.SSBLAS_STATUS_INVALID_VALUE
    gd.ta[2] = 0
    gd.k[0] = 0                        # k = 0: that instance's C stays untouched
    gd.reset_c()
    assert gd.call() == 0
    np.testing.assert_array_equal(gd.results()[0], probs[0].C)


def test_grouped_long_k_instances():
    """Instances whose K spans many pre-pass chunks (and an odd number of K blocks), in every
    layout, next to small ones: Ozaki bit-exact, BF16x3 and int8 within their bounds."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    probs = []
    for i, (ta, tb) in enumerate([(0, 0), (0, 1), (1, 0), (1, 1)]):
        probs.append(W.make_problem("f64", ta, tb, 70 + 31 * i, 45 + 17 * i, 1100 - 97 * i, 1, 1.0, 0.0,
                                    seed=300 + i, dist="expspread"))
        probs.append(W.make_problem("f32", ta, tb, 90 + 13 * i, 33 + 29 * i, 900 + 61 * i, 1, 0.5, 0.25,
                                    seed=400 + i))
        probs.append(W.make_problem("i8", ta, tb, 40 + 9 * i, 70 + 5 * i, 1000 + 33 * i, 1, 1, 1, seed=500 + i))
    probs += W.grouped_problems(count=12, seed=3, lo=1, hi=64)
    S.set_math_mode(3)
    try:
        gd = runner.GroupedDevice(probs)
        for rep in range(2):
            gd.reset_c()
            assert gd.call(device_arrays=True) == 0
            for p, C in zip(probs, gd.results()):
                _check(p, C, 3)
    finally:
        S.set_math_mode(0)


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_grouped_ozaki_tile_configurations(cfg):
    """Every configuration of the grouped path (0: 128 x 64 Ozaki tiles, one accumulator, tiles
    from the device-side queue; 1: 128 x 32 tiles, two accumulators, queue; 2: 128 x 32 tiles in
    the static order) gives the bit-exact Ozaki result, fresh and replayed."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner
    S.set_math_mode(3)
    S.set_kernel_config("grouped", cfg)
    try:
        probs = _mixed(count=40, seed=17)
        gd = runner.GroupedDevice(probs)
        for rep in range(3):
            gd.reset_c()
            assert gd.call(device_arrays=True) == 0
            for p, C in zip(probs, gd.results()):
                _check(p, C, 3)
    finally:
        S.set_kernel_config("grouped", -1)
        S.set_math_mode(0)


def test_grouped_ozaki_nonfinite_inputs():
    """The grouped Ozaki path follows the batched path's rule for Inf and NaN entries (zero
    digits for the row / column, quiet NaN in every C(i, j) it touches), bit-exact against the
    CPU restatement."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    probs = [W.make_problem("f64", ta, tb, 40 + 17 * i, 33 + 9 * i, 90 + 61 * i, 1, 1.0, 0.0, seed=700 + i,
                            dist="expspread") for i, (ta, tb) in enumerate([(0, 0), (1, 1), (0, 1), (1, 0)])]
    probs[0].op_a(0)[5, 2] = np.inf
    probs[1].op_b(0)[7, 4] = np.nan
    probs[2].op_a(0)[0, 0] = -np.inf
    probs[2].op_b(0)[3, 30] = np.inf
    S.set_math_mode(1)
    try:
        gd = runner.GroupedDevice(probs)
        for rep in range(2):
            gd.reset_c()
            assert gd.call(device_arrays=True) == 0
            for p, C in zip(probs, gd.results()):
                _check(p, C, 1)
        res = gd.results()
        assert np.isnan(res[0][0][5 + 0 * probs[0].ldc]) and np.isnan(probs[0].c_view(res[0], 0)[5, :]).all()
        assert np.isnan(probs[1].c_view(res[1], 0)[:, 4]).all()
        assert not np.isnan(probs[3].c_view(res[3], 0)).any()
    finally:
        S.set_math_mode(0)


def test_grouped_ozaki_subnormal_rows():
    """Rows of op(A) and columns of op(B) made of subnormals (below 2^-1042, where the row
    maximum comes from the low words, and above it), in instances of every layout: the grouped
    pre-pass finds the exponents of the CPU restatement (bit-exact product)."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    rng = np.random.default_rng(21)
    tiny = 2.0 ** -1074
    probs = []
    for i, (ta, tb) in enumerate([(0, 0), (1, 1), (0, 1), (1, 0)]):
        p = W.make_problem("f64", ta, tb, 50 + 13 * i, 36 + 7 * i, 70 + 45 * i, 1, 1.0, 0.0, seed=800 + i,
                           dist="expspread")
        opa, opb = p.op_a(0), p.op_b(0)
        opa[1, :] = rng.integers(-2 ** 31, 2 ** 31, p.k) * tiny
        opa[2, :] = rng.integers(-2 ** 48, 2 ** 48, p.k) * tiny
        opa[4, :] = -(rng.integers(0, 2 ** 12, p.k) * tiny)
        opb[:, 0] = rng.integers(-2 ** 31, 2 ** 31, p.k) * tiny
        opb[:, 3] = rng.standard_normal(p.k) * 2.0 ** 1000
        probs.append(p)
    S.set_math_mode(1)
    try:
        gd = runner.GroupedDevice(probs)
        gd.reset_c()
        assert gd.call(device_arrays=True) == 0
        for p, C in zip(probs, gd.results()):
            _check(p, C, 1)
    finally:
        S.set_math_mode(0)


@pytest.mark.parametrize("mode", [0, 3])
def test_grouped_transposed_orientation(mode):
    """Ozaki instances whose transposed product fills the 128-row tiles better (m small, n large)
    are computed as C^T = op(B)^T op(A)^T and written back transposed; the other kinds keep the
    direct orientation. Every kind, every op(A)/op(B) combination, beta != 0 and C with a padded
    leading dimension."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    S.set_math_mode(mode)
    try:
        probs, seed = [], 300
        for row in ("f64", "f32", "i8"):
            al, be = (2, -1) if row == "i8" else (0.75, 0.5)
            for ta in (0, 1):
                for tb in (0, 1):
                    for m, n, k in ((20, 300, 70), (300, 20, 70), (5, 129, 33), (129, 5, 33), (1, 200, 9)):
                        seed += 1
                        probs.append(W.make_problem(row, ta, tb, m, n, k, 1, al, be, ldc=m + 3, seed=seed,
                                                    dist="expspread" if row == "f64" else "uniform"))
        gd = runner.GroupedDevice(probs)
        for rep in range(3):
            gd.reset_c()
            assert gd.call(device_arrays=True) == 0
            for p, C in zip(probs, gd.results()):
                _check(p, C, mode)
                # the padding rows of C (m <= i < ldc) are untouched
                np.testing.assert_array_equal(C.reshape(p.n, p.ldc)[:, p.m:], p.C.reshape(p.n, p.ldc)[:, p.m:])
    finally:
        S.set_math_mode(0)


@pytest.mark.parametrize("gcfg", [0, 1, 2])
def test_grouped_ozaki_tile_shapes(gcfg):
    """Ozaki instances on 128 x 64 tiles (0), on the shape their size bucket selects -- here long-K
    instances on 128 x 64 and short ones on 128 x 32 tiles, in one call (1), and all on 128 x 32
    tiles in the static order (2): bit-exact against the restatement in every case."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    rng = np.random.default_rng(gcfg)
    probs = []
    for i in range(24):
        m, n = (int(x) for x in rng.integers(20, 300, 2))
        k = int(rng.choice([40, 200, 700, 1500]))
        probs.append(W.make_problem("f64", i % 2, (i // 2) % 2, m, n, k, 1, 1.0, 0.5 if i % 3 == 0 else 0.0,
                                    seed=900 + i, dist="expspread", name=f"o{i}"))
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_kernel_config("grouped", gcfg)
    try:
        gd = runner.GroupedDevice(probs)
        for _ in range(2):
            gd.reset_c()
            assert gd.call(device_arrays=True) == 0
            for p, C in zip(probs, gd.results()):
                np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, 7)[1].view(np.uint64), err_msg=p.name)
    finally:
        S.set_kernel_config("grouped", -1)
        S.set_math_mode(0)


@pytest.mark.parametrize("row,forced", [("f64", -1), ("f64", 2), ("f32", -1), ("f32", 1)])
def test_grouped_plain_tensor_and_ffma_tiles(row, forced):
    """Plain instances of a grouped call on the batched call's kernels: fp64 on the FP64 tensor
    cores (DMMA), fp32 on the cp.async FFMA tiles -- one launch per op(A) / op(B) layout present,
    tiles longest k first; forcing the DMMA configuration 2 (fp64) or the SIMT configuration 1
    (fp32) sends them to the register-tiled SIMT kernel instead. Every layout, ragged and tiny
    shapes, beta = 0 and beta != 0, each within 4 k u of the FP64-exact oracle, fresh plan and
    graph replay."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    shapes = [(1, 1, 1), (70, 33, 5), (64, 64, 64), (130, 200, 97), (256, 96, 300), (17, 150, 16)]
    probs = [W.make_problem(row, ta, tb, m, n, k, 1, 0.75, 0.0 if i % 2 else -0.5, seed=400 + 10 * i + 2 * ta + tb)
             for i, (m, n, k) in enumerate(shapes) for ta in (0, 1) for tb in (0, 1)]
    key = "dmma" if row == "f64" else "simt"
    u = 2.0 ** -53 if row == "f64" else 2.0 ** -24
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    S.set_kernel_config(key, forced)
    try:
        gd = runner.GroupedDevice(probs)
        for rep in range(3):            # plan (profiled), capture, replay
            gd.reset_c()
            S.set_profiling(rep == 0)
            assert gd.call(device_arrays=True) == 0
            if rep == 0:
                prof = S.get_profile()
                S.set_profiling(False)
                want = "simt_grouped" if forced >= 0 else ("dmma_grouped" if row == "f64" else "sgemm_grouped")
                assert want in prof and set(prof) <= {want}, prof
                # one launch per layout, or one SIMT launch for all
                assert S.last_run_info()["kernel_launches"] == (1 if forced >= 0 else 4)
            for p, C in zip(probs, gd.results()):
                assert O.normalized_error(p, C) <= 4 * max(p.k, 1) * u, p.name
    finally:
        S.set_profiling(False)
        S.set_kernel_config(key, -1)
        S.set_math_mode(0)
