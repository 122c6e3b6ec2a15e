"""The device copies of host pointer arrays kept across calls (api.cpp, device_pointer_arrays).

Calls with host arrays of device pointers reuse the device arrays of a recent call with the same
pointer values. Six layouts (more than the four kept) are called in rotation, with the pointer
arrays of some calls permuted and the stream switched between calls, without a synchronisation
between them; every result must equal the oracle's."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def S():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    yield S
    S.set_stream(None)
    S.set_sync_mode(True)
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)


def test_rotating_layouts_and_streams(S):
    import torch
    from ssblasex_b200 import runner, workloads as W
    from oracle import oracle as O
    probs = [W.make_problem("i8", 1, 0, 40 + 8 * i, 24 + 4 * i, 64, 3 + i, 1, 0, seed=500 + i) for i in range(6)]
    dps = [runner.DeviceProblem(p) for p in probs]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    S.set_sync_mode(False)
    calls = 0
    for rnd in range(3):
        for i, (p, dp) in enumerate(zip(probs, dps)):
            Ah, Bh, Ch = dp.host_arrays()
            if (rnd + i) % 3 == 2:
                # the same instances in reverse order: another key, the same results
                rev = lambda arr: (ct.c_void_p * p.batch)(*list(arr)[::-1])
                Ah, Bh, Ch = rev(Ah), rev(Bh), rev(Ch)
            stream = streams[(rnd + i) % 2]
            S.set_stream(stream.cuda_stream)
            al, be = np.array([p.alpha], p.scale_dtype), np.array([p.beta], p.scale_dtype)
            ta, tb, tc = p.types
            st = S.lib().ssblasGemmBatchedEx(p.transa, p.transb, p.m, p.n, p.k, al.ctypes.data, Ah, ta, p.lda, Bh,
                                             tb, p.ldb, be.ctypes.data, Ch, tc, p.ldc, p.batch, 0, 0)
            assert st == 0
            calls += 1
    torch.cuda.synchronize()
    for p, dp in zip(probs, dps):
        np.testing.assert_array_equal(dp.C.cpu().numpy().reshape(p.C.shape), O.restated_gemm(p)[1])
    assert calls == 18
