"""ssblasex_b200 -- ssblasGemmBatchedEx for NVIDIA B200 (sm_100a).

Python mirror of the library's C ABI (include/ssblasBatch.h). The names, argument order, enum
values and status codes are those of the reference library (hirokitokura/ssblasEx,
include/ssblasBatch.h:15-57, include/ssblasBatch_type.h); every call goes through
libssblas_b200.so, whose kernels are hand-written CUDA for sm_100a. There is no CPU fallback:
importing this package fails if the shared library is missing.
"""
from __future__ import annotations

import ctypes as ct
import os
import pathlib

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "libssblas_b200.so"

# ---- enums (values of the reference's ssblasBatch_type.h) ----------------------------------
SSBLAS_STATUS_SUCCESS = 0
SSBLAS_STATUS_ALLOC_FAILED = 1
SSBLAS_STATUS_INVALID_VALUE = 2
SSBLAS_STATUS_INTERNAL_ERROR = 3
SSBLAS_STATUS_NOTIMPLEMENTED_ERROR = 4
SSBLAS_STATUS_NOT_COMPUTED_ERROR = 5
STATUS_NAMES = {0: "SSBLAS_STATUS_SUCCESS", 1: "SSBLAS_STATUS_ALLOC_FAILED",
                2: "SSBLAS_STATUS_INVALID_VALUE", 3: "SSBLAS_STATUS_INTERNAL_ERROR",
                4: "SSBLAS_STATUS_NOTIMPLEMENTED_ERROR", 5: "SSBLAS_STATUS_NOT_COMPUTED_ERROR"}

SSBLAS_OP_N, SSBLAS_OP_T, SSBLAS_OP_C = 0, 1, 2
SSBLAS_R_8I, SSBLAS_R_8U, SSBLAS_R_16F, SSBLAS_R_32I, SSBLAS_R_32F, SSBLAS_R_64F = range(6)
SSBLAS_COMPUTE_DEFAULT_TYPE, SSBLAS_COMPUTE_32I, SSBLAS_COMPUTE_32F = 0, 1, 2
SSBLAS_COMPUTE_DEFAULT = 0

# extensions
SSBLAS_MATH_PLAIN, SSBLAS_MATH_FP64_OZAKI, SSBLAS_MATH_FP32_BF16X3 = 0, 1, 2
PATH_NAMES = {0: "none", 1: "simt", 2: "i8_tcgen05", 3: "ozaki_tcgen05", 4: "bf16x3_tcgen05", 5: "grouped",
              6: "dmma", 11: "f16_tcgen05"}
# type and semantics extensions (ssblasSetExtensions)
SSBLAS_EXT_NONE, SSBLAS_EXT_R16F, SSBLAS_EXT_R8U, SSBLAS_EXT_OP_C, SSBLAS_EXT_K0_BETA, SSBLAS_EXT_COMPUTE_TYPE = (
    0, 1, 2, 4, 8, 16)

EXPORTED_SYMBOLS = (
    "ssblasGemmBatchedEx", "ssblasGemmBatchedEx_64", "ssblasGemmGroupedBatchedEx",
    "ssblasSetStream", "ssblasGetStream", "ssblasSetSyncMode", "ssblasSetMathMode",
    "ssblasGetMathMode", "ssblasSetOzakiSlices", "ssblasGetLastRunInfo", "ssblasReleaseWorkspace",
    "ssblasSetProfiling", "ssblasGetProfile", "ssblasGemmBatchedExNoAlloc",
    "ssblasSetKernelConfig", "ssblasReloadTuning", "ssblasSetOzakiTolerance", "ssblasGetOzakiSlices",
    "ssblasSetFaultInjection", "ssblasSetExtensions", "ssblasGetExtensions",
)


class KernelProfile(ct.Structure):
    _fields_ = [("name", ct.c_char * 48), ("launches", ct.c_int), ("total_ms", ct.c_double)]


class RunInfo(ct.Structure):
    _fields_ = [("path", ct.c_int), ("slices", ct.c_int), ("kernel_launches", ct.c_int),
                ("device_error", ct.c_int), ("split_k", ct.c_int)]


_lib = None


def lib() -> ct.CDLL:
    """The loaded libssblas_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python -m ssblasex_b200.build` first "
                              "(there is no CPU fallback)")
        L = ct.CDLL(str(LIB_PATH))
        vp, l, i = ct.c_void_p, ct.c_long, ct.c_int
        gemm_args = [i, i, l, l, l, vp, vp, i, l, vp, i, l, vp, vp, i, l, l, i, i]
        for name in ("ssblasGemmBatchedEx", "ssblasGemmBatchedEx_64", "ssblasGemmBatchedExNoAlloc"):
            f = getattr(L, name)
            f.argtypes = gemm_args
            f.restype = i
        L.ssblasGemmGroupedBatchedEx.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                                 vp, vp, vp, vp, l, vp, i, i]
        L.ssblasGemmGroupedBatchedEx.restype = i
        L.ssblasSetStream.argtypes = [vp]
        L.ssblasGetStream.argtypes = [ct.POINTER(vp)]
        L.ssblasSetSyncMode.argtypes = [i]
        L.ssblasSetMathMode.argtypes = [i]
        L.ssblasGetMathMode.argtypes = [ct.POINTER(i)]
        L.ssblasSetOzakiSlices.argtypes = [i]
        L.ssblasSetOzakiTolerance.argtypes = [ct.c_double]
        L.ssblasGetOzakiSlices.argtypes = [ct.POINTER(i)]
        L.ssblasSetFaultInjection.argtypes = [i]
        L.ssblasSetExtensions.argtypes = [i]
        L.ssblasGetExtensions.argtypes = [ct.POINTER(i)]
        L.ssblasGetLastRunInfo.argtypes = [ct.POINTER(RunInfo)]
        L.ssblasReleaseWorkspace.argtypes = []
        L.ssblasSetProfiling.argtypes = [i]
        L.ssblasGetProfile.argtypes = [ct.POINTER(KernelProfile), i, ct.POINTER(i)]
        L.ssblasSetKernelConfig.argtypes = [i, i]
        L.ssblasReloadTuning.argtypes = []
        for name in EXPORTED_SYMBOLS[3:]:
            getattr(L, name).restype = i
        _lib = L
    return _lib


def ssblasGemmBatchedEx(transa, transb, m, n, k, alpha, A, Atype, lda, B, Btype, ldb, beta, C,
                        Ctype, ldc, batchCount, computeType=SSBLAS_COMPUTE_DEFAULT_TYPE,
                        algo=SSBLAS_COMPUTE_DEFAULT) -> int:
    """Direct call of the C entry point. alpha/beta: addresses of host scalars of the row's scale
    type; A/B/C: addresses of pointer arrays (host or device memory). Returns the status code."""
    return lib().ssblasGemmBatchedEx(transa, transb, m, n, k, alpha, A, Atype, lda, B, Btype, ldb,
                                     beta, C, Ctype, ldc, batchCount, computeType, algo)


def ssblasGemmBatchedEx_64(*args) -> int:
    return lib().ssblasGemmBatchedEx_64(*args)


def ssblasGemmGroupedBatchedEx(*args) -> int:
    return lib().ssblasGemmGroupedBatchedEx(*args)


def set_stream(stream_handle: int | None) -> int:
    return lib().ssblasSetStream(stream_handle or None)


def set_sync_mode(synchronous: bool) -> int:
    return lib().ssblasSetSyncMode(1 if synchronous else 0)


def set_math_mode(mode: int) -> int:
    return lib().ssblasSetMathMode(mode)


def get_math_mode() -> int:
    v = ct.c_int()
    lib().ssblasGetMathMode(ct.byref(v))
    return v.value


def set_ozaki_slices(slices: int) -> int:
    return lib().ssblasSetOzakiSlices(slices)


def set_ozaki_tolerance(tolerance: float) -> int:
    """Per-term error target of the automatic Ozaki slice count (0 = the default 2^-51)."""
    return lib().ssblasSetOzakiTolerance(float(tolerance))


def get_ozaki_slices() -> int:
    """Slice count the next fp64 Ozaki call will use."""
    v = ct.c_int()
    lib().ssblasGetOzakiSlices(ct.byref(v))
    return v.value


def ozaki_term_bound(slices: int) -> float:
    """Per-term error bound (S + 1) * 2^(2 - 8S) of the Ozaki emulation, in units of
    |alpha| * 2^(e_i + f_j) (the row and column power-of-two scales)."""
    import math
    return (slices + 1) * math.ldexp(1.0, 2 - 8 * slices)


SSBLAS_FAULT_NONE, SSBLAS_FAULT_SKIP_COPY, SSBLAS_FAULT_ALLOC = 0, 1, 2


def set_extensions(flags: int) -> int:
    """Enables type / semantics extensions (SSBLAS_EXT_* flags OR-ed; 0 = the reference's behaviour)."""
    return lib().ssblasSetExtensions(flags)


def get_extensions() -> int:
    v = ct.c_int()
    lib().ssblasGetExtensions(ct.byref(v))
    return v.value


def set_fault_injection(fault: int) -> int:
    """Arms a one-shot test fault (SSBLAS_FAULT_SKIP_COPY / SSBLAS_FAULT_ALLOC); 0 disarms."""
    return lib().ssblasSetFaultInjection(fault)


def last_run_info() -> dict:
    info = RunInfo()
    lib().ssblasGetLastRunInfo(ct.byref(info))
    return {"path": PATH_NAMES.get(info.path, str(info.path)), "slices": info.slices,
            "kernel_launches": info.kernel_launches, "device_error": info.device_error,
            "split_k": info.split_k}


def release_workspace() -> int:
    return lib().ssblasReleaseWorkspace()


def set_profiling(enable: bool) -> int:
    return lib().ssblasSetProfiling(1 if enable else 0)


def get_profile() -> dict:
    """{kernel name: (launches, total ms)} of the library's launches since set_profiling(True)."""
    n = ct.c_int()
    lib().ssblasGetProfile(None, 0, ct.byref(n))
    arr = (KernelProfile * max(n.value, 1))()
    lib().ssblasGetProfile(arr, n.value, ct.byref(n))
    return {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms) for i in range(n.value)}


PATH_IDS = {"simt": 1, "i8_tcgen05": 2, "ozaki_tcgen05": 3, "bf16x3_tcgen05": 4, "grouped": 5, "dmma": 6,
            "ozaki_slicer": 7, "splitk_i8": 8, "splitk_ozaki": 9, "ozaki_pipeline": 10, "f16_tcgen05": 11,
            "grouped_ozaki_tile": 12}


def set_kernel_config(path: str, config: int) -> int:
    """Force configuration `config` of a kernel family ("i8_tcgen05", "ozaki_tcgen05", ...);
    -1 returns to the tuned / default choice."""
    return lib().ssblasSetKernelConfig(PATH_IDS[path], config)


def reload_tuning() -> int:
    return lib().ssblasReloadTuning()
