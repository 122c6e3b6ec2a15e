"""Calls ssblasGemmBatchedEx on a workloads.Problem through the C ABI.

torch provides device memory and streams here (plumbing only); all arithmetic runs in
libssblas_b200.so. Three pointer conventions are exercised, matching the C ABI:

  "device_array"   device array of device pointers (cuBLAS batched convention)
  "host_array"     host array of device pointers
  "host_matrices"  host array of host pointers -- the reference's own convention; the library
                   stages the matrices through device memory
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import lib
from .workloads import Problem

_TORCH_DTYPES = None


def _torch():
    import torch
    return torch


def torch_dtype(np_dtype):
    torch = _torch()
    return {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
            np.dtype(np.int8): torch.int8, np.dtype(np.int32): torch.int32}[np.dtype(np_dtype)]


class DeviceProblem:
    """Device copies of a Problem's operands (one contiguous tensor per operand)."""

    def __init__(self, p: Problem, device="cuda", C=None):
        torch = _torch()
        self.p = p
        self.A = torch.from_numpy(p.A).to(device)
        self.B = torch.from_numpy(p.B).to(device)
        self.C = torch.from_numpy(p.C if C is None else C).to(device)
        self.device = device
        self._ptr_dev = None

    def reset_c(self, C=None):
        torch = _torch()
        self.C.copy_(torch.from_numpy(self.p.C if C is None else C))

    def ptrs(self, t):
        base = t.data_ptr()
        stride = t.stride(0) * t.element_size()
        return [base + b * stride for b in range(self.p.batch)]

    def host_arrays(self):
        b = self.p.batch
        arrs = [(ct.c_void_p * b)(*self.ptrs(t)) for t in (self.A, self.B, self.C)]
        return arrs

    def device_arrays(self):
        torch = _torch()
        if self._ptr_dev is None:
            self._ptr_dev = [torch.tensor(self.ptrs(t), dtype=torch.int64, device=self.device)
                             for t in (self.A, self.B, self.C)]
        return self._ptr_dev


def _scalars(p: Problem):
    al = np.array([p.alpha], dtype=p.scale_dtype)
    be = np.array([p.beta], dtype=p.scale_dtype)
    return al, be


def call(p: Problem, mode: str = "device_array", dp: DeviceProblem | None = None,
         host_C: np.ndarray | None = None, use_64: bool = False, **over):
    """Runs one call. Returns (status, C as numpy). For "host_matrices" the numpy arrays of p
    (and host_C, default a copy of p.C) are passed directly."""
    al, be = _scalars(p)
    ta, tb, tc = over.pop("types", p.types)
    args = dict(transa=p.transa, transb=p.transb, m=p.m, n=p.n, k=p.k, lda=p.lda, ldb=p.ldb,
                ldc=p.ldc, batch=p.batch)
    args.update(over)
    fn = lib().ssblasGemmBatchedEx_64 if use_64 else lib().ssblasGemmBatchedEx
    if mode == "host_matrices":
        C = p.C.copy() if host_C is None else host_C
        nb = max(p.batch, 1)
        mk = lambda arr: (ct.c_void_p * nb)(*[arr.ctypes.data + b * arr.strides[0] for b in range(nb)])
        Ap, Bp, Cp = mk(p.A), mk(p.B), mk(C)
        st = fn(args["transa"], args["transb"], args["m"], args["n"], args["k"], al.ctypes.data, Ap,
                ta, args["lda"], Bp, tb, args["ldb"], be.ctypes.data, Cp, tc, args["ldc"],
                args["batch"], 0, 0)
        return st, C
    dp = dp or DeviceProblem(p)
    if mode == "host_array":
        Ap, Bp, Cp = dp.host_arrays()
        st = fn(args["transa"], args["transb"], args["m"], args["n"], args["k"], al.ctypes.data, Ap,
                ta, args["lda"], Bp, tb, args["ldb"], be.ctypes.data, Cp, tc, args["ldc"],
                args["batch"], 0, 0)
    elif mode == "device_array":
        Ad, Bd, Cd = dp.device_arrays()
        st = fn(args["transa"], args["transb"], args["m"], args["n"], args["k"], al.ctypes.data,
                Ad.data_ptr(), ta, args["lda"], Bd.data_ptr(), tb, args["ldb"], be.ctypes.data,
                Cd.data_ptr(), tc, args["ldc"], args["batch"], 0, 0)
    else:
        raise ValueError(mode)
    return st, dp.C.cpu().numpy()


class GroupedDevice:
    """Device copies of a list of single-instance Problems, packed into one buffer per dtype,
    plus the per-group argument arrays of ssblasGemmGroupedBatchedEx (one group per problem)."""

    def __init__(self, probs, device="cuda"):
        torch = _torch()
        self.probs = probs
        self.device = device
        self.tensors = []
        ptrs = {"A": [], "B": [], "C": []}
        for p in probs:
            a = torch.from_numpy(p.A[0]).to(device)
            b = torch.from_numpy(p.B[0]).to(device)
            c = torch.from_numpy(p.C[0]).to(device)
            self.tensors.append((a, b, c))
            ptrs["A"].append(a.data_ptr()); ptrs["B"].append(b.data_ptr()); ptrs["C"].append(c.data_ptr())
        G = len(probs)
        L = lambda xs: np.array(xs, dtype=np.int64)
        I = lambda xs: np.array(xs, dtype=np.int32)
        self.ta = I([p.transa for p in probs]); self.tb = I([p.transb for p in probs])
        self.m = L([p.m for p in probs]); self.n = L([p.n for p in probs]); self.k = L([p.k for p in probs])
        self.lda = L([p.lda for p in probs]); self.ldb = L([p.ldb for p in probs]); self.ldc = L([p.ldc for p in probs])
        self.at = I([p.types[0] for p in probs]); self.bt = I([p.types[1] for p in probs]); self.ct = I([p.types[2] for p in probs])
        self.gs = L([1] * G)
        self.scal = [(np.array([p.alpha], dtype=p.scale_dtype), np.array([p.beta], dtype=p.scale_dtype)) for p in probs]
        self.alpha = (ct.c_void_p * G)(*[s[0].ctypes.data for s in self.scal])
        self.beta = (ct.c_void_p * G)(*[s[1].ctypes.data for s in self.scal])
        self.host_ptrs = {k: (ct.c_void_p * G)(*v) for k, v in ptrs.items()}
        self.dev_ptrs = {k: torch.tensor(v, dtype=torch.int64, device=device) for k, v in ptrs.items()}

    def reset_c(self):
        torch = _torch()
        for p, (_, _, c) in zip(self.probs, self.tensors):
            c.copy_(torch.from_numpy(p.C[0]))

    def call(self, device_arrays: bool = True) -> int:
        d = (lambda k: self.dev_ptrs[k].data_ptr()) if device_arrays else (lambda k: ct.addressof(self.host_ptrs[k]))
        a = lambda arr: arr.ctypes.data
        return lib().ssblasGemmGroupedBatchedEx(
            a(self.ta), a(self.tb), a(self.m), a(self.n), a(self.k), ct.addressof(self.alpha), d("A"), a(self.at),
            a(self.lda), d("B"), a(self.bt), a(self.ldb), ct.addressof(self.beta), d("C"), a(self.ct), a(self.ldc),
            len(self.probs), a(self.gs), 0, 0)

    def results(self):
        return [c.cpu().numpy()[None, :] for (_, _, c) in self.tensors]
