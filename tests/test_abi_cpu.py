"""The C-ABI library loads on a CPU-only host, exports every entry point of include/*.h, and
applies the reference's argument conventions before touching a GPU."""
import ctypes as ct
import os
import pathlib
import re
import subprocess
import sys

import numpy as np
import pytest

from golden_cases import load_status_cases

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*ssblasStatus_t\s+(ssblas\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_entry_point():
    import ssblasex_b200 as S
    names = declared_functions()
    assert {"ssblasGemmBatchedEx", "ssblasGemmBatchedEx_64", "ssblasGemmGroupedBatchedEx"} <= names
    L = S.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(S.EXPORTED_SYMBOLS) >= names
    out = subprocess.run(["nm", "-D", "--defined-only", str(S.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert names <= exported
    assert all(e.startswith("ssblas") for e in exported)   # nothing else leaks out


def test_enums_match_reference_values():
    hdr = (ROOT / "include" / "ssblasBatch_type.h").read_text()
    for name in ["SSBLAS_STATUS_SUCCESS = 0", "SSBLAS_OP_N = 0", "SSBLAS_OP_T = 1", "SSBLAS_OP_C = 2"]:
        assert name in hdr
    order = ["SSBLAS_R_8I", "SSBLAS_R_8U", "SSBLAS_R_16F", "SSBLAS_R_32I", "SSBLAS_R_32F", "SSBLAS_R_64F"]
    pos = [hdr.index(o + ",") if o + "," in hdr else hdr.index(o + "\n") for o in order]
    assert pos == sorted(pos)


@pytest.mark.parametrize("use_64", [False, True])
def test_status_codes_before_any_device_work(golden, use_64):
    """Degenerate calls return the reference's status without a GPU (they never reach CUDA)."""
    from ssblasex_b200 import runner
    for p, over, ref_C, ref_st in load_status_cases(golden):
        st, C = runner.call(p, mode="host_matrices", use_64=use_64, **over)
        assert st == ref_st, (p.name, st, ref_st)
        np.testing.assert_array_equal(C, ref_C, err_msg=p.name)


def test_invalid_arguments_the_reference_does_not_check():
    from ssblasex_b200 import runner, workloads as W
    import ssblasex_b200 as S
    p = W.make_problem("f32", 0, 0, 9, 8, 7, 2, 1.0, 0.0, seed=1)
    assert runner.call(p, mode="host_matrices", lda=8)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    assert runner.call(p, mode="host_matrices", ldc=3)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    # op C on the int8 row: the reference reads through NULL; here it is rejected
    p8 = W.make_problem("i8", 0, 0, 9, 8, 7, 2, 1, 0, seed=1)
    assert runner.call(p8, mode="host_matrices", transa=2)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    al = np.array([1.0], np.float32)
    arr = (ct.c_void_p * 2)()
    st = S.lib().ssblasGemmBatchedEx(0, 0, 4, 4, 4, None, arr, 4, 4, arr, 4, 4, al.ctypes.data, arr, 4, 4, 2, 0, 0)
    assert st == S.SSBLAS_STATUS_INVALID_VALUE


def test_math_mode_and_settings():
    import ssblasex_b200 as S
    assert S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI | S.SSBLAS_MATH_FP32_BF16X3) == 0
    assert S.get_math_mode() == 3
    assert S.set_math_mode(8) == S.SSBLAS_STATUS_INVALID_VALUE
    assert S.set_math_mode(0) == 0
    assert S.set_ozaki_slices(2) == S.SSBLAS_STATUS_INVALID_VALUE
    assert S.set_ozaki_slices(0) == 0


def test_debug_dump_is_the_reference_text():
    spec_path = ROOT / "tests" / "golden" / "make_golden.py"
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", spec_path)
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    import ssblasex_b200 as S
    got = mg.dump_text(str(S.LIB_PATH))
    want = (ROOT / "tests" / "golden" / "debug_dump.txt").read_text()
    assert got == want


def test_noalloc_refuses_sizes_whose_scratch_product_overflows():
    """The allocation-free entry point sizes its scratch with overflow-checked products and refuses
    a problem before any CUDA call: here (no GPU) a refusal that came later would read as
    NOTIMPLEMENTED or INTERNAL_ERROR, not INVALID_VALUE."""
    import ssblasex_b200 as S
    al = np.array([1.0], np.float64)
    arr = (ct.c_void_p * 1)()
    f = S.lib().ssblasGemmBatchedExNoAlloc
    R = S.SSBLAS_R_64F
    cases = [
        # 7 * 2^26 * 16384 * 2^26 bytes wraps a 64-bit size; every factor alone fits the array
        (1 << 26, 1, 16384, 1 << 26),
        # a dimension larger than the whole array
        (1 << 40, 1, 16, 1),
        (1, 1 << 40, 16, 1),
        (1, 1, 16, 1 << 40),
        # fits no wrap, still too big: 7 * (4096 + 4096) * 1024 * 2 bytes = 117 MB
        (4096, 4096, 1024, 2),
    ]
    for m, n, k, batch in cases:
        st = f(0, 0, m, n, k, al.ctypes.data, arr, R, m, arr, R, k, al.ctypes.data, arr, R, m, batch, 0, 0)
        assert st == S.SSBLAS_STATUS_INVALID_VALUE, (m, n, k, batch, st)
    # k beyond the exact int32 range of one piece
    st = f(0, 0, 8, 8, 16385, al.ctypes.data, arr, R, 8, arr, R, 16385, al.ctypes.data, arr, R, 8, 1, 0, 0)
    assert st == S.SSBLAS_STATUS_INVALID_VALUE


def test_per_device_tables(tmp_path):
    """The per-device tables (csrc/per_device.h) keep one entry per device ordinal: a kernel
    attribute set on device 0 is set again on device 1, a failed set-up is retried, and ordinals
    outside the table are refused without touching it."""
    src = tmp_path / "t.cpp"
    src.write_text(r'''
#include "per_device.h"
#include <cstdio>
using namespace ssb;
int main() {
  bool done[kMaxDevices] = {};
  int calls = 0, fail = 1;
  auto init = [&] { ++calls; return fail ? 7 : 0; };
  if (once_per_device(done, 0, init, -9) != 7 || calls != 1 || done[0]) return 1;     // failure not cached
  fail = 0;
  if (once_per_device(done, 0, init, -9) != 0 || calls != 2 || !done[0]) return 2;
  if (once_per_device(done, 0, init, -9) != 0 || calls != 2) return 3;                 // cached
  if (once_per_device(done, 1, init, -9) != 0 || calls != 3 || !done[1]) return 4;     // per device
  if (once_per_device(done, -1, init, -9) != -9 || calls != 3) return 5;               // refused
  if (once_per_device(done, kMaxDevices, init, -9) != -9 || calls != 3) return 6;
  for (int d = 2; d < kMaxDevices; ++d) if (done[d]) return 7;
  std::puts("ok");
  return 0;
}
''')
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "ssblasex_b200" / "csrc"), str(src), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout)


def test_staged_copy_pieces(tmp_path):
    """The byte arithmetic of the staged host copies (csrc/hostcopy_plan.h): for random instance
    sizes, pitches, column layouts, staging windows and part counts, every byte of every instance
    lands exactly once at its place -- instance b at b * pitch on the device side; for the copy
    back only the first row_bytes of each column -- and no byte between instances (or in the
    caller's column padding) is written."""
    src = tmp_path / "t.cpp"
    src.write_text(r"""
#include "hostcopy_plan.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>
using namespace ssb;
int main() {
  std::mt19937_64 rng(7);
  auto U = [&](long lo, long hi) { return lo + (long)(rng() % (unsigned long)(hi - lo + 1)); };
  for (int trial = 0; trial < 400; ++trial) {
    // gather: instance b (bytes) to b * pitch
    {
      const long batch = U(1, 40);
      const size_t bytes = U(1, 5000), pitch = bytes + U(0, 300);
      const size_t total = pitch * (batch - 1) + bytes;
      std::vector<std::vector<unsigned char>> inst(batch, std::vector<unsigned char>(bytes));
      for (auto& v : inst) for (auto& x : v) x = (unsigned char)rng();
      std::vector<unsigned char> dev(total, 0xEE);
      std::vector<int> hits(total, 0);
      const size_t W = U(1, 20000);
      const int parts = (int)U(1, 17);
      for (size_t c0 = 0; c0 < total; c0 += W) {
        const size_t c1 = c0 + W < total ? c0 + W : total;
        for (int part = 0; part < parts; ++part) {
          size_t p0, p1;
          window_part(c0, c1, part, parts, &p0, &p1);
          gather_pieces(p0, p1, pitch, batch, bytes, [&](long b, size_t in_inst, size_t at, size_t len) {
            if (at < p0 || at + len > p1 || in_inst + len > bytes) { std::printf("range\n"); std::exit(1); }
            std::memcpy(&dev[at], &inst[b][in_inst], len);
            for (size_t i = 0; i < len; ++i) ++hits[at + i];
          });
        }
      }
      for (long b = 0; b < batch; ++b)
        for (size_t x = 0; x < pitch && b * pitch + x < total; ++x) {
          const size_t at = b * pitch + x;
          if (x < bytes ? (hits[at] != 1 || dev[at] != inst[b][x]) : (hits[at] != 0 || dev[at] != 0xEE)) {
            std::printf("gather trial %d b %ld x %zu\n", trial, b, x);
            return 2;
          }
        }
    }
    // scatter: the first row_bytes of each of cols columns (ld_bytes apart) of instance b
    {
      const long batch = U(1, 30), cols = U(1, 40);
      const size_t row_bytes = U(1, 400), ld_bytes = row_bytes + U(0, 64);
      const size_t span = ld_bytes * (cols - 1) + row_bytes, pitch = span + U(0, 200);
      const size_t total = pitch * (batch - 1) + span;
      std::vector<unsigned char> dev(total);
      for (auto& x : dev) x = (unsigned char)rng();
      std::vector<std::vector<unsigned char>> host(batch, std::vector<unsigned char>(ld_bytes * cols, 0xEE));
      std::vector<std::vector<int>> hits(batch, std::vector<int>(ld_bytes * cols, 0));
      const size_t W = U(1, 9000);
      const int parts = (int)U(1, 17);
      for (size_t c0 = 0; c0 < total; c0 += W) {
        const size_t c1 = c0 + W < total ? c0 + W : total;
        for (int part = 0; part < parts; ++part) {
          size_t p0, p1;
          window_part(c0, c1, part, parts, &p0, &p1);
          scatter_pieces(p0, p1, pitch, batch, ld_bytes, row_bytes, cols,
                         [&](long b, size_t in_inst, size_t at, size_t len) {
                           if (at < p0 || at + len > p1 || in_inst + len > ld_bytes * cols) {
                             std::printf("range\n");
                             std::exit(3);
                           }
                           std::memcpy(&host[b][in_inst], &dev[at], len);
                           for (size_t i = 0; i < len; ++i) ++hits[b][in_inst + i];
                         });
        }
      }
      for (long b = 0; b < batch; ++b)
        for (long j = 0; j < cols; ++j)
          for (size_t r = 0; r < ld_bytes; ++r) {
            const size_t x = j * ld_bytes + r;
            const bool in = r < row_bytes;
            if (in ? (hits[b][x] != 1 || host[b][x] != dev[b * pitch + x]) : (hits[b][x] != 0 || host[b][x] != 0xEE)) {
              std::printf("scatter trial %d b %ld col %ld r %zu\n", trial, b, j, r);
              return 4;
            }
          }
    }
  }
  std::puts("ok");
  return 0;
}
""")
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "ssblasex_b200" / "csrc"), str(src), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout)


def test_fault_injection_setter():
    import ssblasex_b200 as S
    for f in (S.SSBLAS_FAULT_SKIP_COPY, S.SSBLAS_FAULT_ALLOC, S.SSBLAS_FAULT_NONE):
        assert S.set_fault_injection(f) == 0
    for bad in (-1, 3, 99):
        assert S.set_fault_injection(bad) == S.SSBLAS_STATUS_INVALID_VALUE


def test_extension_flags_and_their_status_rules():
    """Extensions are off by default; each changes a status rule in the documented way, checked
    before any device work (no GPU here)."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    try:
        assert S.get_extensions() == 0
        assert S.set_extensions(32) == S.SSBLAS_STATUS_INVALID_VALUE
        p = W.make_problem("f32", 0, 0, 9, 8, 7, 2, 1.0, 0.0, seed=1)
        # computeType is ignored without the extension (the reference's behaviour) ...
        assert S.set_extensions(S.SSBLAS_EXT_COMPUTE_TYPE) == 0
        al = np.array([1.0], np.float32)
        arr = (ct.c_void_p * 2)()
        f = S.lib().ssblasGemmBatchedEx
        # ... and checked against the row with it: 32I on the fp32 row is refused
        assert f(0, 0, 4, 4, 4, al.ctypes.data, arr, 4, 4, arr, 4, 4, al.ctypes.data, arr, 4, 4, 2,
                 S.SSBLAS_COMPUTE_32I, 0) == S.SSBLAS_STATUS_INVALID_VALUE
        assert f(0, 0, 4, 4, 4, al.ctypes.data, arr, 4, 4, arr, 4, 4, al.ctypes.data, arr, 4, 4, 2,
                 7, 0) == S.SSBLAS_STATUS_INVALID_VALUE
        # k < 0 is refused under the k = 0 extension (the reference treats it as k = 0)
        S.set_extensions(S.SSBLAS_EXT_K0_BETA)
        assert runner.call(p, mode="host_matrices", k=-1)[0] == S.SSBLAS_STATUS_INVALID_VALUE
        S.set_extensions(0)
        assert runner.call(p, mode="host_matrices", k=-1)[0] == S.SSBLAS_STATUS_SUCCESS
        # fp16 and unsigned int8 rows exist only with their flags
        for row in ("f16", "f16c32", "u8", "u8s8"):
            q = W.make_problem(row, 0, 0, 9, 8, 7, 2, 1, 0, seed=1)
            assert runner.call(q, mode="host_matrices")[0] == S.SSBLAS_STATUS_INVALID_VALUE
        # op C without the extension
        assert runner.call(p, mode="host_matrices", transb=2)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    finally:
        S.set_extensions(0)


def _run_with_env(code, **env):
    import os
    import subprocess
    import sys
    e = dict(os.environ)
    e.update(env)
    e["PYTHONPATH"] = str(ROOT) + os.pathsep + e.get("PYTHONPATH", "")
    r = subprocess.run([sys.executable, "-c", code], env=e, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return r


def test_environment_knobs():
    """SSBLAS_OZAKI_SLICES / SSBLAS_OZAKI_TOLERANCE set the slice choice of a process (as the
    setters do; out-of-range values are ignored), and SSBLAS_LOG prints one line per call on
    stderr with the status -- here of calls refused before any device work."""
    code = "import ssblasex_b200 as S; print(S.get_ozaki_slices())"
    assert _run_with_env(code).stdout.strip() == "7"
    assert _run_with_env(code, SSBLAS_OZAKI_SLICES="5").stdout.strip() == "5"
    assert _run_with_env(code, SSBLAS_OZAKI_SLICES="12").stdout.strip() == "7"
    assert _run_with_env(code, SSBLAS_OZAKI_TOLERANCE="1e-6").stdout.strip() == "3"
    assert _run_with_env(code, SSBLAS_OZAKI_TOLERANCE="0x1p-56").stdout.strip() == "8"
    call = ("import ssblasex_b200 as S\n"
            "st = S.lib().ssblasGemmBatchedEx(0, 0, 0, 4, 4, None, None, S.SSBLAS_R_32F, 4, None, S.SSBLAS_R_32F, 4,"
            " None, None, S.SSBLAS_R_32F, 4, 1, 0, 0)\n"
            "print(st)\n")
    r = _run_with_env(call, SSBLAS_LOG="1")
    assert r.stdout.strip() == str(S_INTERNAL_ERROR)
    assert "ssblas: ssblasGemmBatchedEx m=0 n=4 k=4 batch=1 status=3" in r.stderr
    assert "ssblas:" not in _run_with_env(call).stderr


S_INTERNAL_ERROR = 3


def test_reference_arm_line():
    """`bench.py --impl reference` (the reference's own CPU implementation, or the C restatement
    where the reference was not built) prints one JSON line with the contract's keys: the
    metric and unit of the GPU arm, an `e2e` with no host<->device bytes, and a `cpu_baseline`
    naming the kind, the threads and the sample."""
    import json
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--workload", "fp32_batch64_128"], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "TFLOP/s" and line["value"] > 0
    assert line["higher_is_better"] is True and line["n_gpus"] == 1 and line["steps"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and "instances" in cb["sample"]
    assert line["config"]["workload"] == "fp32_batch64_128"


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 runs the reference arm; the other ranks exit 0 without work."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0", "--workload", "fp32_batch64_128"], capture_output=True, text=True,
                       timeout=600, cwd=str(ROOT), env=env)
    assert r.returncode == 0 and r.stdout.strip() == "", (r.returncode, r.stdout[-500:], r.stderr[-500:])
