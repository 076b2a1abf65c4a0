"""Host logic of the serving engine on the CPU: the range allocator behind its HARQ,
payload and staging arenas (syn::RangeAlloc), exercised by tests/range_alloc_check.cpp
linked against the built library."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "syndrome_b200", "csrc")
LIBDIR = os.path.join(ROOT, "syndrome_b200")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


def test_range_alloc_randomized():
    if not os.path.exists(os.path.join(LIBDIR, "libsyndrome_b200.so")):
        pytest.skip("library not built")
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "range_alloc_check")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I" + CSRC, "-I" + CUDA_INC,
                           os.path.join(HERE, "range_alloc_check.cpp"), "-L" + LIBDIR, "-lsyndrome_b200",
                           "-Wl,-rpath," + LIBDIR, "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
