"""Builds libsyndrome_b200.so in place (syndrome_b200/libsyndrome_b200.so).

Device code is compiled for sm_100a only, without fast-math, with FMA contraction
disabled (-fmad=false) and denormals preserved, so the f32 decoder performs the
same IEEE operations as the reference.  Host code gets -ffp-contract=off for the
same reason (channel simulation).

    python -m syndrome_b200.build          # incremental
    python -m syndrome_b200.build --force  # full rebuild
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsyndrome_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math,-pthread",
          "-I" + CSRC, "-I" + INCLUDE]
DEVICE = ["-fmad=false", "-ftz=false", "-prec-div=true", "-prec-sqrt=true", "-Xptxas", "-O3"]

SOURCES = ["graph.cpp", "encoder.cpp", "channel.cpp", "tb.cpp", "frames.cpp", "serve.cpp", "serve_cont.cpp", "serve_load.cpp", "mixed.cpp", "wifi_mixed.cpp", "capi.cpp", "ldpc_kernels.cu", "nr_kernels.cu", "nr_pair_kernels.cu", "serve_kernels.cu", "encoder_kernels.cu", "nr_f32_kernels.cu"]
HEADERS = ["smem_limit.h", "nr_graph.cuh", "nr_pair.cuh", "graph.h", "tb.h", "frames.h", "serve.h", "serve_kernels.h", "serve_device.cuh", "encoder.h", "channel.h", "decoder.h", "graph_tables.h", "base_graph_tables.inc",
           "nr_kernels.h", "nr_layered_tables.h", "mixed.h", "wifi_mixed.h"]


def _newest_header():
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "syndrome_ldpc.h")]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _compile(src, force, extra):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if not force and os.path.exists(obj):
        if os.path.getmtime(obj) >= max(os.path.getmtime(path), _newest_header()):
            return obj, False
    cmd = [NVCC] + ARCH + COMMON + extra + ["-c", path, "-o", obj]
    if src.endswith(".cu"):
        cmd[1:1] = DEVICE
    subprocess.check_call(cmd)
    return obj, True


def build(force=False, verbose=True, extra=None):
    os.makedirs(BUILD, exist_ok=True)
    extra = list(extra or [])
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, extra), SOURCES))
    objs = [o for o, _ in results]
    changed = any(c for _, c in results)
    if changed or force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        subprocess.check_call([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread"])
        os.replace(tmp, LIB)
        if verbose:
            print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
