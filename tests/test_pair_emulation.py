"""CPU check of the paired (two codewords per 32-bit word) int8 arithmetic of the 5G NR
kernel against the oracle.

tests/pair_emu.cpp runs the row update of syndrome_b200/csrc/nr_pair.cuh -- the code
the sm_100a kernel inlines -- on the host; every output (iterations used, posterior,
C->V messages) must be bit-identical to the oracle's scalar restatement of
src/qc_ldpc.rs:1486-1758 for both codewords of a pair.  The GPU parity tests check the
kernel itself through the C ABI."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import _oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "syndrome_b200", "csrc")
_EMU = None


def emu():
    global _EMU
    if _EMU is None:
        out_dir = os.path.join(HERE, "_build")
        os.makedirs(out_dir, exist_ok=True)
        so = os.path.join(out_dir, "libpair_emu.so")
        srcs = [os.path.join(HERE, "pair_emu.cpp"), os.path.join(CSRC, "nr_pair.cuh"),
                os.path.join(CSRC, "nr_graph.cuh"), os.path.join(CSRC, "nr_layered_tables.h")]
        if not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(s) for s in srcs):
            subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-I" + CSRC, "-o", so + ".tmp",
                                   srcs[0]])
            os.replace(so + ".tmp", so)
        L = ctypes.CDLL(so)
        L.pair_emu_decode.restype = ctypes.c_int
        L.pair_emu_decode.argtypes = ([ctypes.c_int] * 2 + [ctypes.c_void_p] + [ctypes.c_int] * 4 +
                                      [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 3)
        _EMU = L
    return _EMU


def emu_pair(code, bg, rows, beta_q, iterations, app_clamp=32767, prologue=False, n_filler=0):
    _, cols, shifts = code.layout()
    shifts = np.ascontiguousarray(shifts, dtype=np.int32)
    a = np.ascontiguousarray(rows[0], dtype=np.int8)
    b = np.ascontiguousarray(rows[1], dtype=np.int8)
    app = np.zeros((2, code.n), np.int16)
    er = np.zeros((2, code.edges * code.z), np.int8)
    it = np.zeros(2, np.int32)
    rc = emu().pair_emu_decode(bg, code.z, shifts.ctypes.data, beta_q, app_clamp, int(prologue), n_filler,
                               a.ctypes.data, b.ctypes.data, iterations, app.ctypes.data, er.ctypes.data,
                               it.ctypes.data)
    assert rc == 0
    return app, er, it


def check_pair(code, bg, rows, beta_q, iterations, app_clamp=32767, prologue=False, n_filler=0, label=""):
    app, er, it = emu_pair(code, bg, rows, beta_q, iterations, app_clamp, prologue, n_filler)
    for lane in range(2):
        inp = rows[lane].astype(np.int16)
        if prologue:
            inp = code.prologue_5g_i8(inp, n_filler, app_clamp)
        ref = code.decode_i8(inp, beta_q, iterations, app_clamp)
        assert it[lane] == ref["iters"], f"{label} lane {lane}: iterations {it[lane]} != {ref['iters']}"
        d = np.nonzero(app[lane] != ref["app"])[0]
        assert d.size == 0, f"{label} lane {lane}: posterior differs at {d[:5]} ({d.size})"
        d = np.nonzero(er[lane] != ref["edge_r"])[0]
        assert d.size == 0, f"{label} lane {lane}: messages differ at {d[:5]} ({d.size})"


def channel_rows(code, count, ebno, seed, n_filler=0):
    rows = []
    for i in range(count):
        info = O.random_bits(seed + 31 * i, code.k - n_filler)
        info = np.concatenate([info, np.zeros(n_filler, np.uint8)])
        cw = code.encode(info)
        rows.append(O.quantize_i16(O.awgn(cw, ebno + 0.5 * i, code.k / code.n, seed + 977 * i)).astype(np.int8))
    return rows


@pytest.mark.parametrize("bg,z", [(0, 2), (0, 13), (0, 52), (1, 7), (1, 44), (1, 96)])
def test_pair_matches_oracle(bg, z):
    code = O.Code.nr(bg, z)
    for ebno in (0.0, 1.5, 3.5):
        rows = channel_rows(code, 2, ebno, 0x7000 + z)
        check_pair(code, bg, rows, 4, 12, label=f"bg{bg + 1} z{z} {ebno}dB")


def test_pair_bg1_z384_lanes_converge_apart():
    """One lane converges early, the other runs to the iteration limit."""
    code = O.Code.nr(0, 384)
    good = channel_rows(code, 1, 3.0, 11)[0]
    bad = channel_rows(code, 1, -1.0, 12)[0]
    check_pair(code, 0, [good, bad], 4, 8, label="bg1 z384 good/bad")
    check_pair(code, 0, [bad, good], 4, 8, label="bg1 z384 bad/good")


@pytest.mark.parametrize("beta_q", [0, 1, 4, 127])
def test_pair_offsets(beta_q):
    code = O.Code.nr(1, 26)
    rows = channel_rows(code, 2, 1.0, 0x33 + beta_q)
    check_pair(code, 1, rows, beta_q, 9, label=f"beta_q {beta_q}")


def test_pair_extremes_and_zero_iterations():
    """Saturated channel values (-128 included), all-zero input, and 0 iterations."""
    code = O.Code.nr(0, 20)
    rng = np.random.default_rng(5)
    sat = rng.choice(np.array([-128, -127, 127], np.int8), size=code.n)
    zero = np.zeros(code.n, np.int8)
    check_pair(code, 0, [sat, zero], 4, 6, label="saturated/zero")
    check_pair(code, 0, [sat, zero], 4, 0, label="0 iterations")


@pytest.mark.parametrize("bg,z,n_filler,clamp", [(0, 64, 100, 32767), (1, 96, 144, 32767), (0, 32, 200, 7874),
                                                   (1, 384, 500, 9000)])
def test_pair_5g_prologue_with_filler(bg, z, n_filler, clamp):
    """Filler bits pinned at app_clamp: the kernel keeps them at the proxy ceiling and
    restores the true posterior on output."""
    code = O.Code.nr(bg, z)
    rows = channel_rows(code, 2, 0.5, 0x4400 + z, n_filler)
    for r in rows:
        r[: 2 * z] = 0
    check_pair(code, bg, rows, 4, 10, clamp, prologue=True, n_filler=n_filler, label=f"filler{n_filler}")


def test_pair_refuses_small_clamps():
    code = O.Code.nr(0, 8)
    rows = channel_rows(code, 2, 1.0, 3)
    _, cols, shifts = code.layout()
    assert emu().pair_emu_decode(0, 8, np.ascontiguousarray(shifts, np.int32).ctypes.data, 4, 3937, 0, 0,
                                 rows[0].ctypes.data, rows[1].ctypes.data, 2,
                                 np.zeros((2, code.n), np.int16).ctypes.data,
                                 np.zeros((2, code.edges * 8), np.int8).ctypes.data,
                                 np.zeros(2, np.int32).ctypes.data) == -1
