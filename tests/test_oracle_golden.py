"""Pins the oracle (the CPU restatement used as the checker) to the reference's
own golden vectors and known-answer tests before anything is compared with it."""
import json
import os

import numpy as np
import pytest

import _oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def unpack(hexstr, n):
    return np.unpackbits(np.frombuffer(bytes.fromhex(hexstr), dtype=np.uint8), bitorder="little")[:n]


def test_fnv1a_checksum_bg1_z384():
    """bench/results/ldpc_{rust,cpp}.checksum: BG1 Z=384, beta 0.25, +-0.5 input, 10 iterations."""
    with open(os.path.join(GOLDEN, "ldpc_checksums.json")) as f:
        g = json.load(f)
    c = O.Code.nr(0, 384)
    llr = np.where(np.arange(c.n) % 2 == 0, 0.5, -0.5).astype(np.float32)
    r = c.decode_f32(llr, 0.25, 10)
    assert r["iters"] == 10
    got = "%016x" % O.fnv1a_hard(r["hard"])
    assert got == g["checksums"]["ldpc_rust.checksum"] == g["checksums"]["ldpc_cpp.checksum"]


def test_convergence_trajectory_wifi27():
    """bench/results/ldpc_convergence.json: encoder output, channel hard decisions
    and the hard decisions after each of the 13 iterations."""
    with open(os.path.join(GOLDEN, "ldpc_convergence_wifi27_r12.json")) as f:
        g = json.load(f)
    c = O.Code.wifi(27, 1, 2)
    n = g["n"]
    info = np.array([((i * 2654435761) >> 31) & 1 for i in range(c.k)], dtype=np.uint8)
    cw = c.encode(info)
    assert np.array_equal(cw, unpack(g["transmitted_codeword"], n))
    llr = O.awgn(cw, g["channel"]["eb_n0_db"], g["channel"]["code_rate"], g["channel"]["seed"])
    assert np.array_equal((llr < 0).astype(np.uint8), unpack(g["frames"][0]["hard_bits"], n))
    r = c.decode_f32(llr, g["code"]["offset_beta"], g["max_iterations"], trace=True)
    assert r["iters"] == g["iterations_used"] == 13
    for i in range(r["iters"]):
        fr = g["frames"][i + 1]
        assert fr["iteration"] == i + 1
        want = unpack(fr["hard_bits"], n)
        assert np.array_equal(r["trace"][i], want), f"iteration {i + 1}"
        assert int(np.sum(want != cw)) == fr["bit_errors"]


def test_quantize_known_answers():
    """src/quantize.rs:387-412."""
    out = O.quantize_i16(np.array([0.0, 1.0, -1.0, 1e9, -np.inf], dtype=np.float32), 8.0)
    assert out.tolist() == [0, 8, -8, 127, -127]
    assert O.quantize_i16(np.array([np.nan], dtype=np.float32), 8.0).tolist() == [0]
    assert O.quantize_i16(np.array([0.0625, -0.0625, 0.1875], dtype=np.float32), 8.0).tolist() == [1, -1, 2]


def test_beta_q_known_answers():
    """src/quantize.rs:368-385."""
    assert O.beta_q(0.5) == 4
    assert O.beta_q(0.125) == 1
    assert O.beta_q(0.0) == 0
    assert O.beta_q(-1.0) == 0
    assert O.beta_q(1e6) == 127
    assert O.beta_q(float("inf")) == 127
    assert O.beta_q(float("nan")) == 127


def test_dimensions():
    """src/qc_ldpc.rs:2829-2845."""
    c = O.Code.nr(0, 384)
    assert (c.n, c.k, c.m, c.edges * c.z, c.maxdeg * c.z) == (26112, 8448, 17664, 121344, 7296)
    c = O.Code.nr(1, 128)
    assert (c.n, c.k, c.edges) == (52 * 128, 10 * 128, 197)
    with pytest.raises(ValueError):
        O.Code.nr(0, 385)


def test_all_zero_converges_quickly():
    """src/qc_ldpc.rs:2862-2880 and tests/wifi_ldpc_integration.rs:133-157."""
    c = O.Code.nr(1, 2)
    r = c.decode_f32(np.full(c.n, 10.0, np.float32), 0.25, 50)
    assert r["iters"] <= 5
    for z in (27, 54, 81):
        for rn, rd in ((1, 2), (2, 3), (3, 4), (5, 6)):
            w = O.Code.wifi(z, rn, rd)
            r = w.decode_f32(np.full(w.n, 5.0, np.float32), 0.25, 10)
            assert r["iters"] == 1 and not r["hard"].any()


@pytest.mark.parametrize("bg,z", [(0, 2), (0, 16), (0, 52), (0, 96), (0, 384), (1, 2), (1, 16), (1, 128), (1, 208)])
def test_encoder_parity_5g(bg, z):
    """src/qc_ldpc.rs:2986-3085: the encoder output satisfies H c = 0."""
    c = O.Code.nr(bg, z)
    assert c.is_sparse_encoder()
    info = O.random_bits(0x1234 + z, c.k)
    cw = c.encode(info)
    assert np.array_equal(cw[: c.k], info)
    assert c.check(cw)


def test_encoder_parity_wifi():
    for z in (27, 54, 81):
        for rn, rd in ((1, 2), (2, 3), (3, 4), (5, 6)):
            c = O.Code.wifi(z, rn, rd)
            cw = c.encode(O.random_bits(z * 7 + rd, c.k))
            assert c.check(cw)


def test_int8_recovers_info_at_high_snr():
    """tests/ldpc_int8_kernel_equivalence.rs:345-382."""
    for bg, z in ((0, 96), (1, 128)):
        c = O.Code.nr(bg, z)
        info = O.random_bits(0x5EED, c.k)
        cw = c.encode(info)
        llr = O.awgn(cw, 6.0, c.k / c.n, 0x600D0000)
        r = c.decode_i8(O.quantize_i16(llr), O.beta_q(0.5), 12)
        assert np.array_equal(r["hard"][: c.k], info)
