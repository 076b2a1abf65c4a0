"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and its host-side parts (encoder, channel, quantizer, argument
validation) agree with the oracle and the reference's error conventions."""
import ctypes
import os
import re

import numpy as np
import pytest

import _oracle as O
import syndrome_b200 as S
from syndrome_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "syndrome_ldpc.h")


def header_functions():
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(syndrome_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.PROTOTYPES, f"{name} has no ctypes prototype"


def test_drop_in_symbols_match_reference_capi():
    """The 13 extern "C" functions of capi/src/lib.rs keep their names."""
    capi = ["syndrome_ldpc_decoder_create", "syndrome_ldpc_decoder_destroy",
            "syndrome_ldpc_decoder_variable_node_count", "syndrome_ldpc_decoder_info_bit_count",
            "syndrome_ldpc_decoder_required_edge_buffer", "syndrome_ldpc_decoder_required_layer_buffer",
            "syndrome_ldpc_decode_5g", "syndrome_ldpc_encoder_create", "syndrome_ldpc_encoder_destroy",
            "syndrome_ldpc_encoder_info_bit_count", "syndrome_ldpc_encoder_codeword_bit_count",
            "syndrome_ldpc_encode_5g"]
    assert set(capi) <= set(header_functions())


@pytest.mark.parametrize("bg,z", [(0, 2), (0, 7), (0, 44), (0, 96), (0, 384), (1, 3), (1, 13), (1, 52), (1, 128),
                                  (1, 384)])
def test_encoder_matches_oracle_5g(bg, z):
    enc = S.QcLdpcEncoder.new(bg, z)
    ref = O.Code.nr(bg, z)
    assert enc.info_bit_count() == ref.k and enc.codeword_bit_count() == ref.n
    info = O.random_bits(0xA5A5 ^ z, ref.k)
    cw = np.zeros(ref.n, dtype=np.uint8)
    enc.encode(info, cw)
    assert np.array_equal(cw, ref.encode(info))


def test_encoder_matches_oracle_wifi_and_batch():
    for z in (27, 54, 81):
        for rn, rd in ((1, 2), (2, 3), (3, 4), (5, 6)):
            enc = S.wifi_ldpc_encoder(z, rn, rd)
            ref = O.Code.wifi(z, rn, rd)
            infos = np.stack([O.random_bits(s * 31 + z, ref.k) for s in range(3)])
            cws = enc.encode_batch(infos, threads=2)
            for i in range(3):
                assert np.array_equal(cws[i], ref.encode(infos[i]))


def test_encode_5g_filler_and_errors():
    enc = S.QcLdpcEncoder.new(S.BaseGraph.Bg2, 16)
    k, n = enc.info_bit_count(), enc.codeword_bit_count()
    info = O.random_bits(7, k - 5)
    cw = np.zeros(n, dtype=np.uint8)
    enc.encode_5g(info, 5, cw)
    full = np.concatenate([info, np.zeros(5, np.uint8)])
    assert np.array_equal(cw, O.Code.nr(1, 16).encode(full))
    with pytest.raises(S.FecError) as e:
        enc.encode_5g(info, k + 1, cw)
    assert e.value.status == _lib.INVALID_PARAM
    with pytest.raises(S.FecError) as e:
        enc.encode_5g(info[:-1], 5, cw)
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.FecError) as e:
        enc.encode(full, np.zeros(n - 1, np.uint8))
    assert e.value.status == _lib.BUFFER_TOO_SMALL


def test_quantizer_and_beta_q_known_answers():
    """src/quantize.rs:368-412."""
    out = S.quantize_llr_i16(np.array([0.0, 1.0, -1.0, 1e9, -np.inf, np.nan], np.float32))
    assert out.tolist() == [0, 8, -8, 127, -127, 0]
    q = S.QuantParams()
    assert [q.beta_q(b) for b in (0.5, 0.125, 0.0, -1.0, 1e6, float("inf"), float("nan"))] == [4, 1, 0, 0, 127, 127, 127]
    x = np.random.default_rng(1).normal(0, 20, 5000).astype(np.float32)
    assert np.array_equal(S.quantize_llr_i16(x), O.quantize_i16(x))


def test_channel_matches_oracle():
    bits = O.random_bits(99, 2000)
    ch = S.AwgnChannel(1.5, 0.5, 139)
    a = ch.transmit(bits[:700])
    b = ch.transmit(bits[700:])
    assert np.array_equal(np.concatenate([a, b]), O.awgn(bits, 1.5, 0.5, 139))
    cws = np.stack([O.random_bits(s, 300) for s in range(4)])
    q = S.awgn_quantized_batch(cws, 1.0, 1 / 3, seeds=[11, 12, 13, 14], tx_begin=20, threads=2)
    for i in range(4):
        want = O.quantize_i16(O.awgn(cws[i], 1.0, 1 / 3, 11 + i))[20:]
        assert np.array_equal(q[i].astype(np.int16), want)


def test_constructor_argument_errors_without_gpu():
    L = _lib.load()
    h = ctypes.c_void_p(1)
    assert L.syndrome_ldpc_decoder_create(2, 384, 0.5, ctypes.byref(h)) == _lib.INVALID_PARAM
    assert h.value is None
    assert L.syndrome_ldpc_decoder_create(0, 385, 0.5, ctypes.byref(h)) == _lib.INVALID_PARAM
    assert L.syndrome_ldpc_decoder_create(0, 384, 0.5, None) == _lib.NULL_POINTER
    assert L.syndrome_ldpc_decoder_create_wifi(27, 1, 3, 0.5, ctypes.byref(h)) == _lib.INVALID_PARAM
    assert L.syndrome_ldpc_encoder_create(5, 384, ctypes.byref(h)) == _lib.INVALID_PARAM
    rows = np.array([0, 0], np.uint8)
    cols = np.array([0, 1], np.uint8)
    shifts = np.array([0, 4], np.int16)  # shift >= z
    assert L.syndrome_ldpc_decoder_create_raw(rows.ctypes.data, cols.ctypes.data, shifts.ctypes.data, 2, 1, 3, 4,
                                              0.5, ctypes.byref(h)) == _lib.INVALID_PARAM
    L.syndrome_ldpc_decoder_destroy(None)
    L.syndrome_ldpc_encoder_destroy(None)


def test_decode_entry_points_reject_null_pointers():
    L = _lib.load()
    assert L.syndrome_ldpc_decode_5g(None, None, 0, 0, None, 0, None, 0, None, 0, 1, None) == _lib.NULL_POINTER
    assert L.syndrome_ldpc_decode_batch_i8(None, None, 0, 0, 1, 0, 0, 8, 8.0, 32767, None, 0, 0, None, None, 0,
                                           None, 0, None, 0, None, 0, None) == _lib.NULL_POINTER
