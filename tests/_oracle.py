"""ctypes binding of the oracle (oracle/liboracle.so): a CPU restatement of the
reference's decode path used only by the tests as the checker.  Nothing in the
decoder package imports this module."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
_LIB = None

_c_int_p = ctypes.POINTER(ctypes.c_int)


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(ORACLE_DIR, "liboracle.so")
        src = os.path.join(ORACLE_DIR, "oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR, "liboracle.so"])
        L = ctypes.CDLL(path)
        L.orc_params_5g.restype = ctypes.c_void_p
        L.orc_params_5g.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_params_wifi.restype = ctypes.c_void_p
        L.orc_params_wifi.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_params_raw.restype = ctypes.c_void_p
        L.orc_params_raw.argtypes = [_c_int_p, _c_int_p, _c_int_p] + [ctypes.c_int] * 4
        L.orc_params_free.argtypes = [ctypes.c_void_p]
        L.orc_params_info.argtypes = [ctypes.c_void_p, _c_int_p]
        L.orc_params_layout.argtypes = [ctypes.c_void_p, _c_int_p, _c_int_p, _c_int_p]
        L.orc_decode_f32.restype = ctypes.c_long
        L.orc_decode_f32.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
        L.orc_init_5g_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
        L.orc_decode_i8.restype = ctypes.c_long
        L.orc_decode_i8.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
        L.orc_prologue_5g_i8.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_int]
        L.orc_beta_q.restype = ctypes.c_int
        L.orc_beta_q.argtypes = [ctypes.c_float, ctypes.c_float]
        L.orc_quantize_i16.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_float]
        L.orc_encode.restype = ctypes.c_int
        L.orc_encode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_encoder_is_sparse.restype = ctypes.c_int
        L.orc_encoder_is_sparse.argtypes = [ctypes.c_void_p]
        L.orc_check_codeword.restype = ctypes.c_int
        L.orc_check_codeword.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_awgn_sigma.restype = ctypes.c_float
        L.orc_awgn_sigma.argtypes = [ctypes.c_float, ctypes.c_float]
        L.orc_awgn_transmit.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_uint64,
                                        ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
        L.orc_segmentation.restype = ctypes.c_int
        L.orc_segmentation.argtypes = [ctypes.c_long, ctypes.c_float, ctypes.c_void_p]
        L.orc_crc24.restype = ctypes.c_uint
        L.orc_crc24.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int]
        L.orc_dlsch_encode.restype = ctypes.c_long
        L.orc_dlsch_encode.argtypes = [ctypes.c_long, ctypes.c_float, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_void_p]
        L.orc_dlsch_decoder_new.restype = ctypes.c_void_p
        L.orc_dlsch_decoder_new.argtypes = [ctypes.c_long, ctypes.c_float, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_float, ctypes.c_int]
        L.orc_dlsch_decoder_free.argtypes = [ctypes.c_void_p]
        L.orc_dlsch_decode.restype = ctypes.c_int
        L.orc_dlsch_decode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_dlsch_flush.argtypes = [ctypes.c_void_p]
        L.orc_fnv1a_hard.restype = ctypes.c_uint64
        L.orc_fnv1a_hard.argtypes = [ctypes.c_void_p, ctypes.c_long]
        _LIB = L
    return _LIB


class Code:
    """One expanded QC-LDPC code in the oracle (reference QcLdpcParams)."""

    def __init__(self, handle):
        if not handle:
            raise ValueError("invalid code parameters")
        self.h = handle
        info = np.zeros(8, dtype=np.int32)
        lib().orc_params_info(self.h, _ptr(info, ctypes.c_int))
        self.mb, self.nb, self.z, self.edges, self.maxdeg, self.n, self.k, self.m = [int(x) for x in info]

    @classmethod
    def nr(cls, bg, z):
        return cls(lib().orc_params_5g(bg, z))

    @classmethod
    def wifi(cls, z, rn, rd):
        return cls(lib().orc_params_wifi(z, rn, rd))

    def __del__(self):
        try:
            lib().orc_params_free(self.h)
        except Exception:
            pass

    def layout(self):
        lo = np.zeros(self.mb + 1, dtype=np.int32)
        c = np.zeros(self.edges, dtype=np.int32)
        s = np.zeros(self.edges, dtype=np.int32)
        lib().orc_params_layout(self.h, _ptr(lo, ctypes.c_int), _ptr(c, ctypes.c_int), _ptr(s, ctypes.c_int))
        return lo, c, s

    def encode(self, info):
        info = np.ascontiguousarray(info, dtype=np.uint8)
        assert info.size == self.k
        cw = np.zeros(self.n, dtype=np.uint8)
        rc = lib().orc_encode(self.h, info.ctypes.data, cw.ctypes.data)
        assert rc == 0
        return cw

    def is_sparse_encoder(self):
        return bool(lib().orc_encoder_is_sparse(self.h))

    def check(self, bits):
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        return bool(lib().orc_check_codeword(self.h, bits.ctypes.data))

    def decode_f32(self, llr, beta, iterations, trace=False):
        llr = np.array(llr, dtype=np.float32, copy=True)
        edge_r = np.zeros(self.edges * self.z, dtype=np.float32)
        hard = np.zeros(self.n, dtype=np.uint8)
        tr = np.zeros((max(iterations, 1), self.n), dtype=np.uint8) if trace else None
        used = lib().orc_decode_f32(self.h, beta, llr.ctypes.data, edge_r.ctypes.data, hard.ctypes.data,
                                    iterations, tr.ctypes.data if trace else None)
        out = dict(iters=int(used), llr=llr, edge_r=edge_r, hard=hard)
        if trace:
            out["trace"] = tr[:used]
        return out

    def init_5g_f32(self, llr, n_filler):
        llr = np.array(llr, dtype=np.float32, copy=True)
        lib().orc_init_5g_f32(self.h, llr.ctypes.data, n_filler)
        return llr

    def decode_i8(self, app, beta_q, iterations, app_clamp=32767):
        app = np.array(app, dtype=np.int16, copy=True)
        edge_r = np.zeros(self.edges * self.z, dtype=np.int8)
        hard = np.zeros(self.n, dtype=np.uint8)
        used = lib().orc_decode_i8(self.h, beta_q, app_clamp, app.ctypes.data, edge_r.ctypes.data,
                                   hard.ctypes.data, iterations)
        return dict(iters=int(used), app=app, edge_r=edge_r, hard=hard)

    def prologue_5g_i8(self, app, n_filler, app_clamp=32767):
        app = np.array(app, dtype=np.int16, copy=True)
        lib().orc_prologue_5g_i8(self.h, app.ctypes.data, n_filler, app_clamp)
        return app


def beta_q(beta, scale=8.0):
    return int(lib().orc_beta_q(beta, scale))


def quantize_i16(llr, scale=8.0):
    llr = np.ascontiguousarray(llr, dtype=np.float32)
    out = np.zeros(llr.size, dtype=np.int16)
    lib().orc_quantize_i16(llr.ctypes.data, out.ctypes.data, llr.size, scale)
    return out


def awgn(bits, ebno_db, rate, seed):
    bits = np.ascontiguousarray(bits, dtype=np.uint8)
    out = np.zeros(bits.size, dtype=np.float32)
    lib().orc_awgn_transmit(ebno_db, rate, seed, bits.ctypes.data, bits.size, out.ctypes.data)
    return out


def awgn_sigma(ebno_db, rate):
    return float(lib().orc_awgn_sigma(ebno_db, rate))


def fnv1a_hard(hard):
    hard = np.ascontiguousarray(hard, dtype=np.uint8)
    return int(lib().orc_fnv1a_hard(hard.ctypes.data, hard.size))


def random_bits(seed, n):
    """xorshift64 bit stream of the reference's int8 equivalence test
    (tests/ldpc_int8_kernel_equivalence.rs:27-37): bit = (s >> 27) & 1."""
    s = (seed | 1) & 0xFFFFFFFFFFFFFFFF
    out = np.zeros(n, dtype=np.uint8)
    M = 0xFFFFFFFFFFFFFFFF
    for i in range(n):
        s ^= (s << 13) & M
        s ^= s >> 7
        s ^= (s << 17) & M
        out[i] = (s >> 27) & 1
    return out


# ------------------------------------------------------------------ DL-SCH --

def segmentation(a, rate):
    """compute_segmentation: (bg, z, c, b, k_prime, k, ncb, n_filler, has_cb_crc, payload) or None."""
    out = np.zeros(10, dtype=np.int64)
    if lib().orc_segmentation(a, rate, out.ctypes.data):
        return None
    return tuple(int(x) for x in out)


def crc24(bits, kind=0):
    b = np.ascontiguousarray(bits, dtype=np.uint8)
    return int(lib().orc_crc24(b.ctypes.data, b.size, kind))


def dlsch_encode(tb, rate, qm, g, rv):
    tb = np.ascontiguousarray(tb, dtype=np.uint8)
    out = np.zeros(g, dtype=np.uint8)
    n = lib().orc_dlsch_encode(tb.size, rate, qm, g, rv, tb.ctypes.data, out.ctypes.data)
    assert n >= 0
    return out[:n]


class DlSchDecoder:
    """transport_block.rs DlSchDecoder with the int8 code-block decode (HARQ f32 sum,
    quantize_llr_i16, decode_5g_i8)."""

    def __init__(self, tb_size, rate, qm, g, iterations=8, beta_q=4, scale=8.0, app_clamp=32767, f32_beta=None):
        self.h = lib().orc_dlsch_decoder_new(tb_size, rate, qm, g, iterations, beta_q, scale, app_clamp)
        assert self.h
        if f32_beta is not None:  # the reference's own f32 code-block decode
            lib().orc_dlsch_set_f32.argtypes = [ctypes.c_void_p, ctypes.c_float]
            lib().orc_dlsch_set_f32(self.h, f32_beta)
        self.tb_size = tb_size
        self.seg = segmentation(tb_size, rate)

    def __del__(self):
        try:
            lib().orc_dlsch_decoder_free(self.h)
        except Exception:
            pass

    def decode(self, rx, rv):
        rx = np.ascontiguousarray(rx, dtype=np.float32)
        c, ncb = self.seg[2], self.seg[6]
        tb = np.zeros(self.tb_size, np.uint8)
        rep = np.zeros(4, np.int32)
        cb = np.zeros(c, np.uint8)
        llr = np.zeros((c, ncb), np.int8)
        its = np.zeros(c, np.int32)
        lib().orc_dlsch_decode(self.h, rx.ctypes.data, rv, tb.ctypes.data, rep.ctypes.data, cb.ctypes.data,
                               llr.ctypes.data, its.ctypes.data)
        return dict(crc_ok=bool(rep[0]), max_iters=int(rep[1]), harq_tx=int(rep[2]), cb_crc=cb.astype(bool),
                    tb=tb if rep[0] else None, llr=llr, iters=its)

    def flush(self):
        lib().orc_dlsch_flush(self.h)


# ---- Wi-Fi shortening / puncturing (src/wifi_rate_matching.rs) ----
def wifi_counts(k, n, payload, target):
    out = np.zeros(2, dtype=np.int64)
    L = lib()
    L.orc_wifi_counts.argtypes = [ctypes.c_long] * 4 + [ctypes.c_void_p]
    rc = L.orc_wifi_counts(k, n, payload, target, out.ctypes.data)
    return None if rc != 0 else (int(out[0]), int(out[1]))


def wifi_encode_shortened(code, payload, target):
    payload = np.ascontiguousarray(payload, dtype=np.uint8)
    out = np.zeros(target, dtype=np.uint8)
    L = lib()
    L.orc_wifi_encode_shortened.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_long,
                                            ctypes.c_void_p]
    rc = L.orc_wifi_encode_shortened(code.h, payload.ctypes.data, payload.size, target, out.ctypes.data)
    assert rc == 0
    return out


def wifi_decode_shortened(code, beta, payload_bits, rx, iterations):
    rx = np.ascontiguousarray(rx, dtype=np.float32)
    cw = np.zeros(code.n, dtype=np.float32)
    edge_r = np.zeros(code.edges * code.z, dtype=np.float32)
    hard = np.zeros(code.n, dtype=np.uint8)
    L = lib()
    L.orc_wifi_decode_shortened.restype = ctypes.c_long
    L.orc_wifi_decode_shortened.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_long, ctypes.c_void_p,
                                            ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_long]
    used = L.orc_wifi_decode_shortened(code.h, beta, payload_bits, rx.ctypes.data, rx.size, cw.ctypes.data,
                                       edge_r.ctypes.data, hard.ctypes.data, iterations)
    assert used >= 0
    return dict(iters=int(used), llr=cw, edge_r=edge_r, hard=hard)


# ---- threaded batch helpers (same single-codeword code, the batch split over threads) ----
def _batch_lib():
    L = lib()
    if not getattr(L, "_batch_bound", False):
        vp, lg = ctypes.c_void_p, ctypes.c_long
        L.orc_batch_channel_i8.restype = ctypes.c_int
        L.orc_batch_channel_i8.argtypes = [vp, vp, lg, vp, ctypes.c_float, vp, ctypes.c_float, lg, vp, lg,
                                           ctypes.c_int]
        L.orc_batch_channel_f32.restype = ctypes.c_int
        L.orc_batch_channel_f32.argtypes = [vp, vp, lg, vp, ctypes.c_float, vp, lg, vp, lg, ctypes.c_int]
        L.orc_decode_i8_batch.restype = None
        L.orc_decode_i8_batch.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, lg, lg, ctypes.c_int, lg, lg, lg,
                                          ctypes.c_int, vp, vp, lg, lg, vp, vp, lg]
        L.orc_decode_f32_batch.restype = None
        L.orc_decode_f32_batch.argtypes = [vp, ctypes.c_float, vp, lg, lg, ctypes.c_int, lg, lg, lg, ctypes.c_int,
                                           vp, vp, lg, lg, vp, lg]
        L._batch_bound = True
    return L


def batch_channel_i8(code, info, ebno, rate, seeds, scale=8.0, tx_begin=0, threads=0):
    """info [count, K] -> int8 LLRs [count, N - tx_begin]: oracle encoder, the reference
    channel over all N bits (seed per row), quantized at `scale`."""
    info = np.ascontiguousarray(info, dtype=np.uint8)
    count = info.shape[0]
    eb = np.ascontiguousarray(np.broadcast_to(np.asarray(ebno, dtype=np.float32), (count,)))
    sd = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64).reshape(count))
    out = np.zeros((count, code.n - tx_begin), dtype=np.int8)
    rc = _batch_lib().orc_batch_channel_i8(code.h, info.ctypes.data, count, eb.ctypes.data, rate, sd.ctypes.data,
                                           scale, tx_begin, out.ctypes.data, out.shape[1], threads)
    assert rc == 0
    return out


def batch_channel_f32(code, info, ebno, rate, seeds, tx_begin=0, threads=0):
    """info [count, K] -> f32 channel LLRs [count, N - tx_begin] (oracle encoder + channel)."""
    info = np.ascontiguousarray(info, dtype=np.uint8)
    count = info.shape[0]
    eb = np.ascontiguousarray(np.broadcast_to(np.asarray(ebno, dtype=np.float32), (count,)))
    sd = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64).reshape(count))
    out = np.zeros((count, code.n - tx_begin), dtype=np.float32)
    rc = _batch_lib().orc_batch_channel_f32(code.h, info.ctypes.data, count, eb.ctypes.data, rate, sd.ctypes.data,
                                            tx_begin, out.ctypes.data, out.shape[1], threads)
    assert rc == 0
    return out


def decode_i8_batch(code, llr, beta_q, iterations, llr_offset=0, nr_prologue=False, n_filler=0, app_clamp=32767,
                    hard_bits=None, detail=0, threads=0):
    """Oracle int8 decode of int8 rows [count, N - llr_offset] (the batched device API's
    input).  Returns iters [count], packed hard bits [count, words] and, for the first
    `detail` codewords, posteriors [detail, N] and messages [detail, E*Z]."""
    llr = np.ascontiguousarray(llr, dtype=np.int8)
    count = llr.shape[0]
    hb = code.n if hard_bits is None else hard_bits
    words = (hb + 31) // 32
    iters = np.zeros(count, np.int32)
    packed = np.zeros((count, words), np.uint32)
    app = np.zeros((max(detail, 0), code.n), np.int16)
    er = np.zeros((max(detail, 0), code.edges * code.z), np.int8)
    _batch_lib().orc_decode_i8_batch(code.h, beta_q, app_clamp, llr.ctypes.data, llr.shape[1], llr_offset,
                                     1 if nr_prologue else 0, n_filler, count, iterations, threads, iters.ctypes.data,
                                     packed.ctypes.data, hb, words, app.ctypes.data, er.ctypes.data, detail)
    return dict(iters=iters, packed=packed, app=app, edge_r=er)


def decode_f32_batch(code, llr, beta, iterations, llr_offset=0, nr_prologue=False, n_filler=0, hard_bits=None,
                     detail=0, threads=0):
    """Oracle f32 decode of f32 rows [count, N - llr_offset]."""
    llr = np.ascontiguousarray(llr, dtype=np.float32)
    count = llr.shape[0]
    hb = code.n if hard_bits is None else hard_bits
    words = (hb + 31) // 32
    iters = np.zeros(count, np.int32)
    packed = np.zeros((count, words), np.uint32)
    app = np.zeros((max(detail, 0), code.n), np.float32)
    _batch_lib().orc_decode_f32_batch(code.h, beta, llr.ctypes.data, llr.shape[1], llr_offset,
                                      1 if nr_prologue else 0, n_filler, count, iterations, threads,
                                      iters.ctypes.data, packed.ctypes.data, hb, words, app.ctypes.data, detail)
    return dict(iters=iters, packed=packed, app=app)
