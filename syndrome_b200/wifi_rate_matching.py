"""Shortening and puncturing of IEEE 802.11 LDPC codewords (src/wifi_rate_matching.rs).

A payload shorter than K is padded with known-zero bits that are not sent
(shortening); trailing parity bits that do not fit the coded-bit budget are not
sent either (puncturing).  The receiver rebuilds the N-length codeword LLRs --
payload, a high-confidence known-zero LLR (1e6) for the shortened bits, the sent
parity, 0 (erasure) for the punctured bits -- and runs the ordinary f32 decode.

The single-codeword functions mirror the reference's (`decode_shortened` rebuilds the
caller's `codeword_llr` on the host and decodes it on the GPU);
`decode_shortened_batch` decodes a batch of received rows that are already in device
memory, and the f32 kernel rebuilds each codeword while it loads it.
"""
import ctypes

import numpy as np

from . import _lib
from .qc_ldpc import BatchResult, FecError, _buf

LLR_KNOWN_ZERO = 1_000_000.0


def shortening_and_puncture_counts(k, n, payload_bits, target_coded_bits):
    """(n_shrt, n_punc) for one codeword (wifi_rate_matching.rs:88).  Raises FecError
    (INVALID_PARAM) if n < k, payload_bits > k, target_coded_bits < payload_bits or
    target_coded_bits > n - (k - payload_bits)."""
    a, b = ctypes.c_size_t(), ctypes.c_size_t()
    _lib.check(_lib.load().syndrome_wifi_shortening_counts(int(k), int(n), int(payload_bits),
                                                           int(target_coded_bits), ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def encode_shortened(encoder, payload, target_coded_bits, out):
    """Payload bits (one per byte, <= K) -> the target_coded_bits sent bits
    (wifi_rate_matching.rs:163); `out` must have exactly target_coded_bits entries."""
    pay = np.ascontiguousarray(payload, dtype=np.uint8)
    op, on = _buf(out, np.uint8, "out")
    _lib.check(_lib.load().syndrome_wifi_encode_shortened(encoder._h, pay.ctypes.data, pay.size,
                                                          int(target_coded_bits), op, on))


def decode_shortened(decoder, payload_bits, rx_llr, codeword_llr, edge_r, layer_scratch, hard_output, iterations):
    """wifi_rate_matching.rs:267.  Rebuilds codeword_llr (length N) from rx_llr and
    decodes it in place; returns the iterations used.  The payload is
    hard_output[:payload_bits]."""
    rx = np.ascontiguousarray(rx_llr, dtype=np.float32)
    used = ctypes.c_size_t(0)
    args = [*_buf(codeword_llr, np.float32, "codeword_llr"), *_buf(edge_r, np.float32, "edge_r"),
            *_buf(layer_scratch, np.float32, "layer_scratch"), *_buf(hard_output, np.uint8, "hard_output")]
    _lib.check(_lib.load().syndrome_wifi_decode_shortened(decoder._h, int(payload_bits), rx.ctypes.data, rx.size,
                                                          *args, int(iterations), ctypes.byref(used)))
    return used.value


def decode_shortened_with_workspace(decoder, payload_bits, rx_llr, workspace, iterations):
    """wifi_rate_matching.rs:346: decode_shortened with the buffers of an
    LdpcWorkspace (the rebuilt posterior ends in workspace.codeword_llr)."""
    return decode_shortened(decoder, payload_bits, rx_llr, workspace.codeword_llr, workspace.edge_r,
                            workspace.layer_scratch, workspace.hard, iterations)


def decode_shortened_batch(decoder, rx, payload_bits, iterations, *, hard_bits=None, want_app=False,
                           want_hard=False, workspace=None, stream=None):
    """Batched device decode of received shortened / punctured codewords.

    rx: float32 CUDA tensor [batch, >= target_coded_bits]; its row length (or
    `target_coded_bits` = rx.shape[1]) is the number of sent bits.  Returns a
    BatchResult (packed hard decisions of the first hard_bits variables, default
    payload_bits; iterations used; optional posteriors and byte hard decisions)."""
    import torch

    if not (isinstance(rx, torch.Tensor) and rx.is_cuda and rx.dim() == 2 and rx.dtype == torch.float32):
        raise TypeError("rx must be a 2-D float32 CUDA tensor [batch, target_coded_bits]")
    if rx.stride(1) != 1:
        raise TypeError("rx rows must be contiguous")
    b, target = rx.shape
    n = decoder.variable_node_count()
    dev = rx.device
    hard_bits = int(payload_bits) if hard_bits is None else int(hard_bits)
    words = max((hard_bits + 31) // 32, 1)
    packed = torch.empty((b, words), dtype=torch.int32, device=dev)
    iters = torch.empty((b,), dtype=torch.int32, device=dev)
    app = torch.empty((b, n), dtype=torch.float32, device=dev) if want_app else None
    hard = torch.empty((b, n), dtype=torch.uint8, device=dev) if want_hard else None
    if workspace is None:
        need = decoder.batch_workspace_size(b, "f32")
        workspace = torch.empty((max(need, 1),), dtype=torch.uint8, device=dev)
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)

    def p(t):
        return t.data_ptr() if t is not None else None

    stride = rx.stride(0) if b > 1 else target
    st = _lib.load().syndrome_wifi_decode_shortened_batch_f32(
        decoder._h, rx.data_ptr(), stride, int(payload_bits), target, b, int(iterations), p(packed), hard_bits,
        packed.stride(0), p(iters), p(app), n, None, 0, p(hard), n, workspace.data_ptr(),
        workspace.numel(), sp)
    _lib.check(st)
    return BatchResult(hard_packed=packed, hard_bits=hard_bits, iters=iters, app=app, edge_r=None, hard=hard)


__all__ = ["LLR_KNOWN_ZERO", "shortening_and_puncture_counts", "encode_shortened", "decode_shortened",
           "decode_shortened_with_workspace", "decode_shortened_batch", "FecError"]
