"""Mixed-shape batches: codewords of any 5G NR base graph and lifting size decoded by
one persistent launch (a device work queue of same-shape tiles), optionally replayed
from a captured CUDA graph.  No counterpart in the reference, which decodes one code
block per call; the per-codeword arithmetic is that of decode_5g_i8
(src/qc_ldpc.rs:1486)."""
import ctypes

import numpy as np

from . import _lib
from .qc_ldpc import QuantParams

CODEWORD_DTYPE = np.dtype([("base_graph", "<i4"), ("z", "<i4"), ("n_filler", "<i4"), ("hard_bits", "<i4"),
                           ("llr_offset", "<i8"), ("out_offset", "<i8")])

LIFTING_SIZES = (2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 18, 20, 22, 24, 26, 28, 30, 32, 36, 40, 44,
                 48, 52, 56, 60, 64, 72, 80, 88, 96, 104, 112, 120, 128, 144, 160, 176, 192, 208, 224, 240, 256,
                 288, 320, 352, 384)


def code_dims(bg, z):
    """(N, K, rows) of 5G NR base graph bg (0 = BG1, 1 = BG2) at lifting size z."""
    nb, mb = (68, 46) if bg == 0 else (52, 42)
    return nb * z, (nb - mb) * z, mb


def tile_capacity(bg, z):
    """Most codewords of this shape one work item (one CTA) holds."""
    return int(_lib.load().syndrome_mixed_tile_capacity(bg, z))


class MixedBatch:
    """A planned batch.  `codewords` is a structured array of CODEWORD_DTYPE (or
    anything convertible): per codeword its base graph, lifting size, filler count,
    number of leading hard decisions to report, byte offset of its N - 2Z int8 LLRs
    in the LLR buffer and word offset of its packed hard decisions."""

    def __init__(self, codewords, offset_beta=0.5, quant=None, iterations=8, tile_hints=None):
        quant = quant or QuantParams()
        cw = np.ascontiguousarray(np.asarray(codewords, dtype=CODEWORD_DTYPE))
        self.codewords = cw
        if isinstance(tile_hints, dict):
            tile_hints = [(bg, z, t) for (bg, z), t in tile_hints.items()]
        hints = np.ascontiguousarray(np.asarray(tile_hints or [], dtype=np.int32).reshape(-1, 3))
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_mixed_plan_create(
            cw.ctypes.data, len(cw), offset_beta, quant.scale, quant.app_clamp, iterations,
            hints.ctypes.data if len(hints) else None, len(hints), ctypes.byref(h)))
        self._h = h.value
        self.iterations = iterations

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.load().syndrome_mixed_plan_destroy(h)
            except Exception:
                pass

    def set_kernel(self, kernel="auto"):
        """"auto" (the paired kernel with most of its check-row state in tensor
        memory, two CTAs per SM, when app_clamp >= 7874 and no codeword reports hard
        decisions past its core columns) or "pair_smem" (all of it in shared memory,
        one CTA per SM).  Returns True when decode runs the tensor-memory form."""
        code = {"auto": 0, "pair_smem": 5}.get(kernel)
        if code is None:
            raise ValueError(f"unknown mixed-batch kernel {kernel!r}")
        tm = ctypes.c_int32(0)
        _lib.check(_lib.load().syndrome_mixed_plan_set_kernel(self._h, code, ctypes.byref(tm)))
        return bool(tm.value)

    def items(self):
        """(base_graph, z, codewords) of each work item in launch order."""
        L = _lib.load()
        n = ctypes.c_size_t(0)
        _lib.check(L.syndrome_mixed_plan_items(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 3), dtype=np.int32)
        _lib.check(L.syndrome_mixed_plan_items(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return [tuple(int(x) for x in r) for r in out]

    def decode(self, llr, out, iters=None, use_graph=False, stream=None):
        """llr: int8 CUDA tensor holding every codeword's LLRs at its offset;
        out: int32 CUDA tensor of packed hard-decision words; iters: optional int32
        CUDA tensor with one entry per codeword."""
        import torch

        for t, name in ((llr, "llr"), (out, "out")):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
                raise TypeError(f"{name} must be a contiguous CUDA tensor")
        if stream is None:
            stream = torch.cuda.current_stream(llr.device)
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        if llr.dtype != torch.int8 or out.dtype != torch.int32:
            raise TypeError("llr must be int8 and out int32")
        if iters is not None and not (iters.is_cuda and iters.dtype == torch.int32 and iters.is_contiguous()):
            raise TypeError("iters must be a contiguous int32 CUDA tensor")
        _lib.check(_lib.load().syndrome_mixed_decode(
            self._h, llr.data_ptr(), llr.numel(), out.data_ptr(), out.numel(),
            iters.data_ptr() if iters is not None else None, iters.numel() if iters is not None else 0,
            int(bool(use_graph)), ctypes.c_void_p(sp)))


WIFI_CODEWORD_DTYPE = np.dtype([("z", "<i4"), ("rate_num", "<i4"), ("rate_den", "<i4"), ("hard_bits", "<i4"),
                                ("llr_offset", "<i8"), ("out_offset", "<i8")])

WIFI_SHAPES = tuple((z, rn, rd) for z in (27, 54, 81) for rn, rd in ((1, 2), (2, 3), (3, 4), (5, 6)))


def wifi_dims(z, rate_num, rate_den):
    """(N, K) of the 802.11 matrix at lifting size z (24 block columns) and rate."""
    n = 24 * z
    return n, n * rate_num // rate_den


class WifiMixedBatch:
    """A planned batch of 802.11 codewords of any mix of the twelve matrices, decoded
    by one persistent f32 launch.  `codewords` is a structured array of
    WIFI_CODEWORD_DTYPE: per codeword its lifting size, rate, number of leading hard
    decisions to report, element offset of its N f32 channel LLRs in the LLR buffer
    and word offset of its packed hard decisions.  No counterpart in the reference,
    which decodes one codeword per call (decode_layered_offset_min_sum,
    src/qc_ldpc.rs:962)."""

    def __init__(self, codewords, offset_beta=0.5, iterations=20, chunk=0):
        cw = np.ascontiguousarray(np.asarray(codewords, dtype=WIFI_CODEWORD_DTYPE))
        self.codewords = cw
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_wifi_mixed_plan_create(cw.ctypes.data, len(cw), offset_beta, iterations,
                                                               chunk, ctypes.byref(h)))
        self._h = h.value
        self.iterations = iterations

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.load().syndrome_wifi_mixed_plan_destroy(h)
            except Exception:
                pass

    def chunks(self):
        """(chunks on the device queue, CTAs of the launch)."""
        n, c = ctypes.c_size_t(0), ctypes.c_size_t(0)
        _lib.check(_lib.load().syndrome_wifi_mixed_plan_chunks(self._h, ctypes.byref(n), ctypes.byref(c)))
        return n.value, c.value

    def decode(self, llr, out, iters=None, use_graph=False, stream=None):
        """llr: float32 CUDA tensor holding every codeword's LLRs at its offset; out:
        int32 CUDA tensor of packed hard-decision words; iters: optional int32 CUDA
        tensor with one entry per codeword."""
        import torch

        for t, name in ((llr, "llr"), (out, "out")):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
                raise TypeError(f"{name} must be a contiguous CUDA tensor")
        if llr.dtype != torch.float32 or out.dtype != torch.int32:
            raise TypeError("llr must be float32 and out int32")
        if iters is not None and not (iters.is_cuda and iters.dtype == torch.int32 and iters.is_contiguous()):
            raise TypeError("iters must be a contiguous int32 CUDA tensor")
        if stream is None:
            stream = torch.cuda.current_stream(llr.device)
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        _lib.check(_lib.load().syndrome_wifi_mixed_decode(
            self._h, llr.data_ptr(), llr.numel(), out.data_ptr(), out.numel(),
            iters.data_ptr() if iters is not None else None, iters.numel() if iters is not None else 0,
            int(bool(use_graph)), ctypes.c_void_p(sp)))
