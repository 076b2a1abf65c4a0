"""5G NR transport blocks (DL-SCH): segmentation, CRC-24A/B and the transport-block
encoder, mirroring syndrome's segmentation.rs (compute_segmentation), crc.rs (Crc24)
and transport_block.rs (DlSchEncoder, DlSchDecoder).  DlSchDecoder decodes one
transport block per call with the reference's f32 code-block decode on the GPU; the
device-resident serving engine (serve.py) decodes many at once with the int8 kernels."""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

MAX_TB_SIZE_BITS = 1_277_992
CRC24A, CRC24B = 0, 1


@dataclass(frozen=True)
class SegmentationParams:
    """segmentation.rs SegmentationParams (n is the circular buffer length N - 2Z)."""
    bg: int
    z: int
    c: int
    b: int
    k_prime: int
    k: int
    n: int
    n_filler: int
    has_cb_crc: bool
    payload: int


def compute_segmentation(tb_size, target_rate):
    out = np.zeros(10, dtype=np.int64)
    _lib.check(_lib.load().syndrome_tb_segmentation(tb_size, target_rate, out.ctypes.data))
    v = [int(x) for x in out]
    return SegmentationParams(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], bool(v[8]), v[9])


def crc24(bits, kind=CRC24A):
    """Crc24::compute over a bit array (one bit per element)."""
    b = np.ascontiguousarray(bits, dtype=np.uint8)
    return int(_lib.load().syndrome_crc24(b.ctypes.data, b.size, kind))


class DlSchEncoder:
    """transport_block.rs DlSchEncoder: TB CRC, segmentation, LDPC encoding, rate matching."""

    def __init__(self, tb_size, target_rate, qm, g):
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_dlsch_encoder_create(tb_size, target_rate, qm, g, ctypes.byref(h)))
        self._h = h.value
        self.tb_size = tb_size
        self.segmentation = compute_segmentation(tb_size, target_rate)

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.load().syndrome_dlsch_encoder_destroy(h)
            except Exception:
                pass

    def output_bits(self):
        return int(_lib.load().syndrome_dlsch_encoder_output_bits(self._h))

    def num_code_blocks(self):
        return int(_lib.load().syndrome_dlsch_encoder_num_code_blocks(self._h))

    def encode(self, tb, rv):
        tb = np.ascontiguousarray(tb, dtype=np.uint8)
        out = np.zeros(self.output_bits(), dtype=np.uint8)
        _lib.check(_lib.load().syndrome_dlsch_encode(self._h, tb.ctypes.data, tb.size, rv, out.ctypes.data, out.size))
        return out


@dataclass(frozen=True)
class DecodeReport:
    """transport_block.rs:140 DecodeReport."""
    crc_ok: bool
    cb_crc: tuple
    max_iters_used: int
    harq_tx_count: int


class _Report(ctypes.Structure):
    _fields_ = [("crc_ok", ctypes.c_int32), ("max_iters_used", ctypes.c_int32), ("harq_tx_count", ctypes.c_int32),
                ("num_code_blocks", ctypes.c_int32)]


class DlSchDecoder:
    """transport_block.rs:405-1060 DlSchDecoder: HARQ f32 soft combining, the 5G
    prologue and the f32 layered decode of all code blocks in one GPU launch, CB
    CRC-24B, TB CRC-24A, HARQ flush on success."""

    def __init__(self, tb_size, target_rate, qm, g, iterations, offset_beta):
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_dlsch_decoder_create(tb_size, target_rate, qm, g, iterations, offset_beta,
                                                            ctypes.byref(h)))
        self._h = h.value
        self.tb_size = tb_size

    @classmethod
    def new(cls, tb_size, target_rate, qm, g, iterations, offset_beta):
        return cls(tb_size, target_rate, qm, g, iterations, offset_beta)

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.load().syndrome_dlsch_decoder_destroy(h)
            except Exception:
                pass

    def with_pipeline(self, n_workers):
        """:729.  Kept for API parity: the code blocks of a call already decode
        concurrently in one batched GPU launch."""
        _lib.check(_lib.load().syndrome_dlsch_decoder_with_pipeline(self._h, n_workers))
        return self

    def worker_count(self):
        return int(_lib.load().syndrome_dlsch_decoder_worker_count(self._h))

    def num_code_blocks(self):
        return int(_lib.load().syndrome_dlsch_decoder_num_code_blocks(self._h))

    def output_bits(self):
        return int(_lib.load().syndrome_dlsch_decoder_output_bits(self._h))

    def decode(self, rx_llr, rv, tb_out):
        """:829.  rx_llr: C * E f32 LLRs; tb_out (uint8, >= tb_size) receives the TB
        bits when the CRCs pass.  Returns a DecodeReport."""
        rx = np.ascontiguousarray(rx_llr, dtype=np.float32)
        if not (isinstance(tb_out, np.ndarray) and tb_out.dtype == np.uint8 and tb_out.flags.c_contiguous):
            raise TypeError("tb_out must be a C-contiguous uint8 numpy array")
        c = self.num_code_blocks()
        cb = np.zeros(c, np.uint8)
        rep = _Report()
        _lib.check(_lib.load().syndrome_dlsch_decode(self._h, rx.ctypes.data, rx.size, rv, tb_out.ctypes.data,
                                                     tb_out.size, ctypes.byref(rep), cb.ctypes.data, c))
        return DecodeReport(bool(rep.crc_ok), tuple(bool(x) for x in cb), int(rep.max_iters_used),
                            int(rep.harq_tx_count))

    def flush_harq(self):
        _lib.load().syndrome_dlsch_decoder_flush_harq(self._h)
