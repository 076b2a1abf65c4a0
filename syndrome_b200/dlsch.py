"""5G NR transport blocks (DL-SCH): segmentation, CRC-24A/B and the transport-block
encoder, mirroring syndrome's segmentation.rs (compute_segmentation), crc.rs (Crc24)
and transport_block.rs (DlSchEncoder).  The decode side is the device-resident
serving engine (serve.py)."""
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
