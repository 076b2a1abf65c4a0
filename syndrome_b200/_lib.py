"""Loads libsyndrome_b200.so and declares the C prototypes of include/syndrome_ldpc.h.

There is no fallback: if the shared library is missing or does not load, every
entry point raises.  Build it with `python -m syndrome_b200.build`."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsyndrome_b200.so")

OK = 0
INVALID_PARAM = -1
CRC_MISMATCH = -2
DECODER_NOT_CONVERGED = -3
BUFFER_TOO_SMALL = -4
NULL_POINTER = -5
PANIC = -6
CUDA_ERROR = -7

PRECISION_INT8 = 0
PRECISION_F32 = 1

_sz = ctypes.c_size_t
_i32 = ctypes.c_int32
_f32 = ctypes.c_float
_vp = ctypes.c_void_p

# name -> (restype, argtypes); mirrors include/syndrome_ldpc.h
PROTOTYPES = {
    "syndrome_ldpc_decoder_create": (_i32, [_i32, _sz, _f32, ctypes.POINTER(_vp)]),
    "syndrome_ldpc_decoder_destroy": (None, [_vp]),
    "syndrome_ldpc_decoder_variable_node_count": (_sz, [_vp]),
    "syndrome_ldpc_decoder_info_bit_count": (_sz, [_vp]),
    "syndrome_ldpc_decoder_required_edge_buffer": (_sz, [_vp]),
    "syndrome_ldpc_decoder_required_layer_buffer": (_sz, [_vp]),
    "syndrome_ldpc_decode_5g": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _sz, _vp]),
    "syndrome_ldpc_encoder_create": (_i32, [_i32, _sz, ctypes.POINTER(_vp)]),
    "syndrome_ldpc_encoder_destroy": (None, [_vp]),
    "syndrome_ldpc_encoder_info_bit_count": (_sz, [_vp]),
    "syndrome_ldpc_encoder_codeword_bit_count": (_sz, [_vp]),
    "syndrome_ldpc_encode_5g": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz]),
    "syndrome_ldpc_decoder_create_wifi": (_i32, [_sz, _sz, _sz, _f32, ctypes.POINTER(_vp)]),
    "syndrome_ldpc_decoder_create_raw": (_i32, [_vp, _vp, _vp, _sz, _sz, _sz, _sz, _f32, ctypes.POINTER(_vp)]),
    "syndrome_ldpc_decoder_check_node_count": (_sz, [_vp]),
    "syndrome_ldpc_decoder_dims": (_i32, [_vp, _vp]),
    "syndrome_ldpc_init_5g_llr": (_i32, [_vp, _vp, _sz, _sz]),
    "syndrome_ldpc_decode": (_i32, [_vp, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _sz, _vp]),
    "syndrome_ldpc_decode_i8": (_i32, [_vp, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _sz, _f32, ctypes.c_int16, _vp]),
    "syndrome_ldpc_decode_5g_i8": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _sz, _f32,
                                          ctypes.c_int16, _vp]),
    "syndrome_ldpc_encoder_create_wifi": (_i32, [_sz, _sz, _sz, ctypes.POINTER(_vp)]),
    "syndrome_ldpc_encode": (_i32, [_vp, _vp, _sz, _vp, _sz]),
    "syndrome_ldpc_encode_batch": (_i32, [_vp, _vp, _sz, _vp, _sz, _sz, _i32]),
    "syndrome_quantize_llr_i16": (None, [_vp, _vp, _sz, _f32]),
    "syndrome_beta_q": (_i32, [_f32, _f32]),
    "syndrome_awgn_llr": (None, [_f32, _f32, ctypes.c_uint64, _vp, _sz, _vp]),
    "syndrome_awgn_quantized_batch": (None, [_vp, _sz, _sz, _sz, _vp, _f32, _vp, _f32, _vp, _sz, _sz, _i32]),
    "syndrome_ldpc_batch_workspace_size": (_sz, [_vp, _i32, _sz]),
    "syndrome_ldpc_decode_batch_i8": (_i32, [_vp, _vp, _sz, _sz, _sz, _i32, _sz, _sz, _f32, ctypes.c_int16,
                                             _vp, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _vp]),
    "syndrome_ldpc_decode_batch_f32": (_i32, [_vp, _vp, _sz, _sz, _sz, _i32, _sz, _sz,
                                              _vp, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _vp]),
    "syndrome_ldpc_decoder_set_kernel": (_i32, [_vp, _i32]),
    "syndrome_ldpc_decode_batch_i8_noalloc": (_i32, [_vp, _vp, _sz, _sz, _sz, _i32, _sz, _sz, _f32, ctypes.c_int16,
                                                     _vp, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz, _vp]),
    "syndrome_mixed_plan_create": (_i32, [_vp, _sz, _f32, _f32, ctypes.c_int16, _sz, _vp, _sz, ctypes.POINTER(_vp)]),
    "syndrome_mixed_plan_destroy": (None, [_vp]),
    "syndrome_mixed_plan_items": (_i32, [_vp, _vp, _sz, ctypes.POINTER(_sz)]),
    "syndrome_mixed_plan_set_kernel": (_i32, [_vp, _i32, ctypes.POINTER(_i32)]),
    "syndrome_mixed_tile_capacity": (_i32, [_i32, _i32]),
    "syndrome_mixed_decode": (_i32, [_vp, _vp, _sz, _vp, _sz, _vp, _sz, _i32, _vp]),
    "syndrome_wifi_mixed_plan_create": (_i32, [_vp, _sz, _f32, _sz, _sz, ctypes.POINTER(_vp)]),
    "syndrome_wifi_mixed_plan_destroy": (None, [_vp]),
    "syndrome_wifi_mixed_plan_chunks": (_i32, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(_sz)]),
    "syndrome_wifi_mixed_decode": (_i32, [_vp, _vp, _sz, _vp, _sz, _vp, _sz, _i32, _vp]),
    "syndrome_tb_segmentation": (_i32, [_sz, _f32, _vp]),
    "syndrome_crc24": (ctypes.c_uint32, [_vp, _sz, _i32]),
    "syndrome_dlsch_encoder_create": (_i32, [_sz, _f32, _sz, _sz, ctypes.POINTER(_vp)]),
    "syndrome_dlsch_encoder_destroy": (None, [_vp]),
    "syndrome_dlsch_encoder_output_bits": (_sz, [_vp]),
    "syndrome_dlsch_encoder_num_code_blocks": (_sz, [_vp]),
    "syndrome_dlsch_encode": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz]),
    "syndrome_serve_create": (_i32, [_vp, ctypes.POINTER(_vp)]),
    "syndrome_serve_destroy": (None, [_vp]),
    "syndrome_serve_submit": (_i32, [_vp, ctypes.c_uint64, _sz, _f32, _sz, _sz, _sz, _vp, _sz, _i32]),
    "syndrome_serve_poll": (_i32, [_vp, _vp, _sz, ctypes.POINTER(_sz), ctypes.c_int64]),
    "syndrome_serve_fetch": (_i32, [_vp, ctypes.c_uint64, _vp, _sz]),
    "syndrome_serve_release": (_i32, [_vp, ctypes.c_uint64]),
    "syndrome_serve_stats": (_i32, [_vp, _vp]),
    "syndrome_serve_core_stats": (_i32, [_vp, _vp]),
    "syndrome_serve_run_load": (_i32, [_vp, _vp, _sz, _vp, _vp, _vp, _sz]),
    "syndrome_wifi_shortening_counts": (_i32, [_sz, _sz, _sz, _sz, ctypes.POINTER(_sz), ctypes.POINTER(_sz)]),
    "syndrome_wifi_encode_shortened": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz]),
    "syndrome_wifi_decode_shortened": (_i32, [_vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _sz, _vp]),
    "syndrome_wifi_decode_shortened_batch_f32": (_i32, [_vp, _vp, _sz, _sz, _sz, _sz, _sz, _vp, _sz, _sz, _vp, _vp,
                                                        _sz, _vp, _sz, _vp, _sz, _vp, _sz, _vp]),
    "syndrome_dlsch_decoder_create": (_i32, [_sz, _f32, _sz, _sz, _sz, _f32, ctypes.POINTER(_vp)]),
    "syndrome_dlsch_decoder_destroy": (None, [_vp]),
    "syndrome_dlsch_decoder_num_code_blocks": (_sz, [_vp]),
    "syndrome_dlsch_decoder_output_bits": (_sz, [_vp]),
    "syndrome_dlsch_decoder_with_pipeline": (_i32, [_vp, _sz]),
    "syndrome_dlsch_decoder_worker_count": (_sz, [_vp]),
    "syndrome_dlsch_decode": (_i32, [_vp, _vp, _sz, _sz, _vp, _sz, _vp, _vp, _sz]),
    "syndrome_dlsch_decoder_flush_harq": (None, [_vp]),
    "syndrome_ldpc_pipeline_create": (_i32, [_vp, _sz, _sz, ctypes.POINTER(_vp)]),
    "syndrome_ldpc_pipeline_destroy": (None, [_vp]),
    "syndrome_ldpc_pipeline_worker_count": (_sz, [_vp]),
    "syndrome_ldpc_pipeline_pool_size": (_sz, [_vp]),
    "syndrome_ldpc_pipeline_acquire": (ctypes.c_int64, [_vp]),
    "syndrome_ldpc_pipeline_submit": (_i32, [_vp, ctypes.c_int64]),
    "syndrome_ldpc_pipeline_try_recv": (ctypes.c_int64, [_vp]),
    "syndrome_ldpc_pipeline_release": (_i32, [_vp, ctypes.c_int64]),
    "syndrome_ldpc_pipeline_frame_llr": (_vp, [_vp, ctypes.c_int64]),
    "syndrome_ldpc_pipeline_frame_hard": (_vp, [_vp, ctypes.c_int64]),
    "syndrome_ldpc_pipeline_frame_iterations": (_sz, [_vp, ctypes.c_int64]),
    "syndrome_ldpc_pipeline_frame_set_tag": (None, [_vp, ctypes.c_int64, _sz]),
    "syndrome_ldpc_pipeline_frame_tag": (_sz, [_vp, ctypes.c_int64]),
    "syndrome_ldpc_encode_batch_device": (_i32, [_vp, _vp, _sz, _vp, _sz, _sz, _vp]),
    "syndrome_serve_set_tiles": (_i32, [_vp, _vp, _sz]),
    "syndrome_last_error": (ctypes.c_char_p, []),
}

_LIB = None


def load():
    """Returns the loaded library; raises OSError if it is not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is not built; run `python -m syndrome_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


class SyndromeError(RuntimeError):
    """A non-zero SyndromeStatus from the library (capi/src/lib.rs:73-94)."""

    NAMES = {INVALID_PARAM: "InvalidParam", CRC_MISMATCH: "CrcMismatch",
             DECODER_NOT_CONVERGED: "DecoderNotConverged", BUFFER_TOO_SMALL: "BufferTooSmall",
             NULL_POINTER: "NullPointer", PANIC: "Panic", CUDA_ERROR: "CudaError"}

    def __init__(self, status, message=""):
        self.status = status
        super().__init__(f"{self.NAMES.get(status, status)}: {message}")


def check(status):
    if status != OK:
        msg = load().syndrome_last_error()
        raise SyndromeError(status, msg.decode() if msg else "")
    return status
