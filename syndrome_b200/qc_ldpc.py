"""Python mirror of syndrome's QC-LDPC decoder API (src/qc_ldpc.rs,
src/wifi_ldpc_tables.rs, src/quantize.rs), backed by the B200 library through
its C ABI.  Method names, argument order and error behaviour follow the
reference: buffers are caller-owned numpy arrays updated in place, wrong lengths
raise FecError(InvalidParam) and short scratch buffers FecError(BufferTooSmall).

The batched methods (decode_batch_i8 / decode_batch_f32) are this library's
GPU-native path: torch CUDA tensors in and out, one launch for many codewords.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import SyndromeError as FecError

DEFAULT_SCALE = 8.0          # src/quantize.rs:182
MSG_MAX = 127                # src/quantize.rs:190
APP_CLAMP_I8 = 127           # src/quantize.rs:194
APP_CLAMP_WIDE = 32767       # src/quantize.rs:205


class BaseGraph:
    Bg1 = 0
    Bg2 = 1


class QuantParams:
    """Fixed-point format (src/quantize.rs:217-305)."""

    def __init__(self, scale=DEFAULT_SCALE, app_clamp=APP_CLAMP_WIDE):
        self.scale = float(scale)
        self.app_clamp = int(app_clamp)

    def with_scale(self, scale):
        return QuantParams(scale, self.app_clamp)

    def with_app_clamp(self, app_clamp):
        return QuantParams(self.scale, app_clamp)

    def beta_q(self, offset_beta):
        return int(_lib.load().syndrome_beta_q(offset_beta, self.scale))


def quantize_llr_i16(llr, out=None, scale=DEFAULT_SCALE):
    """src/quantize.rs:331: clamp(round_half_away(llr * scale), +-127), NaN -> 0."""
    llr = np.ascontiguousarray(llr, dtype=np.float32)
    if out is None:
        out = np.empty(llr.size, dtype=np.int16)
    assert out.dtype == np.int16 and out.flags.c_contiguous and out.size == llr.size
    _lib.load().syndrome_quantize_llr_i16(llr.ctypes.data, out.ctypes.data, llr.size, scale)
    return out


def _buf(a, dtype, name):
    if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous or not a.flags.writeable:
        raise TypeError(f"{name} must be a writable C-contiguous numpy array of {np.dtype(dtype).name}")
    return a.ctypes.data, a.size


class LdpcWorkspace:
    """Owning buffer bundle (src/qc_ldpc.rs:1919-1963)."""

    def __init__(self, n, edge, layer, dtype=np.float32):
        self.codeword_llr = np.zeros(n, dtype=dtype)
        self.edge_r = np.zeros(edge, dtype=dtype)
        self.layer_scratch = np.zeros(layer, dtype=dtype)
        self.hard = np.zeros(n, dtype=np.uint8)

    def hard_output(self):
        return self.hard

    def posterior_llr(self):
        return self.codeword_llr


class BatchResult:
    """Device outputs of one batched decode (torch tensors)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


class QcLdpcDecoder:
    """Layered offset min-sum decoder on the GPU (reference: src/qc_ldpc.rs:481)."""

    def __init__(self, handle, offset_beta):
        self._h = handle
        self.offset_beta = float(offset_beta)
        L = _lib.load()
        dims = (ctypes.c_size_t * 5)()
        _lib.check(L.syndrome_ldpc_decoder_dims(self._h, dims))
        self.z, self.num_row_blocks, self.num_col_blocks, self.edge_count, self.max_layer_degree = [int(x) for x in dims]
        self._ws = {}

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.load().syndrome_ldpc_decoder_destroy(h)
            except Exception:
                pass

    # ---- construction (src/qc_ldpc.rs:517-580, src/wifi_ldpc_tables.rs:521) ----
    @classmethod
    def new(cls, base_graph, offset_beta):
        return cls.with_lifting_size(base_graph, 384 if base_graph == BaseGraph.Bg1 else 128, offset_beta)

    @classmethod
    def with_lifting_size(cls, base_graph, z, offset_beta):
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_ldpc_decoder_create(int(base_graph), int(z), offset_beta, ctypes.byref(h)))
        return cls(h.value, offset_beta)

    @classmethod
    def from_raw_edges(cls, entries, num_row_blocks, num_col_blocks, z, offset_beta):
        e = np.asarray(entries, dtype=np.int64).reshape(-1, 3)
        r = np.ascontiguousarray(e[:, 0], dtype=np.uint8)
        c = np.ascontiguousarray(e[:, 1], dtype=np.uint8)
        s = np.ascontiguousarray(e[:, 2], dtype=np.int16)
        if np.any(e[:, :2] < 0) or np.any(e[:, :2] > 255):
            raise FecError(_lib.INVALID_PARAM, "raw edge row/col out of range")
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_ldpc_decoder_create_raw(
            r.ctypes.data, c.ctypes.data, s.ctypes.data, len(e), num_row_blocks, num_col_blocks, z,
            offset_beta, ctypes.byref(h)))
        return cls(h.value, offset_beta)

    # ---- sizing (src/qc_ldpc.rs:582-601, 736) ----
    def variable_node_count(self):
        return int(_lib.load().syndrome_ldpc_decoder_variable_node_count(self._h))

    def check_node_count(self):
        return int(_lib.load().syndrome_ldpc_decoder_check_node_count(self._h))

    def required_edge_buffer(self):
        return int(_lib.load().syndrome_ldpc_decoder_required_edge_buffer(self._h))

    def required_layer_buffer(self):
        return int(_lib.load().syndrome_ldpc_decoder_required_layer_buffer(self._h))

    def info_bit_count_5g(self):
        return int(_lib.load().syndrome_ldpc_decoder_info_bit_count(self._h))

    def workspace(self, dtype=np.float32):
        return LdpcWorkspace(self.variable_node_count(), self.required_edge_buffer(),
                             self.required_layer_buffer(), dtype)

    # ---- f32 decode (src/qc_ldpc.rs:644-874) ----
    def init_5g_llr(self, llr, n_filler):
        p, n = _buf(llr, np.float32, "llr")
        _lib.check(_lib.load().syndrome_ldpc_init_5g_llr(self._h, p, n, n_filler))

    def decode_layered_offset_min_sum(self, llr, edge_r, layer_scratch, hard_output, iterations):
        used = ctypes.c_size_t(0)
        args = [*_buf(llr, np.float32, "llr"), *_buf(edge_r, np.float32, "edge_r"),
                *_buf(layer_scratch, np.float32, "layer_scratch"), *_buf(hard_output, np.uint8, "hard_output")]
        _lib.check(_lib.load().syndrome_ldpc_decode(self._h, *args, iterations, ctypes.byref(used)))
        return used.value

    def decode_5g(self, llr, n_filler, edge_r, layer_scratch, hard_output, iterations):
        used = ctypes.c_size_t(0)
        lp, ln = _buf(llr, np.float32, "llr")
        args = [*_buf(edge_r, np.float32, "edge_r"), *_buf(layer_scratch, np.float32, "layer_scratch"),
                *_buf(hard_output, np.uint8, "hard_output")]
        _lib.check(_lib.load().syndrome_ldpc_decode_5g(self._h, lp, ln, n_filler, *args, iterations,
                                                       ctypes.byref(used)))
        return used.value

    def decode_with_workspace(self, llr, workspace, iterations):
        """src/qc_ldpc.rs:1851-1862: the posterior stays in the caller's llr, the hard
        decisions land in workspace.hard_output(); workspace.codeword_llr is left
        untouched (it is the staging buffer of reconstruction-style decodes,
        :1951-1954).  A workspace built for a different code fails the decode's size
        checks (BUFFER_TOO_SMALL or INVALID_PARAM), as in :2765-2783."""
        return self.decode_layered_offset_min_sum(llr, workspace.edge_r, workspace.layer_scratch, workspace.hard,
                                                  iterations)

    def decode_5g_with_workspace(self, llr, n_filler, workspace, iterations):
        """src/qc_ldpc.rs:1887-1903 (decode_5g over the workspace's buffers)."""
        return self.decode_5g(llr, n_filler, workspace.edge_r, workspace.layer_scratch, workspace.hard, iterations)

    # ---- int8 decode (src/qc_ldpc.rs:1345-1524) ----
    def decode_layered_offset_min_sum_i8(self, app, edge_r, layer_scratch, hard_output, iterations,
                                         quant=None):
        quant = quant or QuantParams()
        used = ctypes.c_size_t(0)
        args = [*_buf(app, np.int16, "app"), *_buf(edge_r, np.int8, "edge_r"),
                *_buf(layer_scratch, np.int8, "layer_scratch"), *_buf(hard_output, np.uint8, "hard_output")]
        _lib.check(_lib.load().syndrome_ldpc_decode_i8(self._h, *args, iterations, quant.scale,
                                                       quant.app_clamp, ctypes.byref(used)))
        return used.value

    def decode_5g_i8(self, app, n_filler, edge_r, layer_scratch, hard_output, iterations, quant=None):
        quant = quant or QuantParams()
        used = ctypes.c_size_t(0)
        ap, an = _buf(app, np.int16, "app")
        args = [*_buf(edge_r, np.int8, "edge_r"), *_buf(layer_scratch, np.int8, "layer_scratch"),
                *_buf(hard_output, np.uint8, "hard_output")]
        _lib.check(_lib.load().syndrome_ldpc_decode_5g_i8(self._h, ap, an, n_filler, *args, iterations,
                                                          quant.scale, quant.app_clamp, ctypes.byref(used)))
        return used.value

    # ---- batched GPU API (no reference counterpart) ----
    KERNELS = {"auto": 0, "generic": 1, "nr": 2, "pair": 3, "generic_global": 4, "pair_smem": 5}

    def set_kernel(self, kernel):
        """Kernel used by batch decodes: "auto", "generic" (layered, any graph; messages
        compressed in shared memory where they fit), "generic_global" (the same with its
        messages in global memory), "nr" (5G NR specialised, one codeword per thread),
        "pair" (5G NR, two codewords per 32-bit word; at Z = 384 most check-row state in
        tensor memory, two codeword pairs per SM) or "pair_smem" (the paired kernel with
        all its state in shared memory, one pair per SM)."""
        _lib.check(_lib.load().syndrome_ldpc_decoder_set_kernel(self._h, self.KERNELS[kernel]))
        return self

    def batch_workspace_size(self, batch, precision="int8"):
        p = _lib.PRECISION_F32 if precision == "f32" else _lib.PRECISION_INT8
        return int(_lib.load().syndrome_ldpc_batch_workspace_size(self._h, p, batch))

    def _batch(self, kind, llr, iterations, llr_offset, nr_prologue, n_filler, quant, hard_bits,
               want_app, want_edge_r, want_hard, workspace, stream, out):
        import torch

        if not (isinstance(llr, torch.Tensor) and llr.is_cuda and llr.dim() == 2):
            raise TypeError("llr must be a 2-D CUDA tensor [batch, stride]")
        if llr.stride(1) != 1:
            raise TypeError("llr rows must be contiguous")
        want_dtype = torch.float32 if kind == "f32" else (torch.int8, torch.int16)
        if (kind == "f32" and llr.dtype != torch.float32) or (kind == "i8" and llr.dtype not in want_dtype):
            raise TypeError(f"llr dtype {llr.dtype} not accepted by decode_batch_{kind}")
        dev = llr.device
        n = self.variable_node_count()
        b = llr.shape[0]
        hard_bits = n if hard_bits is None else int(hard_bits)
        words = (hard_bits + 31) // 32
        out = out or {}
        packed = out.get("hard_packed")
        if packed is None:
            packed = torch.empty((b, max(words, 1)), dtype=torch.int32, device=dev)
        iters = out.get("iters")
        if iters is None:
            iters = torch.empty((b,), dtype=torch.int32, device=dev)
        app = edge_r = hard = None
        app_dtype = torch.float32 if kind == "f32" else torch.int16
        edge_dtype = torch.float32 if kind == "f32" else torch.int8
        if want_app:
            app = out.get("app") if out.get("app") is not None else torch.empty((b, n), dtype=app_dtype, device=dev)
        if want_edge_r:
            edge_r = torch.empty((b, self.required_edge_buffer()), dtype=edge_dtype, device=dev)
        if want_hard:
            hard = torch.empty((b, n), dtype=torch.uint8, device=dev)
        # f32: a workspace also when the messages go to edge_r (the 5G NR Z=384 kernel keeps
        # its extension-column posteriors there)
        if workspace is None and (edge_r is None or kind == "f32"):
            need = self.batch_workspace_size(b, "f32" if kind == "f32" else "int8")
            workspace = self._ws.get((dev, kind))
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty((max(need, 1),), dtype=torch.uint8, device=dev)
                self._ws[(dev, kind)] = workspace
        ws_ptr = workspace.data_ptr() if workspace is not None else None
        ws_bytes = workspace.numel() * workspace.element_size() if workspace is not None else 0
        if stream is None:
            stream = torch.cuda.current_stream(dev)
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        L = _lib.load()

        def p(t):
            return t.data_ptr() if t is not None else None

        if llr.shape[1] < n - llr_offset:
            raise FecError(_lib.INVALID_PARAM, f"llr rows hold {llr.shape[1]} values, need {n - llr_offset}")
        # a size-1 leading dimension may carry any stride; the row length is what matters then
        common = dict(stride=llr.stride(0) if b > 1 else llr.shape[1])
        if kind == "i8":
            if llr.dtype == torch.int16:
                raise TypeError("decode_batch_i8 takes int8 channel LLRs; use the host API for int16 posteriors")
            st = L.syndrome_ldpc_decode_batch_i8(
                self._h, llr.data_ptr(), common["stride"], llr_offset, b, int(bool(nr_prologue)), n_filler,
                iterations, quant.scale, quant.app_clamp, p(packed), hard_bits, packed.stride(0), p(iters),
                p(app), n, p(edge_r), self.required_edge_buffer(), p(hard), n, ws_ptr, ws_bytes, sp)
        else:
            st = L.syndrome_ldpc_decode_batch_f32(
                self._h, llr.data_ptr(), common["stride"], llr_offset, b, int(bool(nr_prologue)), n_filler,
                iterations, p(packed), hard_bits, packed.stride(0), p(iters), p(app), n, p(edge_r),
                self.required_edge_buffer(), p(hard), n, ws_ptr, ws_bytes, sp)
        _lib.check(st)
        return BatchResult(hard_packed=packed, hard_bits=hard_bits, iters=iters, app=app, edge_r=edge_r, hard=hard)

    def decode_batch_i8(self, llr, iterations, *, llr_offset=0, nr_prologue=False, n_filler=0, quant=None,
                        hard_bits=None, want_app=False, want_edge_r=False, want_hard=False, workspace=None,
                        stream=None, out=None):
        """Decodes int8 channel LLRs llr[b, j] (variable llr_offset + j) of a batch
        of codewords with the int8 LOMS kernel.  With nr_prologue the decode_5g_i8
        initialisation is applied (filler = app_clamp, [0, 2Z) = 0)."""
        return self._batch("i8", llr, iterations, llr_offset, nr_prologue, n_filler, quant or QuantParams(),
                           hard_bits, want_app, want_edge_r, want_hard, workspace, stream, out)

    def decode_batch_f32(self, llr, iterations, *, llr_offset=0, nr_prologue=False, n_filler=0,
                         hard_bits=None, want_app=False, want_edge_r=False, want_hard=False, workspace=None,
                         stream=None, out=None):
        """Batched f32 LOMS (decode_layered_offset_min_sum / decode_5g semantics)."""
        return self._batch("f32", llr, iterations, llr_offset, nr_prologue, n_filler, None,
                           hard_bits, want_app, want_edge_r, want_hard, workspace, stream, out)


def wifi_ldpc_decoder(z, rate_num, rate_den, offset_beta):
    """src/wifi_ldpc_tables.rs:521."""
    h = ctypes.c_void_p()
    _lib.check(_lib.load().syndrome_ldpc_decoder_create_wifi(z, rate_num, rate_den, offset_beta, ctypes.byref(h)))
    return QcLdpcDecoder(h.value, offset_beta)


class QcLdpcEncoder:
    """Systematic encoder (src/qc_ldpc.rs:2408-2618); runs on the host."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.load().syndrome_ldpc_encoder_destroy(h)
            except Exception:
                pass

    @classmethod
    def new(cls, base_graph, z):
        h = ctypes.c_void_p()
        _lib.check(_lib.load().syndrome_ldpc_encoder_create(int(base_graph), int(z), ctypes.byref(h)))
        return cls(h.value)

    def info_bit_count(self):
        return int(_lib.load().syndrome_ldpc_encoder_info_bit_count(self._h))

    def codeword_bit_count(self):
        return int(_lib.load().syndrome_ldpc_encoder_codeword_bit_count(self._h))

    def encode(self, info_bits, codeword):
        info = np.ascontiguousarray(info_bits, dtype=np.uint8)
        cp, cn = _buf(codeword, np.uint8, "codeword")
        _lib.check(_lib.load().syndrome_ldpc_encode(self._h, info.ctypes.data, info.size, cp, cn))

    def encode_5g(self, info_bits, n_filler, codeword):
        info = np.ascontiguousarray(info_bits, dtype=np.uint8)
        cp, cn = _buf(codeword, np.uint8, "codeword")
        _lib.check(_lib.load().syndrome_ldpc_encode_5g(self._h, info.ctypes.data, info.size, n_filler, cp, cn))

    def encode_batch(self, info_bits, threads=0):
        """info_bits uint8 [count, K] -> codewords uint8 [count, N] (host threads)."""
        info = np.ascontiguousarray(info_bits, dtype=np.uint8)
        count, k = info.shape
        cw = np.empty((count, self.codeword_bit_count()), dtype=np.uint8)
        _lib.check(_lib.load().syndrome_ldpc_encode_batch(self._h, info.ctypes.data, k, cw.ctypes.data,
                                                          cw.shape[1], count, threads))
        return cw


    def encode_batch_device(self, info_bits, stream=None):
        """info_bits: uint8 CUDA tensor [count, K] (one bit per byte) -> uint8 CUDA
        tensor [count, N] of codewords, encoded on the GPU (same codewords as
        encode_batch)."""
        import torch

        if not (isinstance(info_bits, torch.Tensor) and info_bits.is_cuda and info_bits.dim() == 2
                and info_bits.dtype == torch.uint8 and info_bits.stride(1) == 1):
            raise TypeError("info_bits must be a 2-D uint8 CUDA tensor with contiguous rows")
        count = info_bits.shape[0]
        cw = torch.empty((count, self.codeword_bit_count()), dtype=torch.uint8, device=info_bits.device)
        if stream is None:
            stream = torch.cuda.current_stream(info_bits.device)
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        stride = info_bits.stride(0) if count > 1 else info_bits.shape[1]
        _lib.check(_lib.load().syndrome_ldpc_encode_batch_device(self._h, info_bits.data_ptr(), stride,
                                                                 cw.data_ptr(), cw.shape[1], count, sp))
        return cw


def wifi_ldpc_encoder(z, rate_num, rate_den):
    """src/wifi_ldpc_tables.rs:490."""
    h = ctypes.c_void_p()
    _lib.check(_lib.load().syndrome_ldpc_encoder_create_wifi(z, rate_num, rate_den, ctypes.byref(h)))
    return QcLdpcEncoder(h.value)


class AwgnChannel:
    """BPSK over AWGN (src/channel_sim.rs:108-221).  Like the reference, the noise
    stream starts from splitmix64(seed); each transmit() continues the stream by
    regenerating it from the start and skipping the symbols already sent."""

    def __init__(self, ebno_db, code_rate, seed):
        self.ebno_db = float(ebno_db)
        self.code_rate = float(code_rate)
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self._sent = 0

    def transmit(self, coded_bits):
        bits = np.ascontiguousarray(coded_bits, dtype=np.uint8)
        total = np.zeros(self._sent + bits.size, dtype=np.uint8)
        total[self._sent:] = bits
        out = np.empty(total.size, dtype=np.float32)
        _lib.load().syndrome_awgn_llr(self.ebno_db, self.code_rate, self.seed, total.ctypes.data, total.size,
                                      out.ctypes.data)
        self._sent = total.size
        return out[total.size - bits.size:]


def awgn_quantized_batch(codewords, ebno_db, code_rate, seeds, scale=DEFAULT_SCALE, tx_begin=0, threads=0):
    """Rows of uint8 codewords [count, N] -> int8 LLRs [count, N - tx_begin] (host threads)."""
    cw = np.ascontiguousarray(codewords, dtype=np.uint8)
    count, n = cw.shape
    eb = np.ascontiguousarray(np.broadcast_to(np.asarray(ebno_db, dtype=np.float32), (count,)))
    sd = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64).reshape(count))
    out = np.empty((count, n - tx_begin), dtype=np.int8)
    _lib.load().syndrome_awgn_quantized_batch(cw.ctypes.data, n, n, tx_begin, eb.ctypes.data, code_rate,
                                              sd.ctypes.data, scale, out.ctypes.data, out.shape[1], count, threads)
    return out
