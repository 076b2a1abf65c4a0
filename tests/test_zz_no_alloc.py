"""The allocation-free entry point, syndrome_ldpc_decode_batch_i8_noalloc.

It exists for callers that cannot allocate device memory while decoding (a
baseband thread under a per-slot deadline, a plug-in whose host owns every device
allocation).  When the caller asks for no message output, the kernel keeps its
check-to-variable messages in a static device array shared by every call; this test
checks, through the C ABI, that two calls in a row on different inputs (the second
one running on the array the first one left behind) give exactly what the
workspace-based entry point gives.  BG1 Z=384 with 600 codewords needs more CTAs
than the array holds slots for (33,554,432 / 121,344 = 276), so the launch is capped
and each CTA walks several groups through the same slot.  With a message output the
kernel writes the messages there instead; that case is checked too.  These shapes are
5G NR graphs, on which the entry runs the decoder's own kernel choice (the NR kernels
keep their state on chip and need no scratch): the static array is exercised with the
generic kernel chosen, and the default choice is checked as well.
Collected last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402
from syndrome_b200 import _lib  # noqa: E402


def make_llr(bg, z, count, ebno, seed):
    enc = S.QcLdpcEncoder.new(bg, z)
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, size=(count, enc.info_bit_count()), dtype=np.uint8)
    cw = enc.encode_batch(info, threads=4)
    rate = enc.info_bit_count() / (enc.codeword_bit_count() - 2 * z)
    return S.awgn_quantized_batch(cw, ebno, rate, seed + np.arange(count), tx_begin=2 * z, threads=4)


def noalloc_call(dec, llr, iters, quant, hard_bits, with_messages):
    """One call of the allocation-free entry.  Without a message output (edge_r NULL)
    the messages live in the static scratch array."""
    b, n = llr.shape[0], dec.variable_node_count()
    dev = llr.device
    out = dict(packed=torch.zeros((b, (hard_bits + 31) // 32), dtype=torch.int32, device=dev),
               iters=torch.zeros((b,), dtype=torch.int32, device=dev),
               app=torch.zeros((b, n), dtype=torch.int16, device=dev),
               hard=torch.zeros((b, n), dtype=torch.uint8, device=dev))
    if with_messages:
        out["edge_r"] = torch.zeros((b, dec.required_edge_buffer()), dtype=torch.int8, device=dev)
    er = out["edge_r"].data_ptr() if with_messages else None
    er_stride = dec.required_edge_buffer() if with_messages else 0
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = _lib.load().syndrome_ldpc_decode_batch_i8_noalloc(
        dec._h, llr.data_ptr(), llr.stride(0), 2 * dec.z, b, 1, 0, iters, quant.scale, quant.app_clamp,
        out["packed"].data_ptr(), hard_bits, out["packed"].stride(0), out["iters"].data_ptr(),
        out["app"].data_ptr(), n, er, er_stride, out["hard"].data_ptr(), n, ctypes.c_void_p(stream))
    _lib.check(st)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("kernel", ["generic", "auto"])
@pytest.mark.parametrize("with_messages", [False, True], ids=["scratch", "messages_out"])
@pytest.mark.parametrize("bg,z,count", [(0, 384, 600), (1, 52, 150)])
def test_noalloc_matches_workspace_entry_point_on_two_calls(bg, z, count, with_messages, kernel):
    dec = S.QcLdpcDecoder.with_lifting_size(bg, z, 0.5).set_kernel(kernel)
    quant = S.QuantParams()
    hard_bits = dec.info_bit_count_5g()
    for call, (ebno, seed) in enumerate(((1.0, 11), (2.0, 12345))):
        llr = torch.from_numpy(make_llr(bg, z, count, ebno, seed)).cuda()
        ref = dec.decode_batch_i8(llr, 8, llr_offset=2 * z, nr_prologue=True, quant=quant, hard_bits=hard_bits,
                                  want_app=True, want_edge_r=with_messages, want_hard=True)
        got = noalloc_call(dec, llr, 8, quant, hard_bits, with_messages)
        # Bit-exact, the tolerance of every int8 test in this suite.
        assert torch.equal(got["iters"], ref.iters), f"call {call}: iterations differ"
        assert torch.equal(got["packed"], ref.hard_packed), f"call {call}: packed hard decisions differ"
        assert torch.equal(got["app"], ref.app), f"call {call}: posteriors differ"
        assert torch.equal(got["hard"], ref.hard), f"call {call}: hard decisions differ"
        if with_messages:
            assert torch.equal(got["edge_r"], ref.edge_r), f"call {call}: messages differ"
