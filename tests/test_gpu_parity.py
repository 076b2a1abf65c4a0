"""Parity of the CUDA decoder with the oracle (the CPU restatement of the
reference's decoder) on identical seeded inputs.

int8 path: iterations used, final posterior, final C->V messages and hard
decisions must be bit-identical (the reference's own bar for its AVX2 kernel,
tests/ldpc_int8_kernel_equivalence.rs:140).  f32 path: iterations and hard
decisions bit-identical; posteriors and messages within 1e-5 relative
(F32_RTOL), the contract tolerance; the kernel is expected to be exact and the
tests report how many values differ at all."""
import json
import os

import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402
from syndrome_b200 import _lib  # noqa: E402

F32_RTOL = 1e-5
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def codewords(code, count, ebno, seed):
    """Encoded random codewords and their channel LLRs (oracle encoder + channel)."""
    rate = code.k / code.n
    cws, llrs = [], []
    for i in range(count):
        s = seed + 7919 * i
        cw = code.encode(O.random_bits(s ^ 0xA5A5A5A5, code.k))
        cws.append(cw)
        llrs.append(O.awgn(cw, ebno, rate, s))
    return np.stack(cws), np.stack(llrs)


def oracle_i8(code, apps, beta_q, iters, app_clamp=32767):
    return [code.decode_i8(a, beta_q, iters, app_clamp) for a in apps]


def gpu_i8(dec, llr_i8, iters, quant, kernel="auto", **kw):
    t = torch.from_numpy(np.ascontiguousarray(llr_i8)).cuda()
    dec.set_kernel(kernel)
    r = dec.decode_batch_i8(t, iters, quant=quant, want_app=True, want_edge_r=True, want_hard=True, **kw)
    torch.cuda.synchronize()
    return r


KERNELS = ["generic", "generic_global", "nr", "pair", "pair_smem"]


def assert_i8_equal(label, ref, r):
    it = r.iters.cpu().numpy()
    app = r.app.cpu().numpy()
    er = r.edge_r.cpu().numpy()
    hard = r.hard.cpu().numpy()
    for b, o in enumerate(ref):
        assert it[b] == o["iters"], f"{label} cw{b}: iterations {it[b]} != {o['iters']}"
        d = np.nonzero(app[b] != o["app"])[0]
        assert d.size == 0, f"{label} cw{b}: posterior differs at {d[:5]} ({d.size} of {app.shape[1]})"
        d = np.nonzero(er[b] != o["edge_r"])[0]
        assert d.size == 0, f"{label} cw{b}: C->V message differs at {d[:5]}"
        assert np.array_equal(hard[b], o["hard"]), f"{label} cw{b}: hard decisions differ"
    packed = r.hard_packed.cpu().numpy().view(np.uint32)
    bits = np.unpackbits(packed.view(np.uint8), axis=1, bitorder="little")[:, : r.hard_bits]
    assert np.array_equal(bits, hard[:, : r.hard_bits]), f"{label}: packed hard bits differ"


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("bg,z", [(0, 2), (0, 7), (0, 44), (0, 96), (1, 13), (1, 52), (1, 128), (1, 384)])
def test_int8_3gpp_graphs(bg, z, kernel):
    """tests/ldpc_int8_kernel_equivalence.rs:172-200 (12 iterations, beta 0.5, scale 8)."""
    code = O.Code.nr(bg, z)
    dec = S.QcLdpcDecoder.with_lifting_size(bg, z, 0.5)
    q = S.QuantParams()
    for ebno in (0.0, 1.5, 4.0):
        _, llr = codewords(code, 4, ebno, 0x10000 ^ (z << 8))
        apps = np.stack([O.quantize_i16(x) for x in llr])
        ref = oracle_i8(code, apps, O.beta_q(0.5), 12)
        r = gpu_i8(dec, apps.astype(np.int8), 12, q, kernel)
        assert_i8_equal(f"bg{bg + 1} z{z} {ebno}dB {kernel}", ref, r)


@pytest.mark.parametrize("kernel", KERNELS)
def test_int8_bg1_z384(kernel):
    """tests/ldpc_int8_kernel_equivalence.rs:202-215 (BG1 Z=384 at 1 dB)."""
    code = O.Code.nr(0, 384)
    dec = S.QcLdpcDecoder.with_lifting_size(0, 384, 0.5)
    _, llr = codewords(code, 3, 1.0, 0x03840000)
    apps = np.stack([O.quantize_i16(x) for x in llr])
    r = gpu_i8(dec, apps.astype(np.int8), 12, S.QuantParams(), kernel)
    assert_i8_equal(f"bg1 z384 {kernel}", oracle_i8(code, apps, 4, 12), r)


@pytest.mark.parametrize("kernel", KERNELS)
def test_int8_nr_punctured_filler_and_clamps(kernel):
    """5G input without the punctured columns, filler bits, and clamps on both sides of
    the bounds the 5G NR kernel relies on (255 and 3938)."""
    for bg, z, n_filler in ((0, 64, 100), (1, 96, 3 * 96 // 2), (0, 384, 0)):
        code = O.Code.nr(bg, z)
        dec = S.QcLdpcDecoder.with_lifting_size(bg, z, 0.5)
        info_len = code.k - n_filler
        if kernel in ("pair", "pair_smem"):  # the paired kernel needs app_clamp >= 3938 (7874 with filler bits)
            clamps = (32767, 7874 if n_filler else 3938)
        else:
            clamps = (32767, 1000, 255)
        for clamp in clamps:
            rows, refs = [], []
            for i in range(3):
                info = np.concatenate([O.random_bits(50 + i, info_len), np.zeros(n_filler, np.uint8)])
                cw = code.encode(info)
                app = O.quantize_i16(O.awgn(cw, 1.0 + i, code.k / code.n, 7 + 31 * i))
                rows.append(app[2 * z:].astype(np.int8))
                full = np.concatenate([np.zeros(2 * z, np.int16), app[2 * z:]])
                refs.append(code.decode_i8(code.prologue_5g_i8(full, n_filler, clamp), 4, 10, clamp))
            r = gpu_i8(dec, np.stack(rows), 10, S.QuantParams().with_app_clamp(clamp), kernel, llr_offset=2 * z,
                       nr_prologue=True, n_filler=n_filler, hard_bits=code.k - n_filler)
            assert_i8_equal(f"bg{bg + 1} z{z} filler{n_filler} clamp{clamp} {kernel}", refs, r)


def test_int8_nr_kernel_rejects_what_it_cannot_serve():
    dec = S.QcLdpcDecoder.with_lifting_size(1, 16, 0.5).set_kernel("nr")
    t = torch.zeros((2, dec.variable_node_count()), dtype=torch.int8, device="cuda")
    with pytest.raises(S.FecError) as e:
        dec.decode_batch_i8(t, 5, quant=S.QuantParams().with_app_clamp(127))
    assert e.value.status == _lib.INVALID_PARAM
    w = S.wifi_ldpc_decoder(27, 1, 2, 0.5).set_kernel("nr")
    with pytest.raises(S.FecError):
        w.decode_batch_i8(torch.zeros((1, w.variable_node_count()), dtype=torch.int8, device="cuda"), 5)


def test_int8_pair_kernel_rejects_small_clamps():
    dec = S.QcLdpcDecoder.with_lifting_size(0, 32, 0.5).set_kernel("pair")
    n = dec.variable_node_count()
    t = torch.zeros((3, n), dtype=torch.int8, device="cuda")
    with pytest.raises(S.FecError) as e:
        dec.decode_batch_i8(t, 5, quant=S.QuantParams().with_app_clamp(3937))
    assert e.value.status == _lib.INVALID_PARAM
    with pytest.raises(S.FecError) as e:
        dec.decode_batch_i8(t[:, 64:], 5, llr_offset=64, nr_prologue=True, n_filler=40,
                            quant=S.QuantParams().with_app_clamp(7873))
    assert e.value.status == _lib.INVALID_PARAM
    dec.decode_batch_i8(t, 5, quant=S.QuantParams().with_app_clamp(3938))
    torch.cuda.synchronize()


@pytest.mark.parametrize("count", [1, 2, 5, 16])
def test_int8_pair_kernel_lanes_finish_apart(count):
    """Codewords of one pair converge at different iterations (SNR spread over the batch),
    odd batch sizes leave a lane without a codeword; BG1 Z=384 takes the compile-time-Z
    instantiations (state in tensor memory, and all in shared memory), Z=192 the
    run-time one with two pairs per CTA."""
    for z, kernel in ((384, "pair"), (384, "pair_smem"), (192, "pair")):
        code = O.Code.nr(0, z)
        dec = S.QcLdpcDecoder.with_lifting_size(0, z, 0.5)
        rows, refs = [], []
        for i in range(count):
            info = O.random_bits(900 + i, code.k)
            cw = code.encode(info)
            app = O.quantize_i16(O.awgn(cw, -0.5 + 0.4 * i, code.k / code.n, 1000 + 13 * i))
            rows.append(app[2 * z:].astype(np.int8))
            full = np.concatenate([np.zeros(2 * z, np.int16), app[2 * z:]])
            refs.append(code.decode_i8(code.prologue_5g_i8(full, 0), 4, 8))
        r = gpu_i8(dec, np.stack(rows), 8, S.QuantParams(), kernel, llr_offset=2 * z, nr_prologue=True,
                   hard_bits=code.k)
        assert_i8_equal(f"{kernel} z{z} count{count}", refs, r)


@pytest.mark.parametrize("kernel", ["auto", "generic_global"])
def test_int8_wifi_matrices(kernel):
    """tests/ldpc_int8_kernel_equivalence.rs:217-236 (auto: messages compressed in
    shared memory; generic_global: in global memory)."""
    for z, rn, rd in ((27, 1, 2), (54, 2, 3), (81, 5, 6), (27, 3, 4), (81, 1, 2)):
        code = O.Code.wifi(z, rn, rd)
        dec = S.wifi_ldpc_decoder(z, rn, rd, 0.5).set_kernel(kernel)
        for ebno in (1.0, 3.0):
            _, llr = codewords(code, 5, ebno, 0x01F10000 ^ (z << 4) ^ rd)
            apps = np.stack([O.quantize_i16(x) for x in llr])
            ref = oracle_i8(code, apps, 4, 12)
            assert_i8_equal(f"wifi {z} {rn}/{rd}", ref, gpu_i8(dec, apps.astype(np.int8), 12, S.QuantParams()))


def test_int8_clamped_posterior_and_offsets():
    """:238-277: APP_CLAMP_I8, beta = 0 and a saturating beta (beta_q = 127)."""
    cases = [((0, 44), 0.5, S.APP_CLAMP_I8), ((1, 88), 0.5, S.APP_CLAMP_I8), ((0, 60), 0.0, 32767),
             ((1, 104), 16.0, 32767)]
    for (bg, z), beta, clamp in cases:
        code = O.Code.nr(bg, z)
        dec = S.QcLdpcDecoder.with_lifting_size(bg, z, beta)
        q = S.QuantParams().with_app_clamp(clamp)
        _, llr = codewords(code, 3, 1.0, 0x0C1A0000 + z)
        apps = np.stack([O.quantize_i16(x) for x in llr])
        ref = oracle_i8(code, apps, O.beta_q(beta), 12, clamp)
        assert_i8_equal(f"bg{bg + 1} z{z} beta{beta} clamp{clamp}", ref, gpu_i8(dec, apps.astype(np.int8), 12, q))


def test_int8_5g_prologue_with_filler():
    """:279-343: decode_5g_i8 with n_filler = 3Z/2, input without the punctured columns."""
    z = 60
    code = O.Code.nr(0, z)
    dec = S.QcLdpcDecoder.with_lifting_size(0, z, 0.5)
    n = code.n
    llr = np.where(np.arange(n) % 5 == 0, -0.75, 1.25).astype(np.float32)
    app0 = O.quantize_i16(llr)
    n_filler = 3 * z // 2
    for clamp in (32767, 127):
        ref = code.decode_i8(code.prologue_5g_i8(app0, n_filler, clamp), 4, 12, clamp)
        tx = app0[2 * z:].astype(np.int8)[None, :]
        r = gpu_i8(dec, tx, 12, S.QuantParams().with_app_clamp(clamp), llr_offset=2 * z, nr_prologue=True,
                   n_filler=n_filler)
        assert_i8_equal(f"5g prologue clamp {clamp}", [ref], r)


@pytest.mark.parametrize("kernel", KERNELS)
def test_int8_zero_iterations_and_many_codewords(kernel):
    code = O.Code.nr(1, 16)
    dec = S.QcLdpcDecoder.with_lifting_size(1, 16, 0.5)
    _, llr = codewords(code, 40, 2.0, 77)
    apps = np.stack([O.quantize_i16(x) for x in llr])
    for iters in (0, 1, 3, 20):
        ref = oracle_i8(code, apps, 4, iters)
        assert_i8_equal(f"iters {iters} {kernel}", ref, gpu_i8(dec, apps.astype(np.int8), iters, S.QuantParams(),
                                                             kernel))


def test_int8_host_api_drop_in():
    """decode_layered_offset_min_sum_i8 / decode_5g_i8 through the host-buffer C entry points."""
    code = O.Code.nr(0, 16)
    dec = S.QcLdpcDecoder.with_lifting_size(0, 16, 0.5)
    _, llr = codewords(code, 1, 1.0, 5)
    app0 = O.quantize_i16(llr[0])
    app0[::37] = 900  # int16 posteriors outside the message range are accepted and clamped
    ref = code.decode_i8(app0, 4, 10)
    app = app0.copy()
    er = np.zeros(dec.required_edge_buffer(), np.int8)
    sc = np.zeros(dec.required_layer_buffer(), np.int8)
    hard = np.zeros(code.n, np.uint8)
    it = dec.decode_layered_offset_min_sum_i8(app, er, sc, hard, 10, S.QuantParams())
    assert it == ref["iters"] and np.array_equal(app, ref["app"]) and np.array_equal(er, ref["edge_r"])
    assert np.array_equal(hard, ref["hard"])
    app = app0.copy()
    it = dec.decode_5g_i8(app, 8, er, sc, hard, 10, S.QuantParams())
    ref = code.decode_i8(code.prologue_5g_i8(app0, 8), 4, 10)
    assert it == ref["iters"] and np.array_equal(app, ref["app"])
    with pytest.raises(S.FecError) as e:
        dec.decode_layered_offset_min_sum_i8(app, er[:-1], sc, hard, 10)
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.FecError) as e:
        dec.decode_layered_offset_min_sum_i8(app[:-1].copy(), er, sc, hard, 10)
    assert e.value.status == _lib.INVALID_PARAM


# ------------------------------------------------------------------ f32 path --

def assert_f32_close(label, ref, r):
    it = r.iters.cpu().numpy()
    app = r.app.cpu().numpy()
    er = r.edge_r.cpu().numpy()
    hard = r.hard.cpu().numpy()
    for b, o in enumerate(ref):
        assert it[b] == o["iters"], f"{label} cw{b}: iterations {it[b]} != {o['iters']}"
        assert np.array_equal(hard[b], o["hard"]), f"{label} cw{b}: hard decisions differ"
        np.testing.assert_allclose(app[b], o["llr"], rtol=F32_RTOL, atol=0, err_msg=f"{label} cw{b} app")
        np.testing.assert_allclose(er[b], o["edge_r"], rtol=F32_RTOL, atol=0, err_msg=f"{label} cw{b} edge_r")
        exact = np.array_equal(app[b].view(np.uint32), o["llr"].view(np.uint32))
        assert exact, f"{label} cw{b}: posterior within tolerance but not bit-identical"


def gpu_f32(dec, llr, iters, **kw):
    t = torch.from_numpy(np.ascontiguousarray(llr, dtype=np.float32)).cuda()
    r = dec.decode_batch_f32(t, iters, want_app=True, want_edge_r=True, want_hard=True, **kw)
    torch.cuda.synchronize()
    return r


def test_f32_golden_checksum():
    with open(os.path.join(GOLDEN, "ldpc_checksums.json")) as f:
        want = json.load(f)["checksums"]["ldpc_rust.checksum"]
    dec = S.QcLdpcDecoder.with_lifting_size(0, 384, 0.25)
    n = dec.variable_node_count()
    llr = np.where(np.arange(n) % 2 == 0, 0.5, -0.5).astype(np.float32)[None, :]
    r = gpu_f32(dec, llr, 10)
    assert int(r.iters[0]) == 10
    assert "%016x" % O.fnv1a_hard(r.hard[0].cpu().numpy()) == want


def test_f32_golden_convergence_trajectory():
    """Running t iterations from scratch reproduces the reference's frame t."""
    with open(os.path.join(GOLDEN, "ldpc_convergence_wifi27_r12.json")) as f:
        g = json.load(f)
    code = O.Code.wifi(27, 1, 2)
    info = np.array([((i * 2654435761) >> 31) & 1 for i in range(code.k)], dtype=np.uint8)
    llr = O.awgn(code.encode(info), 0.0, 0.5, 139)
    dec = S.wifi_ldpc_decoder(27, 1, 2, 0.25)
    for t in range(1, g["iterations_used"] + 1):
        r = gpu_f32(dec, llr[None, :], t)
        want = np.unpackbits(np.frombuffer(bytes.fromhex(g["frames"][t]["hard_bits"]), np.uint8),
                             bitorder="little")[: g["n"]]
        assert int(r.iters[0]) == t
        assert np.array_equal(r.hard[0].cpu().numpy(), want), f"frame {t}"
    r = gpu_f32(dec, llr[None, :], g["max_iterations"])
    assert int(r.iters[0]) == g["iterations_used"]


@pytest.mark.parametrize("kernel", ["auto", "generic_global"])
@pytest.mark.parametrize("kind,a,b", [("nr", 0, 32), ("nr", 1, 52), ("nr", 0, 384), ("wifi", 27, (1, 2)),
                                      ("wifi", 81, (5, 6)), ("wifi", 54, (3, 4)), ("wifi", 81, (2, 3)),
                                      ("nr", 0, 2)])
def test_f32_graphs(kind, a, b, kernel):
    """auto: the 5G NR f32 kernel or the generic kernel with messages compressed in
    shared memory (every 802.11 matrix; 5G NR at small Z); generic_global: messages in
    global memory."""
    if kind == "nr":
        code, dec = O.Code.nr(a, b), S.QcLdpcDecoder.with_lifting_size(a, b, 0.5)
    else:
        code, dec = O.Code.wifi(a, *b), S.wifi_ldpc_decoder(a, *b, 0.5)
    dec.set_kernel(kernel)
    for ebno in (0.5, 2.0):
        _, llr = codewords(code, 3, ebno, 0xF320000 + code.z)
        ref = [code.decode_f32(x, 0.5, 20) for x in llr]
        assert_f32_close(f"{kind} {a} {b} {ebno} {kernel}", ref, gpu_f32(dec, llr, 20))


def test_f32_5g_prologue_and_drop_in():
    """syndrome_ldpc_decode_5g (capi/src/lib.rs:290) against init_5g_llr + decode."""
    z = 24
    code = O.Code.nr(1, z)
    dec = S.QcLdpcDecoder.with_lifting_size(1, z, 0.25)
    _, llr = codewords(code, 1, 1.0, 42)
    x = llr[0]
    ref = code.decode_f32(code.init_5g_f32(x, 13), 0.25, 15)
    buf = x.copy()
    er = np.zeros(dec.required_edge_buffer(), np.float32)
    sc = np.zeros(dec.required_layer_buffer(), np.float32)
    hard = np.zeros(code.n, np.uint8)
    it = dec.decode_5g(buf, 13, er, sc, hard, 15)
    assert it == ref["iters"] and np.array_equal(hard, ref["hard"])
    assert np.array_equal(buf.view(np.uint32), ref["llr"].view(np.uint32))
    assert np.array_equal(er.view(np.uint32), ref["edge_r"].view(np.uint32))
    r = gpu_f32(dec, x[None, 2 * z:], 15, llr_offset=2 * z, nr_prologue=True, n_filler=13)
    assert int(r.iters[0]) == ref["iters"] and np.array_equal(r.hard[0].cpu().numpy(), ref["hard"])
    with pytest.raises(S.FecError) as e:
        dec.decode_5g(buf, 13, er, sc[:-1], hard, 15)
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.FecError) as e:
        dec.decode_5g(buf, 13, er, sc, hard[:-1].copy(), 15)
    assert e.value.status == _lib.INVALID_PARAM


def test_f32_adversarial_inputs():
    """fuzz/fuzz_targets/fuzz_ldpc_decode.rs: NaN, +-inf, zeros, huge values.

    Finite inputs (zeros, 1e30) must match exactly.  With NaN or infinite inputs
    the decode must complete with sane outputs; bit parity is not claimed there
    because a NaN created on the GPU (inf - inf) carries CUDA's canonical sign
    bit where x86 produces a negative NaN, and the sign bit feeds the sign XOR."""
    code = O.Code.nr(1, 8)
    dec = S.QcLdpcDecoder.with_lifting_size(1, 8, 0.3)
    rng = np.random.default_rng(3)
    x = rng.normal(0, 3, (4, code.n)).astype(np.float32)
    x[0, ::7] = np.nan
    x[1, ::5] = np.inf
    x[1, 1::5] = -np.inf
    x[2] = 0.0
    x[3, ::3] = 1e30
    ref = [code.decode_f32(v, 0.3, 6) for v in x]
    r = gpu_f32(dec, x, 6)
    it, hard = r.iters.cpu().numpy(), r.hard.cpu().numpy()
    app = r.app.cpu().numpy()
    for b in (2, 3):
        assert it[b] == ref[b]["iters"] and np.array_equal(hard[b], ref[b]["hard"])
        assert np.array_equal(app[b].view(np.uint32), ref[b]["llr"].view(np.uint32))
    for b in (0, 1):
        assert 1 <= it[b] <= 6 and set(np.unique(hard[b])) <= {0, 1}


@pytest.mark.parametrize("bg,z,count", [(0, 384, 2), (1, 384, 2), (0, 128, 7), (1, 52, 17), (0, 15, 61),
                                         (1, 2, 3), (0, 208, 3), (1, 320, 2)])
def test_f32_nr_compressed_kernel_matches_oracle_and_generic(bg, z, count):
    """The f32 5G NR kernel (compressed messages in shared memory, extension posteriors
    in a global workspace; at Z < 384 several codewords per CTA, each stopping on its
    own): bit-identical posteriors, messages, hard decisions and iteration counts to the
    oracle and to the generic f32 kernel, with the 5G prologue and filler bits, from
    noisy to clean channels, batches that leave the last CTA's group part-filled."""
    code = O.Code.nr(bg, z)
    dec = S.QcLdpcDecoder.with_lifting_size(bg, z, 0.5)
    for ebno, n_filler, iters in ((0.5, 0, 6), (1.5, min(120, z), 12), (4.0, 0, 20)):
        _, llr = codewords(code, count, ebno, 0xF384000 + bg * 7 + n_filler + z)
        ref = [code.decode_f32(code.init_5g_f32(x, n_filler), 0.5, iters) for x in llr]
        tx = np.ascontiguousarray(llr[:, 2 * z:])
        kw = dict(llr_offset=2 * z, nr_prologue=True, n_filler=n_filler)
        fast = gpu_f32(dec.set_kernel("auto"), tx, iters, **kw)
        assert_f32_close(f"bg{bg + 1} z{z} f32 {ebno} dB", ref, fast)
        slow = gpu_f32(dec.set_kernel("generic"), tx, iters, **kw)
        for name in ("iters", "app", "edge_r", "hard", "hard_packed"):
            a, b = getattr(fast, name).cpu().numpy(), getattr(slow, name).cpu().numpy()
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
    dec.set_kernel("auto")


def test_workspace_decode_matches_raw_buffer_decode():
    """src/qc_ldpc.rs:2785-2816: the workspace path and the raw-buffer path are the same
    decode (BG2 Z=3, weak structured LLRs, 8 iterations); the workspace's posterior
    staging buffer stays untouched by a plain decode (:1951-1954)."""
    for bg, z, five_g in ((1, 3, False), (0, 24, True)):
        dec = S.QcLdpcDecoder.with_lifting_size(bg, z, 0.25)
        n = dec.variable_node_count()
        llr_in = np.where(np.arange(n) % 7 == 0, -0.5, 1.5).astype(np.float32)
        llr_raw = llr_in.copy()
        edge_r = np.zeros(dec.required_edge_buffer(), np.float32)
        scratch = np.zeros(dec.required_layer_buffer(), np.float32)
        hard_raw = np.zeros(n, np.uint8)
        llr_ws = llr_in.copy()
        ws = dec.workspace()
        if five_g:
            it_raw = dec.decode_5g(llr_raw, 5, edge_r, scratch, hard_raw, 8)
            it_ws = dec.decode_5g_with_workspace(llr_ws, 5, ws, 8)
        else:
            it_raw = dec.decode_layered_offset_min_sum(llr_raw, edge_r, scratch, hard_raw, 8)
            it_ws = dec.decode_with_workspace(llr_ws, ws, 8)
        assert it_raw == it_ws
        assert np.array_equal(hard_raw, ws.hard_output())
        assert np.array_equal(llr_raw.view(np.uint32), llr_ws.view(np.uint32))
        assert not ws.posterior_llr().any(), "a plain decode wrote the workspace's staging buffer"


def test_workspace_from_wrong_decoder_is_rejected():
    """src/qc_ldpc.rs:2765-2783: a workspace sized for another code is rejected by the
    decode's size checks instead of being silently misused."""
    small = S.QcLdpcDecoder.with_lifting_size(1, 2, 0.25)
    large = S.QcLdpcDecoder.with_lifting_size(0, 2, 0.25)
    ws_small = small.workspace()
    llr = np.full(large.variable_node_count(), 5.0, np.float32)
    with pytest.raises(S.FecError) as e:
        large.decode_with_workspace(llr, ws_small, 5)
    assert e.value.status in (_lib.BUFFER_TOO_SMALL, _lib.INVALID_PARAM)
    with pytest.raises(S.FecError):
        large.decode_5g_with_workspace(llr, 0, ws_small, 5)


@pytest.mark.parametrize("llr_offset,pad,prologue", [(768, 3, True), (776, 0, True), (10064, 0, False), (0, 0, False)])
def test_int8_pair_tm_load_paths(llr_offset, pad, prologue):
    """The Z = 384 paired kernel loads rows with 128-bit loads when every row starts on a
    16-byte boundary (row pointer, stride and llr_offset multiples of 16) and byte by byte
    otherwise; an llr_offset past the core columns erases extension variables too.  Both
    paths, against the oracle (BG1 Z=384, 3 codewords)."""
    code = O.Code.nr(0, 384)
    dec = S.QcLdpcDecoder.with_lifting_size(0, 384, 0.5)
    _, llr = codewords(code, 3, 1.5, 0x7E57 + llr_offset)
    rows = np.stack([O.quantize_i16(x)[llr_offset:] for x in llr]).astype(np.int8)
    width = rows.shape[1]
    big = torch.zeros((3, width + pad), dtype=torch.int8, device="cuda")
    big[:, :width] = torch.from_numpy(rows).cuda()
    t = big[:, :width]
    dec.set_kernel("pair")
    r = dec.decode_batch_i8(t, 8, llr_offset=llr_offset, nr_prologue=prologue, quant=S.QuantParams(),
                            want_app=True, want_edge_r=True, want_hard=True)
    torch.cuda.synchronize()
    dec.set_kernel("auto")
    ref = O.decode_i8_batch(code, rows, O.beta_q(0.5), 8, llr_offset=llr_offset, nr_prologue=prologue,
                            hard_bits=code.n, detail=3)
    assert np.array_equal(r.iters.cpu().numpy(), ref["iters"])
    assert np.array_equal(r.app.cpu().numpy(), ref["app"])
    assert np.array_equal(r.edge_r.cpu().numpy(), ref["edge_r"])
    assert np.array_equal(r.hard_packed.cpu().numpy().view(np.uint32), ref["packed"])
