"""Wi-Fi shortened / punctured decode on the GPU against the oracle
(src/wifi_rate_matching.rs:267 decode_shortened).

Both forms -- the reference-shaped single-codeword call with host buffers and the
batched device call whose kernel rebuilds each codeword while loading it -- must give
the oracle's iteration count and hard decisions exactly and its posterior within
F32_RTOL relative (the f32 contract tolerance; the kernel is expected to be exact),
over all 12 802.11 matrices with genuine shortening and puncturing, noisy channels
and the edge cases (no shortening, all parity punctured, an empty payload)."""
import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402
from syndrome_b200 import _lib  # noqa: E402
from syndrome_b200 import wifi_rate_matching as W  # noqa: E402

F32_RTOL = 1e-5
BETA = 0.25
ALL_12 = [(z, rn, rd) for z in (27, 54, 81) for rn, rd in ((1, 2), (2, 3), (3, 4), (5, 6))]


def cases(k, n):
    pay = k // 3
    max_coded = n - (k - pay)
    return [(pay, max_coded - max_coded // 5), ((2 * k) // 3, n - k // 3 - 7), (k, n), (k, k), (0, 5)]


def received(enc, pay, tgt, ebno, seed):
    rng = np.random.default_rng(seed)
    payload = rng.integers(0, 2, pay, dtype=np.uint8)
    coded = np.zeros(tgt, np.uint8)
    W.encode_shortened(enc, payload, tgt, coded)
    rate = max(pay, 1) / max(tgt, 1)
    return payload, S.AwgnChannel(ebno, rate, seed).transmit(coded)


def same(label, it, hard, app, ref):
    assert it == ref["iters"], f"{label}: iterations {it} != {ref['iters']}"
    assert np.array_equal(hard, ref["hard"]), f"{label}: hard decisions differ"
    np.testing.assert_allclose(app, ref["llr"], rtol=F32_RTOL, atol=0, err_msg=f"{label}: posterior")


@pytest.mark.parametrize("z,rn,rd", ALL_12)
def test_host_decode_shortened_matches_oracle(z, rn, rd):
    dec = S.wifi_ldpc_decoder(z, rn, rd, BETA)
    enc = S.wifi_ldpc_encoder(z, rn, rd)
    code = O.Code.wifi(z, rn, rd)
    for i, (pay, tgt) in enumerate(cases(code.k, code.n)):
        payload, rx = received(enc, pay, tgt, 1.0 + 0.5 * i, 1000 * z + 10 * rn + i)
        ws = dec.workspace()
        it = W.decode_shortened_with_workspace(dec, pay, rx, ws, 20)
        ref = O.wifi_decode_shortened(code, BETA, pay, rx, 20)
        same(f"Z={z} R={rn}/{rd} P={pay} T={tgt}", it, ws.hard, ws.codeword_llr, ref)


@pytest.mark.parametrize("z,rn,rd", [(27, 1, 2), (54, 3, 4), (81, 5, 6), (81, 2, 3)])
def test_batched_decode_shortened_matches_oracle(z, rn, rd):
    dec = S.wifi_ldpc_decoder(z, rn, rd, BETA)
    enc = S.wifi_ldpc_encoder(z, rn, rd)
    code = O.Code.wifi(z, rn, rd)
    for pay, tgt in cases(code.k, code.n):
        rows, refs = [], []
        for b in range(24):
            _, rx = received(enc, pay, tgt, -0.5 + 0.2 * b, 77 * z + b)
            rows.append(rx)
            refs.append(O.wifi_decode_shortened(code, BETA, pay, rx, 12))
        pad = np.zeros((len(rows), tgt + 3), np.float32)  # rows longer than the sent bits
        pad[:, :tgt] = np.stack(rows) if tgt else 0
        rx_d = torch.from_numpy(pad).cuda()[:, :tgt] if tgt else torch.from_numpy(pad).cuda()[:, :0]
        r = W.decode_shortened_batch(dec, rx_d, pay, 12, hard_bits=code.n, want_app=True, want_hard=True)
        torch.cuda.synchronize()
        it, hard, app = r.iters.cpu().numpy(), r.hard.cpu().numpy(), r.app.cpu().numpy()
        bits = np.unpackbits(r.hard_packed.cpu().numpy().view(np.uint8), axis=1, bitorder="little")[:, : code.n]
        for b in range(len(rows)):
            same(f"Z={z} R={rn}/{rd} P={pay} T={tgt} cw{b}", int(it[b]), hard[b], app[b], refs[b])
            assert np.array_equal(bits[b], refs[b]["hard"])


def test_decode_shortened_errors():
    dec = S.wifi_ldpc_decoder(27, 1, 2, BETA)
    n = dec.variable_node_count()
    ws = dec.workspace()
    with pytest.raises(S.SyndromeError) as e:  # payload above K
        W.decode_shortened_with_workspace(dec, 325, np.zeros(400, np.float32), ws, 5)
    assert e.value.status == _lib.INVALID_PARAM
    with pytest.raises(S.SyndromeError) as e:  # more sent bits than N - n_shrt
        W.decode_shortened_with_workspace(dec, 100, np.zeros(425, np.float32), ws, 5)
    assert e.value.status == _lib.INVALID_PARAM
    with pytest.raises(S.SyndromeError) as e:  # codeword buffer not N long
        W.decode_shortened(dec, 100, np.zeros(400, np.float32), np.zeros(n - 1, np.float32), ws.edge_r,
                           ws.layer_scratch, ws.hard, 5)
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.SyndromeError) as e:  # device rows shorter than the sent bits claim
        x = torch.zeros((4, 400), dtype=torch.float32, device="cuda")
        _lib.check(_lib.load().syndrome_wifi_decode_shortened_batch_f32(
            dec._h, x.data_ptr(), 300, 100, 400, 4, 5, None, 0, 0, None, None, 0, None, 0, None, 0, None, 0, None))
    assert e.value.status == _lib.INVALID_PARAM
