"""The reference's per-TB f32 DlSchDecoder and its LdpcPipeline frame API on the GPU.

DlSchDecoder (transport_block.rs:405-1060): every transmission's report (crc_ok,
per-code-block CRC, max iterations, HARQ transmission count) and, when the CRCs pass,
the TB bits must equal the oracle's restatement of the reference's f32 chain (HARQ f32
sum, prepare_cb_llr, decode_layered_offset_min_sum, CRC-24B/A, flush on success) over
RV 0, 2, 3, 1 retransmission sequences.

LdpcPipeline (ldpc_pipeline.rs:288-598): every frame comes back with the oracle's
f32 decode of its LLRs (iterations, hard decisions and posterior, exact), its tag
intact, in any order; acquire returns None when the whole pool is in use."""
import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402
from syndrome_b200 import _lib  # noqa: E402

RVS = (0, 2, 3, 1)
BETA = 0.5
CASES = [  # tb_size, rate, qm, g, Eb/N0
    (100, 0.5, 1, 248, 0.0),
    (500, 0.8, 2, 700, 1.0),
    (3000, 0.7, 4, 4288, 0.5),
    (8425, 0.85, 1, 10000, 1.5),
    (20000, 0.6, 2, 33334, 0.3),
]


def transmissions(a, r, qm, g, eb, seed):
    rng = np.random.default_rng(seed)
    tb = rng.integers(0, 2, a, dtype=np.uint8)
    enc = S.DlSchEncoder(a, r, qm, g)
    return tb, [S.AwgnChannel(eb, r, seed * 17 + i).transmit(enc.encode(tb, rv)) for i, rv in enumerate(RVS)]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_dlsch_decoder_f32_matches_oracle(case):
    a, r, qm, g, eb = CASES[case]
    tb, llrs = transmissions(a, r, qm, g, eb, 900 + case)
    dec = S.DlSchDecoder(a, r, qm, g, 8, BETA)
    ref = O.DlSchDecoder(a, r, qm, g, iterations=8, f32_beta=BETA)
    assert dec.output_bits() == llrs[0].size
    for n, rv in enumerate(RVS):
        out = np.zeros(a, np.uint8)
        got = dec.decode(llrs[n], rv, out)
        want = ref.decode(llrs[n], rv)
        label = f"A={a} R={r} Qm={qm} tx {n + 1}"
        assert got.crc_ok == want["crc_ok"], label
        assert got.harq_tx_count == want["harq_tx"], label
        assert got.max_iters_used == want["max_iters"], label
        assert list(got.cb_crc) == list(want["cb_crc"]), label
        if got.crc_ok:
            assert np.array_equal(out, want["tb"]) and np.array_equal(out, tb), label
            break


def test_dlsch_decoder_flush_pipeline_and_errors():
    a, r, qm, g, eb = CASES[2]
    tb, llrs = transmissions(a, r, qm, g, eb, 5)
    dec = S.DlSchDecoder(a, r, qm, g, 8, BETA)
    assert dec.worker_count() == 0 and dec.with_pipeline(4).worker_count() == 4
    out = np.zeros(a, np.uint8)
    first = dec.decode(llrs[0], 0, out)
    dec.flush_harq()
    again = dec.decode(llrs[0], 0, out)  # after a flush the accumulators start over
    assert again == first and again.harq_tx_count == 1
    with pytest.raises(S.SyndromeError) as e:
        dec.decode(llrs[0][:-1], 0, out)
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.SyndromeError) as e:
        dec.decode(llrs[0], 0, np.zeros(a - 1, np.uint8))
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.SyndromeError) as e:
        dec.decode(llrs[0], 4, out)
    assert e.value.status == _lib.INVALID_PARAM
    with pytest.raises(S.SyndromeError) as e:
        dec.with_pipeline(0)
    assert e.value.status == _lib.INVALID_PARAM
    for bad in [(0, 0.5, 2, 700), (500, 0.5, 2, 701), (500, 0.5, 0, 700)]:
        with pytest.raises(S.SyndromeError) as e:
            S.DlSchDecoder(*bad, 8, BETA)
        assert e.value.status == _lib.INVALID_PARAM


def frames_for(code, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        info = rng.integers(0, 2, code.k, dtype=np.uint8)
        out.append(O.awgn(code.encode(info), 0.5 + 0.1 * (i % 20), code.k / code.n, seed + i))
    return out


@pytest.mark.parametrize("workers", [1, 3])
def test_pipeline_frames_match_oracle(workers):
    dec = S.wifi_ldpc_decoder(27, 1, 2, BETA)
    code = O.Code.wifi(27, 1, 2)
    pipe = S.LdpcPipeline.with_workers(dec, 12, workers)
    assert pipe.worker_count() == workers
    llrs = frames_for(code, 600, 40 + workers)
    want = [code.decode_f32(x, BETA, 12) for x in llrs]
    got = {}
    nxt = 0
    held_max = 0
    while len(got) < len(llrs):
        progressed = False
        while nxt < len(llrs):
            f = pipe.acquire()
            if f is None:
                break
            f.llr_mut()[:] = llrs[nxt]
            f.set_tag(nxt)
            pipe.submit(f)
            nxt += 1
            progressed = True
        held_max = max(held_max, nxt - len(got))
        while (f := pipe.try_recv()) is not None:
            t = f.tag()
            got[t] = (f.iterations_used(), f.hard().copy(), f.llr_mut().copy())
            pipe.release(f)
            progressed = True
        if not progressed:
            import time
            time.sleep(0.0005)
    assert held_max <= pipe.pool_size()
    for t, (it, hard, app) in got.items():
        w = want[t]
        assert it == w["iters"], f"frame {t}: iterations"
        assert np.array_equal(hard, w["hard"]), f"frame {t}: hard decisions"
        assert np.array_equal(app.view(np.uint32), w["llr"].view(np.uint32)), f"frame {t}: posterior"


def test_pipeline_back_pressure_and_misuse():
    dec = S.QcLdpcDecoder.with_lifting_size(1, 52, BETA)
    code = O.Code.nr(1, 52)
    pipe = S.LdpcPipeline.new(dec, 6)
    held = []
    while (f := pipe.acquire()) is not None:
        held.append(f)
    assert len(held) == pipe.pool_size()
    with pytest.raises(S.SyndromeError):
        pipe.release(S.LdpcFrame(pipe, -1))
    x = frames_for(code, 1, 3)[0]
    f = held.pop()
    f.llr_mut()[:] = x
    pipe.submit(f)
    with pytest.raises(S.SyndromeError):  # already submitted
        pipe.submit(f)
    for h in held:  # an acquired frame may go back unsubmitted
        pipe.release(h)
    while (r := pipe.try_recv()) is None:
        pass
    w = code.decode_f32(x, BETA, 6)
    assert r.index == f.index and r.iterations_used() == w["iters"] and np.array_equal(r.hard(), w["hard"])
    pipe.release(r)
    with pytest.raises(S.SyndromeError):  # released twice
        pipe.release(r)


def test_dlsch_decoder_f32_256qam_and_repetition():
    for i, (a, r, qm, g, eb) in enumerate([(40000, 0.8, 8, 50000, 3.0), (200, 0.5, 2, 2600, -1.0)]):
        tb, llrs = transmissions(a, r, qm, g, eb, 1200 + i)
        dec = S.DlSchDecoder(a, r, qm, g, 8, BETA)
        ref = O.DlSchDecoder(a, r, qm, g, iterations=8, f32_beta=BETA)
        for n, rv in enumerate(RVS):
            out = np.zeros(a, np.uint8)
            got = dec.decode(llrs[n], rv, out)
            want = ref.decode(llrs[n], rv)
            assert (got.crc_ok, got.harq_tx_count, got.max_iters_used) == (want["crc_ok"], want["harq_tx"],
                                                                           want["max_iters"])
            assert list(got.cb_crc) == list(want["cb_crc"])
            if got.crc_ok:
                assert np.array_equal(out, tb)
                break
