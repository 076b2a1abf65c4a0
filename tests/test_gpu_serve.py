"""Transport-block serving on the GPU against the oracle's DL-SCH chain.

Every transmission's report (crc_ok, per-code-block CRC, max iterations, HARQ
transmission count) and, when the CRCs pass, the decoded payload must equal those of
the oracle's restatement of DlSchDecoder::decode (src/transport_block.rs:829) with the
int8 code-block decode (HARQ f32 sum -> quantize_llr_i16 -> decode_5g_i8), over
retransmission sequences that exercise HARQ soft combining (RV 0, 2, 3, 1), several
modulation orders and sizes from one code block to many.  Also: a transport block
gives the same result alone and in a mix, and admission by HBM budget completes.

Both engines run the same checks: the continuous one (the default: one persistent
kernel takes each transmission's code blocks as they arrive) and the step one."""
import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402
from syndrome_b200 import _lib  # noqa: E402

RVS = (0, 2, 3, 1)


def make_tb(tb_size, rate, qm, g, ebno, seed):
    """Seeded payload and its four RV transmissions' f32 LLRs (BPSK/AWGN per bit)."""
    rng = np.random.default_rng(seed)
    tb = rng.integers(0, 2, tb_size, dtype=np.uint8)
    enc = S.DlSchEncoder(tb_size, rate, qm, g)
    llrs = []
    for i, rv in enumerate(RVS):
        bits = enc.encode(tb, rv)
        llrs.append(S.AwgnChannel(ebno, rate, seed * 17 + i).transmit(bits))
    return tb, llrs


CASES = [  # tb_size, rate, qm, g, Eb/N0
    (100, 0.5, 1, 248, 0.0),
    (500, 0.8, 2, 700, 1.0),
    (3000, 0.7, 4, 4288, 0.5),
    (8425, 0.85, 1, 10000, 1.5),
    (20000, 0.6, 2, 33334, 0.3),
    (60000, 0.9, 6, 66666, 2.0),
]


def run_sequences(server, cases, seed0=0, max_tx=4):
    """Submits every TB, retransmits failures with the next RV; returns the reports
    per TB id in transmission order and the payloads of the passing decodes."""
    data, reports, payloads = {}, {}, {}
    for i, (a, r, qm, g, eb) in enumerate(cases):
        tid = seed0 + i
        data[tid] = (a, r, qm, g, make_tb(a, r, qm, g, eb, 1000 + tid))
        server.submit(tid, a, r, qm, g, RVS[0], data[tid][4][1][0])
        reports[tid] = []
    outstanding = len(cases)
    while outstanding:
        for res in server.wait(1):
            tid = res["tb_id"]
            reports[tid].append(res)
            a, r, qm, g, (tb, llrs) = data[tid]
            n = len(reports[tid])
            if res["crc_ok"]:
                payloads[tid] = server.fetch(tid, a)
                server.release(tid)
                outstanding -= 1
            elif n < max_tx:
                server.submit(tid, a, r, qm, g, RVS[n], llrs[n])
            else:
                server.release(tid)
                outstanding -= 1
    return data, reports, payloads


def check_against_oracle(data, reports, payloads, iterations=8):
    for tid, (a, r, qm, g, (tb, llrs)) in data.items():
        ref = O.DlSchDecoder(a, r, qm, g, iterations=iterations, beta_q=4, scale=8.0)
        for n, got in enumerate(reports[tid]):
            want = ref.decode(llrs[n], RVS[n])
            label = f"tb {tid} (A={a}, R={r}, Qm={qm}) tx {n + 1}"
            assert got["crc_ok"] == want["crc_ok"], label
            assert got["harq_tx_count"] == want["harq_tx"], label
            assert got["max_iters_used"] == want["max_iters"], label
            assert got["cb_crc"] == list(want["cb_crc"]), label
            if want["crc_ok"]:
                assert np.array_equal(payloads[tid], want["tb"]), label
                assert np.array_equal(payloads[tid], tb), label + ": CRC passed on a wrong payload"


ENGINES = [dict(), dict(engine="steps"), dict(engine="steps", kernel="pair_smem")]


@pytest.mark.parametrize("cfg", ENGINES)
def test_serve_matches_oracle_with_harq(cfg):
    server = S.Server(iterations=8, **cfg)
    data, reports, payloads = run_sequences(server, CASES)
    assert any(len(v) > 1 for v in reports.values()), "no retransmission happened: raise the noise"
    assert any(v[-1]["crc_ok"] for v in reports.values())
    check_against_oracle(data, reports, payloads)
    server.close()


@pytest.mark.parametrize("cfg", [dict(max_step_code_blocks=200),
                                 dict(max_step_code_blocks=200, engine="steps"),
                                 dict(max_step_code_blocks=200, latency_steps=1, backlog_code_blocks=1, engine="steps"),
                                 dict(steps_in_flight=16, latency_steps=16, engine="steps")])
def test_serve_same_result_alone_and_in_a_mix(cfg):
    """A result does not depend on what else is in flight, nor on how many steps run
    at once (the backlog policy's settings)."""
    alone = S.Server()
    d1, r1, p1 = run_sequences(alone, [CASES[3]], seed0=50)
    alone.close()
    mixed = S.Server(**cfg)
    cases = [CASES[0], CASES[4], CASES[3], CASES[1], CASES[5], CASES[2]]
    d2, r2, p2 = run_sequences(mixed, cases, seed0=48)  # CASES[3] gets id 50 here too
    mixed.close()
    strip = lambda reps: [{k: v for k, v in x.items() if k != "latency_us"} for x in reps]  # noqa: E731
    assert strip(r1[50]) == strip(r2[50])
    if 50 in p1:
        assert np.array_equal(p1[50], p2[50])


def test_serve_device_and_host_llrs_agree():
    a, r, qm, g, eb = CASES[2]
    tb, llrs = make_tb(a, r, qm, g, eb, 77)
    out = []
    for dev in (False, True):
        s = S.Server()
        x = torch.from_numpy(llrs[0]).cuda() if dev else llrs[0]
        s.submit(1, a, r, qm, g, 0, x)
        res = s.wait(1)[0]
        res.pop("latency_us")
        out.append((res, s.fetch(1, a)))
        s.close()
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])


def test_serve_small_harq_budget_admits_in_turn():
    """A budget that holds one large transport block at a time: later ones wait for
    memory and everything still completes."""
    seg = S.compute_segmentation(60000, 0.9)
    budget = seg.c * seg.n * 4 + 4096
    s = S.Server(harq_bytes=budget)
    cases = [(60000, 0.9, 2, 80000, 4.0)] * 3
    data, reports, payloads = run_sequences(s, cases, seed0=300)
    assert all(rep[-1]["crc_ok"] for rep in reports.values())
    assert s.stats()["harq_bytes_used"] == 0
    check_against_oracle(data, reports, payloads)
    s.close()


def test_serve_errors():
    s = S.Server()
    a, r, qm, g, eb = CASES[0]
    tb, llrs = make_tb(a, r, qm, g, eb, 5)
    s.submit(9, a, r, qm, g, 0, llrs[0])
    with pytest.raises(S.SyndromeError) as e:
        s.submit(9, a, r, qm, g, 2, llrs[1])  # still in flight
    assert e.value.status == _lib.INVALID_PARAM
    s.wait(1)
    with pytest.raises(S.SyndromeError):
        s.submit(9, a + 1, r, qm, g, 2, llrs[1])  # same id, other parameters
    with pytest.raises(S.SyndromeError) as e:
        s.submit(10, a, r, qm, g, 0, llrs[0][:-1])
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.SyndromeError):
        s.submit(11, a, r, qm, g, 4, llrs[0])
    s.release(9)
    s.close()


def test_serve_open_loop_load():
    """Poisson arrivals over a small pool with retransmissions: every arrival completes,
    latencies are positive and ordered percentiles come back."""
    pool = []
    for i, (a, r, qm, g, eb) in enumerate(CASES[:5]):
        tb, llrs = make_tb(a, r, qm, g, eb + 1.0, 500 + i)
        pool.append(dict(tb_size=a, target_rate=r, qm=qm, g=g, llrs=[torch.from_numpy(x).cuda() for x in llrs]))
    s = S.Server(max_step_code_blocks=256)
    rep = s.run_load(pool, offered_tb_per_s=2000.0, duration_s=0.25, seed=3, latencies=True)
    assert rep["tbs"] > 100 and rep["transmissions"] >= rep["tbs"]
    lat = rep["latencies_us"]
    assert (lat > 0).all() and 0 < rep["p50_us"] <= rep["p99_us"] <= rep["max_us"]
    assert s.stats()["tbs_held"] == 0 and s.stats()["harq_bytes_used"] == 0
    s.close()


@pytest.mark.parametrize("engine", ["continuous", "steps"])
def test_serve_large_transport_blocks_match_oracle(engine):
    """Transport blocks of 36 and 152 code blocks (the largest TB size): the
    desegmented payload and the TB CRC folded over every block must match the oracle
    and the transmitted bits."""
    cases = [(300000, 0.75, 2, 400002, 4.0), (1277992, 0.9, 6, 1419996, 5.0), (300000, 0.75, 2, 400002, 1.2)]
    server = S.Server(iterations=8, engine=engine)
    data, reports, payloads = run_sequences(server, cases, seed0=700)
    assert any(v[-1]["crc_ok"] for v in reports.values())
    check_against_oracle(data, reports, payloads)
    server.close()


@pytest.mark.parametrize("engine", ["continuous", "steps"])
def test_serve_256qam_and_repetition_match_oracle(engine):
    """Qm = 8 (the combine's interleaved gather) and a code block sent almost twice
    over (E close to 2 * ncb, up to three contributions per buffer position)."""
    cases = [(40000, 0.8, 8, 50000, 3.0), (200, 0.5, 2, 2600, -1.0), (200, 0.5, 2, 2600, 2.0)]
    server = S.Server(iterations=8, engine=engine)
    data, reports, payloads = run_sequences(server, cases, seed0=800)
    check_against_oracle(data, reports, payloads)
    server.close()


def test_serve_continuous_kernel_exits_when_idle_and_relaunches():
    """With a short idle limit the persistent kernel exits between transmissions that
    arrive far apart; the next transmission relaunches it, with the same results as a
    server that stays up."""
    import time

    a, r, qm, g, eb = CASES[3]
    tb, llrs = make_tb(a, r, qm, g, eb, 91)
    outs = []
    for idle in (50, 0):
        s = S.Server(idle_us=idle)
        got = []
        for k in range(3):
            s.submit(40 + k, a, r, qm, g, 0, llrs[0])
            res = s.wait(1)[0]
            res.pop("latency_us")
            got.append((res["crc_ok"], res["max_iters_used"], tuple(res["cb_crc"]), s.fetch(40 + k, a).tobytes()))
            s.release(40 + k)
            time.sleep(0.02)  # well past the 50 us idle limit
        if idle:
            assert s.stats()["steps"] == 3, "the kernel should have exited and been relaunched per transmission"
        outs.append(got)
        s.close()
    assert outs[0] == outs[1]


def test_serve_rejects_unknown_engine():
    with pytest.raises(ValueError):
        S.Server(engine="batch")


@pytest.mark.parametrize("engine", ["continuous", "steps"])
def test_serve_core_stats(engine):
    """The continuous engine reports its kernel's work items and phase times (each
    phase within the busy time); the step engine reports zeros."""
    s = S.Server(engine=engine)
    data, reports, payloads = run_sequences(s, CASES[:3], seed0=900)
    c = s.core_stats()
    s.close()
    if engine == "steps":
        assert all(v == 0 for v in c.values())
        return
    assert c["items"] >= sum(len(v) for v in reports.values())
    parts = c["combine_us"] + c["decode_us"] + c["crc_us"] + c["finish_us"]
    assert 0 < c["decode_us"] and parts <= c["busy_us"] * 1.001 + 1.0
    assert c["loops"] > 0
