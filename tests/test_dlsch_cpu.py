"""Transport-block host logic against the oracle: segmentation (segmentation.rs:265),
CRC-24A/B (crc.rs), the transport-block encoder (transport_block.rs:303, including the
rate-matching walk of rate_matching.rs, here in closed form) and the reference's own
unit-test properties for these functions."""
import numpy as np
import pytest

import _oracle as O
import syndrome_b200 as S
from syndrome_b200 import _lib


def test_segmentation_matches_oracle_sweep():
    rng = np.random.default_rng(1)
    sizes = [1, 24, 100, 292, 293, 500, 3824, 3825, 8424, 8425, 10000, 100000, 1277992]
    sizes += [int(x) for x in np.exp(rng.uniform(np.log(1), np.log(1277992), 300))]
    for a in sizes:
        for r in (0.1, 0.25, 0.26, 0.5, 0.67, 0.68, 0.9):
            p = S.compute_segmentation(a, r)
            assert O.segmentation(a, r) == (p.bg, p.z, p.c, p.b, p.k_prime, p.k, p.n, p.n_filler,
                                            int(p.has_cb_crc), p.payload), (a, r)


def test_segmentation_reference_properties():
    """segmentation.rs tests: base-graph boundaries, K' covers B', limits."""
    assert S.compute_segmentation(292, 0.9).bg == 1
    assert S.compute_segmentation(293, 0.5).bg == 1
    assert S.compute_segmentation(293, 0.68).bg == 0
    assert S.compute_segmentation(4000, 0.5).bg == 0
    assert S.compute_segmentation(9999, 0.25).bg == 1
    p = S.compute_segmentation(100, 0.5)
    assert p.c == 1 and not p.has_cb_crc and p.n_filler == p.k - p.k_prime
    for a in (10000, 8425):
        p = S.compute_segmentation(a, 0.5)
        b_prime = p.b + p.c * 24
        assert p.bg == 0 and p.c > 1 and p.has_cb_crc and p.b == a + 24
        assert 0 <= p.k_prime * p.c - b_prime < p.c
    assert S.compute_segmentation(8425, 0.5).c == 2
    assert S.compute_segmentation(5000, 0.8).n == 66 * S.compute_segmentation(5000, 0.8).z
    with pytest.raises(S.SyndromeError) as e:
        S.compute_segmentation(S.dlsch.MAX_TB_SIZE_BITS + 1, 0.5)
    assert e.value.status == _lib.INVALID_PARAM
    with pytest.raises(S.SyndromeError):
        S.compute_segmentation(0, 0.5)


def test_crc24_matches_oracle_and_round_trips():
    rng = np.random.default_rng(2)
    for n in (0, 1, 7, 8, 9, 24, 100, 1000, 8424):
        bits = rng.integers(0, 2, n, dtype=np.uint8)
        for kind in (S.dlsch.CRC24A, S.dlsch.CRC24B):
            c = S.crc24(bits, kind)
            assert c == O.crc24(bits, kind)
            tail = np.array([(c >> (23 - i)) & 1 for i in range(24)], np.uint8)
            assert S.crc24(np.concatenate([bits, tail]), kind) == 0  # attach then check
    assert S.crc24(np.zeros(24, np.uint8)) == 0
    flip = np.array([1, 0, 1, 1, 0, 0, 1, 0, 1, 1, 0, 1, 1, 0, 0, 0], np.uint8)
    c = S.crc24(flip)
    tail = np.array([(c >> (23 - i)) & 1 for i in range(24)], np.uint8)
    bad = np.concatenate([flip, tail])
    bad[0] ^= 1
    assert S.crc24(bad) != 0


@pytest.mark.parametrize("a,rate,qm,g", [(100, 0.5, 1, 248), (500, 0.3, 2, 1700), (3000, 0.7, 4, 4288),
                                         (8425, 0.5, 1, 17000), (20000, 0.85, 6, 23532), (40000, 0.2, 1, 200000),
                                         (9000, 0.9, 8, 10000)])
def test_tb_encoder_matches_oracle(a, rate, qm, g):
    rng = np.random.default_rng(a)
    tb = rng.integers(0, 2, a, dtype=np.uint8)
    enc = S.DlSchEncoder(a, rate, qm, g)
    for rv in range(4):
        got = enc.encode(tb, rv)
        want = O.dlsch_encode(tb, rate, qm, g, rv)
        assert got.size == want.size == enc.output_bits()
        d = np.nonzero(got != want)[0]
        assert d.size == 0, f"rv {rv}: {d.size} bits differ, first {d[:5]}"


def test_tb_encoder_errors():
    with pytest.raises(S.SyndromeError):
        S.DlSchEncoder(0, 0.5, 1, 512)
    with pytest.raises(S.SyndromeError):
        S.DlSchEncoder(100, 0.5, 0, 512)
    with pytest.raises(S.SyndromeError):
        S.DlSchEncoder(100, 0.5, 1, 0)
    with pytest.raises(S.SyndromeError):
        S.DlSchEncoder(100, 0.5, 3, 512)  # G not a multiple of Qm
    enc = S.DlSchEncoder(100, 0.5, 1, 248)
    with pytest.raises(S.SyndromeError) as e:
        enc.encode(np.zeros(99, np.uint8), 0)
    assert e.value.status == _lib.BUFFER_TOO_SMALL
    with pytest.raises(S.SyndromeError) as e:
        enc.encode(np.zeros(100, np.uint8), 4)
    assert e.value.status == _lib.INVALID_PARAM


def _llr(bits, ebno, rate, seed):
    return S.AwgnChannel(ebno, rate, seed).transmit(bits)


def test_oracle_chain_decodes_the_encoder_output():
    """transport_block.rs encoder_decoder_noiseless_roundtrip and
    harq_combining_recovers_a_block_that_fails_alone, on the oracle chain fed by this
    library's encoder (the oracle decoder is what the GPU engine is checked against)."""
    rng = np.random.default_rng(11)
    for a, rate, qm, g in ((100, 0.5, 1, 248), (8425, 0.5, 2, 17000), (30000, 0.8, 4, 37500)):
        tb = rng.integers(0, 2, a, dtype=np.uint8)
        enc = S.DlSchEncoder(a, rate, qm, g)
        bits = enc.encode(tb, 0)
        dec = O.DlSchDecoder(a, rate, qm, g, iterations=8)
        noiseless = np.where(bits == 0, 4.0, -4.0).astype(np.float32)
        r = dec.decode(noiseless, 0)
        assert r["crc_ok"] and np.array_equal(r["tb"], tb) and r["harq_tx"] == 1 and all(r["cb_crc"])
    # a block that fails alone is recovered by combining a second redundancy version
    a, rate, qm, g = 3000, 0.85, 1, 3530
    tb = rng.integers(0, 2, a, dtype=np.uint8)
    enc = S.DlSchEncoder(a, rate, qm, g)
    for seed in range(20):
        dec = O.DlSchDecoder(a, rate, qm, g, iterations=8)
        first = dec.decode(_llr(enc.encode(tb, 0), 1.0, rate, seed), 0)
        if first["crc_ok"]:
            continue
        second = dec.decode(_llr(enc.encode(tb, 2), 1.0, rate, 1000 + seed), 2)
        assert second["harq_tx"] == 2
        if second["crc_ok"]:
            assert np.array_equal(second["tb"], tb)
            break
    else:
        pytest.fail("no seed showed HARQ combining recovering a failed block")
