"""Wi-Fi shortening and puncturing on the host (src/wifi_rate_matching.rs).

The oracle's restatement is pinned by the reference's own cases (the doc example of
shortening_and_puncture_counts and the reference's rejection tests, a noiseless round
trip through every 802.11 matrix); the library's counts and shortened encoder must
equal it.  Decoding is on the GPU (test_gpu_wifi_shortened.py)."""
import numpy as np
import pytest

import _oracle as O
import syndrome_b200 as S
from syndrome_b200 import _lib
from syndrome_b200 import wifi_rate_matching as W

ALL_12 = [(z, rn, rd) for z in (27, 54, 81) for rn, rd in ((1, 2), (2, 3), (3, 4), (5, 6))]


def test_counts_reference_cases():
    # wifi_rate_matching.rs:108-113 (doc example) and the tests at :398-435
    for f in (O.wifi_counts, W.shortening_and_puncture_counts):
        assert f(324, 648, 100, 400) == (224, 24)
        assert f(324, 648, 324, 648) == (0, 0)
    for bad in [(324, 648, 325, 648), (324, 648, 100, 99), (324, 648, 100, 425), (648, 324, 10, 20)]:
        assert O.wifi_counts(*bad) is None
        with pytest.raises(S.SyndromeError) as e:
            W.shortening_and_puncture_counts(*bad)
        assert e.value.status == _lib.INVALID_PARAM


def test_counts_sweep_matches_oracle():
    rng = np.random.default_rng(7)
    for _ in range(3000):
        k = int(rng.integers(0, 2000))
        n = int(rng.integers(max(k - 5, 0), k + 2000))
        pay = int(rng.integers(0, k + 3))
        tgt = int(rng.integers(0, n + 3))
        want = O.wifi_counts(k, n, pay, tgt)
        if want is None:
            with pytest.raises(S.SyndromeError):
                W.shortening_and_puncture_counts(k, n, pay, tgt)
        else:
            assert W.shortening_and_puncture_counts(k, n, pay, tgt) == want


def cases(k, n):
    """(payload_bits, target_coded_bits) pairs: genuine shortening and puncturing as in
    the reference's round-trip test, none of either, all parity punctured, one bit."""
    pay = k // 3
    max_coded = n - (k - pay)
    return [(pay, max_coded - max_coded // 5), (k, n), (k, k), ((2 * k) // 3, n - k // 3 - 7), (1, 1), (0, 5)]


@pytest.mark.parametrize("z,rn,rd", ALL_12)
def test_encode_shortened_matches_oracle(z, rn, rd):
    enc = S.wifi_ldpc_encoder(z, rn, rd)
    code = O.Code.wifi(z, rn, rd)
    rng = np.random.default_rng(z * 100 + rn)
    for pay, tgt in cases(code.k, code.n):
        payload = rng.integers(0, 2, pay, dtype=np.uint8)
        out = np.zeros(tgt, np.uint8)
        W.encode_shortened(enc, payload, tgt, out)
        assert np.array_equal(out, O.wifi_encode_shortened(code, payload, tgt)), (pay, tgt)
        assert np.array_equal(out[:pay], payload)
    with pytest.raises(S.SyndromeError) as e:
        W.encode_shortened(enc, np.zeros(10, np.uint8), 40, np.zeros(39, np.uint8))
    assert e.value.status == _lib.BUFFER_TOO_SMALL


@pytest.mark.parametrize("z,rn,rd", ALL_12)
def test_oracle_noiseless_round_trip(z, rn, rd):
    """wifi_rate_matching.rs:440-495: strong noiseless LLRs return the payload exactly."""
    code = O.Code.wifi(z, rn, rd)
    pay = code.k // 3
    max_coded = code.n - (code.k - pay)
    tgt = max_coded - max_coded // 5
    payload = (np.arange(pay) % 2).astype(np.uint8)
    coded = O.wifi_encode_shortened(code, payload, tgt)
    rx = np.where(coded == 0, 8.0, -8.0).astype(np.float32)
    r = O.wifi_decode_shortened(code, 0.25, pay, rx, 20)
    assert np.array_equal(r["hard"][:pay], payload)
