"""GPU batch encoder (src/qc_ldpc.rs:2592-2727 QcLdpcEncoder::encode, unique
codewords) against the host encoder and the oracle's parity check: every codeword of
a batch must equal the host encoder's byte for byte and satisfy H c = 0, for 5G NR
BG1/BG2 at small, odd and maximal lifting sizes and the twelve 802.11 matrices."""
import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402
from syndrome_b200 import _lib  # noqa: E402

WIFI = [(z, rn, rd) for z in (27, 54, 81) for rn, rd in ((1, 2), (2, 3), (3, 4), (5, 6))]


def check(enc, code, count, seed):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (count, enc.info_bit_count()), dtype=np.uint8)
    want = enc.encode_batch(info)
    got = enc.encode_batch_device(torch.from_numpy(info).cuda()).cpu().numpy()
    assert np.array_equal(got, want)
    for i in range(min(count, 4)):
        assert code.check(got[i])


@pytest.mark.parametrize("bg,z", [(0, 2), (0, 15), (0, 384), (1, 7), (1, 52), (1, 384)])
def test_device_encoder_nr(bg, z):
    check(S.QcLdpcEncoder.new(bg, z), O.Code.nr(bg, z), 300 if z < 384 else 40, 10 * z + bg)


@pytest.mark.parametrize("z,rn,rd", WIFI)
def test_device_encoder_wifi(z, rn, rd):
    check(S.wifi_ldpc_encoder(z, rn, rd), O.Code.wifi(z, rn, rd), 200, z + rn)


def test_device_encoder_strides_and_errors():
    enc = S.QcLdpcEncoder.new(1, 13)
    k, n = enc.info_bit_count(), enc.codeword_bit_count()
    info = np.random.default_rng(3).integers(0, 2, (17, k + 5), dtype=np.uint8)
    d_info = torch.from_numpy(info).cuda()
    out = torch.zeros((17, n + 9), dtype=torch.uint8, device="cuda")
    L = _lib.load()
    _lib.check(L.syndrome_ldpc_encode_batch_device(enc._h, d_info.data_ptr(), k + 5, out.data_ptr(), n + 9, 17, None))
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy()[:, :n], enc.encode_batch(info[:, :k]))
    assert not out.cpu().numpy()[:, n:].any()  # nothing written past N
    with pytest.raises(S.SyndromeError) as e:
        _lib.check(L.syndrome_ldpc_encode_batch_device(enc._h, d_info.data_ptr(), k - 1, out.data_ptr(), n, 1, None))
    assert e.value.status == _lib.BUFFER_TOO_SMALL
