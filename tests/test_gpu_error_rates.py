"""Error-rate agreement of the GPU decoder with the reference's published curves.

Bit-exactness to the oracle (the other GPU tests) fixes every decoded bit for given
channel values; these tests check the statistical claims on top of that, with the
reference's own Monte Carlo statistics:

* the BLER waterfall the reference records for BG1 Z=384, every bit transmitted
  (R = 0.3235), f32 layered offset min-sum, beta 0.25, 10 iterations
  (src/bin/ber_sim.rs:77-190, bench/results/ber_rust.json, README.md:834-838):
  50 block errors in 283 frames at 1.0 dB, 0 in 500 at 1.5 dB.  The GPU's count
  must agree with the recorded one as two binomial samples: their Wilson intervals
  overlap and a pooled two-proportion z-test does not reject equality at 5 %.  (The
  recorded point itself is not required to lie inside the GPU's interval: at 283
  frames it carries +-0.045 of sampling error of its own, more than the GPU's
  1000-frame interval is wide);
* the int8 gates of tests/ldpc_int8_quantization_loss.rs: the default fixed-point
  format is not resolvably worse than f32 on the same channel realisations
  (:649-695, BG1 Z=32, 0.75 dB, beta 0.5, 10 iterations), and holding the
  posterior to +-127 is resolvably worse than the wide posterior (:609-646, 1.0 dB).

Intervals: the Wilson score interval of src/montecarlo.rs:320-350 and the paired
log-ratio interval of tests/ldpc_int8_quantization_loss.rs:147-185, restated
below.  Channel realisations come from the oracle's encoder and channel; the decode
is the GPU's.
"""
import math

import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402

Z95 = 1.959963984540054  # two-sided 95 % normal quantile (MonteCarloConfig's default)


def wilson(events, samples, z=Z95):
    """src/montecarlo.rs:320-350: Wilson score interval, exact endpoints at 0 and n."""
    if samples == 0:
        return 0.0, 1.0
    n = float(samples)
    p = events / n
    z2 = z * z
    denom = 1.0 + z2 / n
    center = (p + z2 / (2.0 * n)) / denom
    half = (z / denom) * math.sqrt(p * (1.0 - p) / n + z2 / (4.0 * n * n))
    lo = 0.0 if events == 0 else max(center - half, 0.0)
    hi = 1.0 if events == samples else min(center + half, 1.0)
    return lo, hi


def log_ratio_ci(f32_errors, i8_errors, f32_only, i8_only):
    """tests/ldpc_int8_quantization_loss.rs:147-185: ln(BLER_i8 / BLER_f32) with the
    delta-method variance of the paired (multinomial) counts."""
    nf, ni = float(f32_errors), float(i8_errors)
    a, b, c = nf - f32_only, float(f32_only), float(i8_only)
    point = math.log(ni / nf)
    d = 1.0 / ni - 1.0 / nf
    half = Z95 * math.sqrt(a * d * d + b / (nf * nf) + c / (ni * ni))
    return point, point - half, point + half


def overlap(a, b):
    return a[0] <= b[1] and b[0] <= a[1]


def two_proportion_z(e1, n1, e2, n2):
    """Pooled two-proportion z statistic of e1/n1 against e2/n2 (0 when both are 0)."""
    p = (e1 + e2) / (n1 + n2)
    se = math.sqrt(p * (1.0 - p) * (1.0 / n1 + 1.0 / n2))
    return 0.0 if se == 0.0 else (e1 / n1 - e2 / n2) / se


def frames(code, count, ebno, seed):
    """Seeded information bits and the channel LLRs of every codeword bit."""
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, size=(count, code.k), dtype=np.uint8)
    seeds = (np.arange(count, dtype=np.uint64) << np.uint64(20)) ^ np.uint64(seed)
    return info, O.batch_channel_f32(code, info, ebno, code.k / code.n, seeds)


def block_errors(packed, info):
    bits = np.unpackbits(packed.cpu().numpy().view(np.uint8), axis=1, bitorder="little")[:, : info.shape[1]]
    return (bits != info).any(axis=1)


def gpu_f32(dec, llr, iterations, k):
    r = dec.decode_batch_f32(torch.from_numpy(llr).cuda(), iterations, hard_bits=k)
    torch.cuda.synchronize()
    return r.hard_packed


def gpu_i8(dec, llr, iterations, k, quant):
    q = np.stack([O.quantize_i16(x, quant.scale) for x in llr]).astype(np.int8)
    r = dec.decode_batch_i8(torch.from_numpy(q).cuda(), iterations, quant=quant, hard_bits=k)
    torch.cuda.synchronize()
    return r.hard_packed


@pytest.mark.parametrize("ebno,count,ref_errors,ref_frames", [(1.0, 1000, 50, 283), (1.5, 500, 0, 500)])
def test_bler_waterfall_matches_reference(ebno, count, ref_errors, ref_frames):
    code = O.Code.nr(0, 384)
    dec = S.QcLdpcDecoder.with_lifting_size(0, 384, 0.25)
    info, llr = frames(code, count, ebno, 0xBE5 + int(ebno * 10))
    errors = int(block_errors(gpu_f32(dec, llr, 10, code.k), info).sum())
    ours, ref = wilson(errors, count), wilson(ref_errors, ref_frames)
    assert overlap(ours, ref), (f"{ebno} dB: GPU BLER {errors}/{count} {ours} and the reference's "
                                f"{ref_errors}/{ref_frames} {ref} do not overlap")
    z = two_proportion_z(errors, count, ref_errors, ref_frames)
    assert abs(z) < Z95, f"{ebno} dB: GPU {errors}/{count} against reference {ref_errors}/{ref_frames}: z = {z:+.2f}"
    if ref_errors:
        assert errors > 0, f"{ebno} dB: no block errors where the reference's waterfall has BLER 0.18"


def paired_counts(z, ebno, count, app_clamp, seed):
    code = O.Code.nr(0, z)
    dec = S.QcLdpcDecoder.with_lifting_size(0, z, 0.5)
    info, llr = frames(code, count, ebno, seed)
    ef = block_errors(gpu_f32(dec, llr, 10, code.k), info)
    ei = block_errors(gpu_i8(dec, llr, 10, code.k, S.QuantParams().with_app_clamp(app_clamp)), info)
    return int(ef.sum()), int(ei.sum()), int((ef & ~ei).sum()), int((ei & ~ef).sum())


def test_int8_default_format_not_resolvably_worse_than_f32():
    """tests/ldpc_int8_quantization_loss.rs:649-695 (its regression guard): on the same
    channel realisations the default int8 format's BLER ratio to f32 has a 95 %
    interval reaching down to 1 or below."""
    counts = paired_counts(32, 0.75, 1500, 32767, 0xF0A70001)
    point, lo, hi = log_ratio_ci(*counts)
    assert counts[0] >= 120 and counts[1] >= 120, f"too few block errors to resolve anything: {counts}"
    assert lo <= 0.0, f"int8 resolvably worse than f32: log ratio {point:+.4f} [{lo:+.4f}, {hi:+.4f}], {counts}"


def test_int8_narrow_posterior_resolvably_worse():
    """tests/ldpc_int8_quantization_loss.rs:609-646: clamping the posterior to +-127
    costs a resolvable amount against the wide (default) posterior."""
    wide = log_ratio_ci(*paired_counts(32, 1.0, 1000, 32767, 0x0A000001))
    narrow = log_ratio_ci(*paired_counts(32, 1.0, 1000, 127, 0x0A000001))
    assert narrow[0] > wide[0], f"narrow {narrow} not worse than wide {wide}"
    assert narrow[1] > wide[2] or wide[1] > narrow[2], f"intervals overlap: narrow {narrow}, wide {wide}"
