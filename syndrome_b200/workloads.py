"""Seeded synthetic batches of the benchmark's mixed-shape workloads, built on the GPU
with this library's encoder (torch for the channel and the rate matching).

* nr_rate_matched: 5G NR code blocks of mixed shape (BG1 with Z in {64, 128, 256,
  384} or BG2 with any lifting size up to 384, each with probability 1/2), filler bits
  uniform in [0, K/5] (information bits K' = K - filler), a target code rate uniform in
  [1/5, 8/9] reached by the RV0 bit selection of the circular buffer
  (src/rate_matching.rs:181-240, :418-450: E = ceil(K'/R) bits from position 0 on,
  filler positions skipped, wrapping at Ncb = N - 2Z; puncturing when E < Ncb - filler,
  repetition when larger), BPSK over AWGN with a per-block Eb/N0 uniform in [0, 3] dB
  at the block's actual rate K'/E, the received LLRs summed back into the circular
  buffer (rate_dematch_llr, :675-700) and quantized to int8 at scale 8, saturating
  at +-127.  Decoded by MixedBatch with the 5G prologue.
* wifi_mixed: 802.11 codewords uniform over the twelve matrices, every bit sent,
  BPSK over AWGN with a per-codeword Eb/N0 uniform in [0.5, 4] dB, f32 LLRs.
  Decoded by WifiMixedBatch.

The reference has no such batches (it decodes one code block per call); the mix
recipes above are this library's choices where the benchmark leaves them open.
"""
import numpy as np

from .mixed import CODEWORD_DTYPE, LIFTING_SIZES, WIFI_CODEWORD_DTYPE, WIFI_SHAPES, wifi_dims
from .qc_ldpc import QcLdpcEncoder, wifi_ldpc_encoder


def awgn_llr(x_bits, rate, ebno_db, gen):
    """LLR = 2y / sigma^2 of BPSK (0 -> +1) over AWGN, sigma^2 = 1 / (2 R Eb/N0);
    rate and ebno_db (tensors or numbers) broadcast against the bits."""
    import torch

    rate = torch.as_tensor(rate, dtype=torch.float64, device=x_bits.device)
    ebno_db = torch.as_tensor(ebno_db, dtype=torch.float64, device=x_bits.device)
    sigma = torch.sqrt(1.0 / (2.0 * rate * 10.0 ** (ebno_db / 10.0)))
    x = 1.0 - 2.0 * x_bits.float()
    return (2.0 * (x + sigma * torch.randn(x.shape, generator=gen, device=x.device)) / (sigma * sigma)).float()


def nr_rate_matched(count, seed, device="cuda", scale=8.0):
    """(records [CODEWORD_DTYPE], int8 LLR tensor, output words, information bits).
    Every record's hard_bits is its K' information bits."""
    import torch

    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    bg = rng.integers(0, 2, count)
    z = np.where(bg == 0, rng.choice([64, 128, 256, 384], count), rng.choice(np.array(LIFTING_SIZES), count))
    kb = np.where(bg == 0, 22, 10)
    k = kb * z
    n_filler = (rng.random(count) * (k // 5 + 1)).astype(np.int64)
    kp = k - n_filler
    rate_t = rng.uniform(0.2, 8.0 / 9.0, count)
    e = np.ceil(kp / rate_t).astype(np.int64)
    ebno = rng.uniform(0.0, 3.0, count)
    ncb = np.where(bg == 0, 66, 50) * z
    pad = (ncb + 15) // 16 * 16
    llr_off = np.concatenate([[0], np.cumsum(pad)[:-1]]).astype(np.int64)
    out_off = np.concatenate([[0], np.cumsum((kp + 31) // 32)[:-1]]).astype(np.int64)
    total = int(pad.sum())
    words = int(((kp + 31) // 32).sum())
    recs = np.zeros(count, CODEWORD_DTYPE)
    recs["base_graph"], recs["z"], recs["n_filler"], recs["hard_bits"] = bg, z, n_filler, kp
    recs["llr_offset"], recs["out_offset"] = llr_off, out_off
    buf = torch.zeros(total, dtype=torch.float32, device=device)
    for b in (0, 1):
        for zz in np.unique(z[bg == b]):
            idx = np.nonzero((bg == b) & (z == zz))[0]
            zz = int(zz)
            enc = QcLdpcEncoder.new(int(b), zz)
            kk = int(kb[idx[0]]) * zz
            info = torch.randint(0, 2, (len(idx), kk), generator=gen, device=device, dtype=torch.uint8)
            col = torch.arange(kk, device=device)[None, :]
            kp_t = torch.from_numpy(kp[idx]).to(device)
            info = torch.where(col < kp_t[:, None], info, torch.zeros_like(info)).contiguous()
            cw = enc.encode_batch_device(info)  # [G, N], filler bits encoded as 0
            # the RV0 selection of every block of the group, flattened: block j sends E_j bits
            ej = torch.from_numpy(e[idx]).to(device)
            blk = torch.repeat_interleave(torch.arange(len(idx), device=device), ej)
            t = torch.arange(int(ej.sum()), device=device) - torch.repeat_interleave(torch.cumsum(ej, 0) - ej, ej)
            nf = torch.from_numpy(n_filler[idx]).to(device)[blk]
            f0 = (kp_t - 2 * zz)[blk]
            q = t % (int(ncb[idx[0]]) - nf)
            pos = q + torch.where(q >= f0, nf, torch.zeros_like(nf))  # circular-buffer position, filler skipped
            bits = cw[blk, 2 * zz + pos]
            rate = torch.from_numpy(kp[idx] / e[idx]).to(device)[blk]
            eb = torch.from_numpy(ebno[idx]).to(device)[blk]
            llr = awgn_llr(bits, rate, eb, gen)
            buf.index_add_(0, torch.from_numpy(llr_off[idx]).to(device)[blk] + pos, llr)
            del blk, t, nf, f0, q, pos, bits, rate, eb, llr
    v = buf * scale
    q8 = torch.clamp(torch.sign(v) * torch.floor(torch.abs(v) + 0.5), -127, 127).to(torch.int8)
    return recs, q8.contiguous(), words, int(kp.sum())


def wifi_mixed(count, seed, device="cuda"):
    """(records [WIFI_CODEWORD_DTYPE], f32 LLR tensor, output words, information bits);
    records report the K information bits of each codeword."""
    import torch

    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    shape_i = rng.integers(0, len(WIFI_SHAPES), count)
    ebno = rng.uniform(0.5, 4.0, count)
    recs = np.zeros(count, WIFI_CODEWORD_DTYPE)
    off = out = 0
    order = []
    for si, s in enumerate(WIFI_SHAPES):  # codewords of one matrix contiguous in the buffer
        idx = np.nonzero(shape_i == si)[0]
        n, k = wifi_dims(*s)
        for i in idx:
            recs[i] = (s[0], s[1], s[2], k, off, out)
            off += n
            out += (k + 31) // 32
        order.append((s, idx))
    buf = torch.empty(off, dtype=torch.float32, device=device)
    bits = 0
    for s, idx in order:
        if len(idx) == 0:
            continue
        n, k = wifi_dims(*s)
        enc = wifi_ldpc_encoder(*s)
        info = torch.randint(0, 2, (len(idx), k), generator=gen, device=device, dtype=torch.uint8)
        cw = enc.encode_batch_device(info)
        eb = torch.from_numpy(ebno[idx]).to(device)[:, None]
        llr = awgn_llr(cw, k / n, eb, gen)
        o = int(recs[idx[0]]["llr_offset"])
        buf[o: o + llr.numel()] = llr.reshape(-1)
        bits += k * len(idx)
    return recs, buf, out, bits
