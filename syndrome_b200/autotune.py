"""Autotuner for the per-shape launch choices.

* Mixed-shape batches and the serving engine: how many codewords of one (base graph,
  lifting size) shape one work item (one CTA) takes.  A full item keeps every thread
  of the CTA busy, but a batch then splits into few items and the last ones leave SMs
  idle; smaller items balance better.  `tune_tiles` times every candidate on seeded
  synthetic LLRs of the shape with CUDA events and keeps the fastest.
* Single-shape batches: which kernel (paired 5G NR, one codeword per thread 5G NR,
  generic layered) decodes a (base graph, lifting size, app_clamp) fastest
  (`tune_kernel`).

Results are plain dicts, saved and loaded as JSON (`save`, `load`) so that a
deployment tunes once per GPU model.  No counterpart in the reference (one code block
per call on CPU threads).  Decoding results do not depend on these choices, only the
time does."""
import json

import numpy as np

from .mixed import CODEWORD_DTYPE, MixedBatch, code_dims, tile_capacity
from .qc_ldpc import QcLdpcDecoder, QcLdpcEncoder, QuantParams


def synthetic_llrs(bg, z, count, ebno_db=1.5, seed=0, scale=8.0, device="cuda"):
    """int8 LLRs (variables 2Z..N) of `count` random codewords of shape (bg, z) sent as
    BPSK over AWGN at Eb/N0 ebno_db, quantized like quantize_llr_i16 (x scale, round,
    clamp to +-127): a seeded stand-in for received code blocks, made on the GPU."""
    import torch

    n, k, _ = code_dims(bg, z)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    info = torch.randint(0, 2, (count, k), generator=gen, device=device, dtype=torch.uint8)
    cw = QcLdpcEncoder.new(bg, z).encode_batch_device(info)
    rate = k / (n - 2 * z)
    sigma = (1.0 / (2.0 * rate * 10.0 ** (ebno_db / 10.0))) ** 0.5
    x = 1.0 - 2.0 * cw[:, 2 * z:].float()
    y = x + sigma * torch.randn(x.shape, generator=gen, device=device)
    return torch.clamp(torch.round(2.0 * y / sigma ** 2 * scale), -127, 127).to(torch.int8).contiguous()


def _time_ms(fn, repeats):
    import torch

    fn()  # warm-up (and graph / plan set-up)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeats):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / repeats


def tile_candidates(bg, z):
    """Item sizes tried for a shape: the CTA's capacity and its halvings down to 2."""
    cap = tile_capacity(bg, z)
    out, t = [], cap
    while t >= 2:
        out.append(t)
        t //= 2
    return out or [cap]


def tune_tiles(shapes, codewords=None, candidates=None, iterations=8, ebno_db=1.5, repeats=3, offset_beta=0.5,
               quant=None, seed=0, sms=148, log=None):
    """{(bg, z): tile} with the fastest item size of each shape.  `codewords` per shape
    defaults to two full waves (2 x sms x capacity); `candidates` may map a shape to
    the tiles to try (default tile_candidates).  `log`, if a list, receives one
    (bg, z, tile, ms, Gbit/s) row per measurement."""
    import torch

    quant = quant or QuantParams()
    best = {}
    for bg, z in shapes:
        cap = tile_capacity(bg, z)
        count = int(codewords or 2 * sms * cap)
        n, k, _ = code_dims(bg, z)
        row = n - 2 * z
        llr = synthetic_llrs(bg, z, count, ebno_db, seed + 1000 * bg + z).reshape(-1)
        words = (k + 31) // 32
        cws = np.zeros(count, dtype=CODEWORD_DTYPE)
        cws["base_graph"], cws["z"], cws["n_filler"], cws["hard_bits"] = bg, z, 0, k
        cws["llr_offset"] = np.arange(count, dtype=np.int64) * row
        cws["out_offset"] = np.arange(count, dtype=np.int64) * words
        out = torch.empty(count * words, dtype=torch.int32, device=llr.device)
        tried = (candidates or {}).get((bg, z)) or tile_candidates(bg, z)
        results = []
        for tile in tried:
            plan = MixedBatch(cws, offset_beta, quant, iterations, tile_hints={(bg, z): int(tile)})
            ms = _time_ms(lambda: plan.decode(llr, out), repeats)
            gbps = count * k / (ms * 1e-3) / 1e9
            results.append((gbps, -int(tile)))
            if isinstance(log, list):
                log.append((bg, z, int(tile), ms, gbps))
            del plan
        best[(bg, z)] = -max(results)[1] if results else cap
    return best


def tune_kernel(bg, z, batch=None, iterations=8, ebno_db=1.5, repeats=3, offset_beta=0.5, quant=None, seed=0,
                log=None):
    """The fastest kernel name ("pair", "nr", "generic" or "generic_global") for plain
    batches of one (bg, z) shape at quant.app_clamp; kernels that do not apply are
    skipped."""
    import torch

    from . import _lib

    quant = quant or QuantParams()
    n, k, _ = code_dims(bg, z)
    batch = int(batch or max(2 * 148 * max(1, 384 // z), 256))
    llr = synthetic_llrs(bg, z, batch, ebno_db, seed)
    dec = QcLdpcDecoder.with_lifting_size(bg, z, offset_beta)
    out = {"hard_packed": torch.empty((batch, (k + 31) // 32), dtype=torch.int32, device=llr.device),
           "iters": torch.empty((batch,), dtype=torch.int32, device=llr.device)}
    best = None
    for name in ("pair", "nr", "generic", "generic_global"):
        dec.set_kernel(name)

        def run():
            dec.decode_batch_i8(llr, iterations, llr_offset=2 * z, nr_prologue=True, quant=quant, hard_bits=k,
                                out=out)

        try:
            ms = _time_ms(run, repeats)
        except _lib.SyndromeError:
            continue  # the kernel does not serve this request
        if isinstance(log, list):
            log.append((bg, z, name, ms))
        if best is None or ms < best[1]:
            best = (name, ms)
    return best[0]


def save(tiles, path, kernels=None):
    """Writes a tuning result ({(bg, z): tile}, optional {(bg, z): kernel}) as JSON."""
    doc = {"tiles": [[int(bg), int(z), int(t)] for (bg, z), t in sorted(tiles.items())]}
    if kernels:
        doc["kernels"] = [[int(bg), int(z), str(kn)] for (bg, z), kn in sorted(kernels.items())]
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)


def load(path):
    """(tiles, kernels) dicts from a file written by save."""
    with open(path) as f:
        doc = json.load(f)
    tiles = {(int(bg), int(z)): int(t) for bg, z, t in doc.get("tiles", [])}
    kernels = {(int(bg), int(z)): str(kn) for bg, z, kn in doc.get("kernels", [])}
    return tiles, kernels
