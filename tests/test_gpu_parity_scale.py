"""Parity of the decode kernels with the oracle at the benchmark's scale.

The small parity tests (test_gpu_parity.py) run a handful of codewords, so each CTA
decodes one group and no CTA prefetches a next one.  At the benchmark's batch sizes
every CTA walks several groups of the batch: it reloads posteriors and clears its
check-row state for each group after the first, and it prefetches the next group's
LLRs into L2 while decoding the current one.  These tests run batches large enough
for every CTA to take several groups, through the same calls the benchmark makes,
and compare every codeword with the oracle:

* int8, 5G NR BG1 Z=384 at Eb/N0 = 1.0 dB, <= 8 iterations, the default kernel
  choice (the benchmark's workload): iteration counts and packed information bits
  of every codeword bit-identical; posteriors and messages bit-identical on a
  subset that spans first, second and later groups of the CTAs; the paired kernel's
  one-pair-per-SM variant gives the same on the same batch;
* the same for BG2 Z=384 and for BG1 at a run-time lifting size (Z = 192, two
  codeword pairs per CTA);
* f32, 5G NR BG1 Z=384: iteration counts and hard decisions bit-identical,
  posteriors within 1e-5 relative (checked bit-identical as well);
* the persistent mixed-shape kernel, both forms, with more work items than CTAs.
"""
import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402

F32_RTOL = 1e-5


def nr_batch(code, count, ebno, seed, punct):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, size=(count, code.k), dtype=np.uint8)
    rate = code.k / (code.n - punct)
    return info, rate, np.arange(count, dtype=np.uint64) + np.uint64(seed)


def unpack(words, bits):
    return np.unpackbits(np.ascontiguousarray(words).view(np.uint8), axis=1, bitorder="little")[:, :bits]


def detail_rows(count, ctas_hint):
    """Codewords whose CTA decodes them as its first, second and later group."""
    rows = {0, 1, 2, 3, count - 1, count - 2}
    for g in (1, 2, 3):
        for off in (0, 1, 7):
            rows.add(min(count - 1, g * ctas_hint * 2 + off))
    return sorted(rows)


@pytest.mark.parametrize("bg,z,count,ebno", [(0, 384, 2400, 1.0), (1, 384, 1800, 1.0), (0, 192, 2400, 1.5)])
def test_int8_batch_matches_oracle_at_scale(bg, z, count, ebno):
    code = O.Code.nr(bg, z)
    punct = 2 * z
    info, rate, seeds = nr_batch(code, count, ebno, 0x5CA1E + 131 * z + bg, punct)
    llr = O.batch_channel_i8(code, info, ebno, rate, seeds, tx_begin=punct)
    dec = S.QcLdpcDecoder.with_lifting_size(bg, z, 0.5)
    quant = S.QuantParams()
    d_llr = torch.from_numpy(llr).cuda()
    B = count
    words = (code.k + 31) // 32
    packed = torch.zeros((B, words), dtype=torch.int32, device="cuda")
    iters = torch.zeros((B,), dtype=torch.int32, device="cuda")
    ws = torch.empty((max(dec.batch_workspace_size(B), 1),), dtype=torch.uint8, device="cuda")
    # the benchmark's call: packed information bits and iteration counts only
    dec.decode_batch_i8(d_llr, 8, llr_offset=punct, nr_prologue=True, quant=quant, hard_bits=code.k,
                        workspace=ws, out={"hard_packed": packed, "iters": iters})
    torch.cuda.synchronize()
    ref = O.decode_i8_batch(code, llr, O.beta_q(0.5), 8, llr_offset=punct, nr_prologue=True, hard_bits=code.k)
    it = iters.cpu().numpy()
    bad = np.nonzero(it != ref["iters"])[0]
    assert bad.size == 0, f"iterations differ on {bad.size} of {B} codewords, first {bad[:8]}"
    got = packed.cpu().numpy().view(np.uint32)
    bad = np.nonzero((got != ref["packed"]).any(axis=1))[0]
    assert bad.size == 0, f"packed information bits differ on {bad.size} of {B} codewords, first {bad[:8]}"
    # the decode is not trivial: some codewords fail, some stop early
    assert 0 < (unpack(got, code.k) == info).all(axis=1).sum() < B or ebno > 1.0
    if z == 384:  # the one-pair-per-SM variant of the paired kernel on the same batch
        dec.set_kernel("pair_smem")
        p2, i2 = torch.zeros_like(packed), torch.zeros_like(iters)
        dec.decode_batch_i8(d_llr, 8, llr_offset=punct, nr_prologue=True, quant=quant, hard_bits=code.k,
                            workspace=ws, out={"hard_packed": p2, "iters": i2})
        torch.cuda.synchronize()
        dec.set_kernel("auto")
        assert torch.equal(i2, iters) and torch.equal(p2, packed), "pair_smem differs from the default kernel"
    # posteriors and messages on a subset spanning several groups per CTA
    r = dec.decode_batch_i8(d_llr, 8, llr_offset=punct, nr_prologue=True, quant=quant, hard_bits=code.k,
                            want_app=True, want_edge_r=True)
    torch.cuda.synchronize()
    assert torch.equal(r.iters.cpu(), iters.cpu()), "iterations differ between the two calls"
    rows = detail_rows(B, 148 * 2)
    sub = O.decode_i8_batch(code, llr[rows], O.beta_q(0.5), 8, llr_offset=punct, nr_prologue=True,
                            hard_bits=code.k, detail=len(rows))
    app = r.app.cpu().numpy()[rows]
    er = r.edge_r.cpu().numpy()[rows]
    for i, b in enumerate(rows):
        d = np.nonzero(app[i] != sub["app"][i])[0]
        assert d.size == 0, f"codeword {b}: posterior differs at {d[:5]} ({d.size} of {code.n})"
        d = np.nonzero(er[i] != sub["edge_r"][i])[0]
        assert d.size == 0, f"codeword {b}: C->V message differs at {d[:5]} ({d.size})"


def test_f32_batch_matches_oracle_at_scale():
    bg, z, count, ebno = 0, 384, 640, 1.0
    code = O.Code.nr(bg, z)
    punct = 2 * z
    info, rate, seeds = nr_batch(code, count, ebno, 0xF5CA1E, punct)
    llr = O.batch_channel_f32(code, info, ebno, rate, seeds, tx_begin=punct)
    dec = S.QcLdpcDecoder.with_lifting_size(bg, z, 0.5)
    r = dec.decode_batch_f32(torch.from_numpy(llr).cuda(), 8, llr_offset=punct, nr_prologue=True,
                             hard_bits=code.k, want_app=True)
    torch.cuda.synchronize()
    rows = detail_rows(count, 148)
    ref = O.decode_f32_batch(code, llr, 0.5, 8, llr_offset=punct, nr_prologue=True, hard_bits=code.k)
    it = r.iters.cpu().numpy()
    bad = np.nonzero(it != ref["iters"])[0]
    assert bad.size == 0, f"iterations differ on {bad.size} of {count} codewords, first {bad[:8]}"
    got = r.hard_packed.cpu().numpy().view(np.uint32)
    bad = np.nonzero((got != ref["packed"]).any(axis=1))[0]
    assert bad.size == 0, f"hard decisions differ on {bad.size} of {count} codewords, first {bad[:8]}"
    sub = O.decode_f32_batch(code, llr[rows], 0.5, 8, llr_offset=punct, nr_prologue=True, hard_bits=code.k,
                             detail=len(rows))
    app = r.app.cpu().numpy()[rows]
    for i, b in enumerate(rows):
        want = sub["app"][i]
        # the contract tolerance (1e-5 relative) ...
        np.testing.assert_allclose(app[i], want, rtol=F32_RTOL, atol=0, err_msg=f"codeword {b}")
        # ... and the kernel's own claim: the same operation order, bit-identical
        assert np.array_equal(app[i].view(np.uint32), want.view(np.uint32)), f"codeword {b}: posteriors not exact"


@pytest.mark.parametrize("kernel", ["auto", "pair_smem"])
def test_mixed_kernel_with_more_items_than_sms(kernel):
    """More work items than CTAs, so persistent CTAs take several items from the
    device queue (the tensor-memory form runs two CTAs per SM: 296 on 148 SMs, the
    shared-memory one 148); Z = 384 items (one codeword pair each) and small-Z items
    mixed."""
    rng = np.random.default_rng(77)
    shapes = [(0, 384)] * 300 + [(1, 384)] * 300 + [(1, int(z)) for z in rng.choice([13, 26, 52, 104], 60)]
    shapes = [shapes[i] for i in rng.permutation(len(shapes))]
    recs, rows, refs = [], [], []
    llr_off, out_off = 0, 0
    for i, (bg, z) in enumerate(shapes):
        code = O.Code.nr(bg, z)
        n_filler = int(rng.integers(0, code.k // 4 + 1))
        info = np.concatenate([rng.integers(0, 2, code.k - n_filler, dtype=np.uint8), np.zeros(n_filler, np.uint8)])
        ebno = float(rng.uniform(0.0, 3.0))
        rate = code.k / (code.n - 2 * z)
        row = O.batch_channel_i8(code, info[None], ebno, rate, [9000 + i], tx_begin=2 * z)[0]
        hard_bits = code.k - n_filler
        recs.append((bg, z, n_filler, hard_bits, llr_off, out_off))
        rows.append(row)
        refs.append((code, row, n_filler, hard_bits))
        llr_off += (row.size + 15) // 16 * 16
        out_off += (hard_bits + 31) // 32
    buf = np.zeros(llr_off, np.int8)
    for (_, _, _, _, off, _), row in zip(recs, rows):
        buf[off: off + row.size] = row
    batch = S.MixedBatch(np.array(recs, dtype=S.CODEWORD_DTYPE), 0.5, S.QuantParams(), 8)
    assert len(batch.items()) > 2 * 148
    assert batch.set_kernel(kernel) == (kernel == "auto")
    llr = torch.from_numpy(buf).cuda()
    out = torch.zeros(max(out_off, 1), dtype=torch.int32, device="cuda")
    iters = torch.zeros(len(refs), dtype=torch.int32, device="cuda")
    batch.decode(llr, out, iters)
    torch.cuda.synchronize()
    words = out.cpu().numpy().view(np.uint32)
    it = iters.cpu().numpy()
    for i, ((code, row, n_filler, hard_bits), rec) in enumerate(zip(refs, batch.codewords)):
        ref = O.decode_i8_batch(code, row[None], O.beta_q(0.5), 8, llr_offset=2 * code.z, nr_prologue=True,
                                n_filler=n_filler, hard_bits=hard_bits)
        assert it[i] == ref["iters"][0], f"codeword {i} {tuple(rec)}: iterations {it[i]} != {ref['iters'][0]}"
        w = words[rec["out_offset"]: rec["out_offset"] + (hard_bits + 31) // 32]
        assert np.array_equal(w, ref["packed"][0]), f"codeword {i} {tuple(rec)}: hard bits differ"
