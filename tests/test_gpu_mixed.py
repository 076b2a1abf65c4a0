"""Mixed-shape persistent decode (one launch over codewords of any BG / Z mix)
against the oracle's decode_5g_i8 path, codeword by codeword: iterations and hard
decisions bit-identical.  The paired cases run both forms of the paired kernel: the
default one with most check-row state in tensor memory (two CTAs per SM) and the
shared-memory one ("pair_smem", one CTA per SM)."""
import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402


def build_mix(shapes, seed, clamp=32767, report_all=False):
    rng = np.random.default_rng(seed)
    recs, rows, refs = [], [], []
    llr_off, out_off = 0, 0
    for i, (bg, z) in enumerate(shapes):
        code = O.Code.nr(bg, z)
        n_filler = int(rng.integers(0, code.k // 3 + 1))
        info = np.concatenate([O.random_bits(seed * 1000 + i, code.k - n_filler), np.zeros(n_filler, np.uint8)])
        cw = code.encode(info)
        ebno = float(rng.uniform(0.0, 3.0))
        app = O.quantize_i16(O.awgn(cw, ebno, code.k / (code.n - 2 * z), seed + 17 * i))
        app[: 2 * z] = 0
        row = app[2 * z:].astype(np.int8)
        ref = code.decode_i8(code.prologue_5g_i8(app, n_filler, clamp), O.beta_q(0.5), 8, clamp)
        hard_bits = code.n if report_all else code.k - n_filler
        recs.append((bg, z, n_filler, hard_bits, llr_off, out_off))
        rows.append(row)
        refs.append((ref, hard_bits))
        llr_off += (row.size + 15) // 16 * 16
        out_off += (hard_bits + 31) // 32
    buf = np.zeros(llr_off, np.int8)
    for (_, _, _, _, off, _), row in zip(recs, rows):
        buf[off: off + row.size] = row
    return np.array(recs, dtype=S.CODEWORD_DTYPE), buf, out_off, refs


def check(batch, buf, n_words, refs, use_graph=False, reps=1):
    llr = torch.from_numpy(buf).cuda()
    out = torch.zeros(max(n_words, 1), dtype=torch.int32, device="cuda")
    iters = torch.zeros(len(refs), dtype=torch.int32, device="cuda")
    for _ in range(reps):
        out.zero_()
        iters.zero_()
        batch.decode(llr, out, iters, use_graph=use_graph)
    torch.cuda.synchronize()
    words = out.cpu().numpy().view(np.uint32)
    it = iters.cpu().numpy()
    for i, ((ref, hard_bits), rec) in enumerate(zip(refs, batch.codewords)):
        assert it[i] == ref["iters"], f"codeword {i} {tuple(rec)}: iterations {it[i]} != {ref['iters']}"
        w = words[rec["out_offset"]: rec["out_offset"] + (hard_bits + 31) // 32]
        bits = np.unpackbits(w.view(np.uint8), bitorder="little")[:hard_bits]
        assert np.array_equal(bits, ref["hard"][:hard_bits]), f"codeword {i} {tuple(rec)}: hard bits differ"


def use_kernel(batch, kernel):
    tm = batch.set_kernel(kernel)
    assert tm == (kernel == "auto"), f"{kernel}: tensor-memory form {tm}"


@pytest.mark.parametrize("kernel", ["auto", "pair_smem"])
def test_mixed_batch_matches_oracle(kernel):
    rng = np.random.default_rng(5)
    shapes = [(1, int(z)) for z in rng.choice([z for z in S.LIFTING_SIZES if z <= 64], 40)]
    shapes += [(0, int(z)) for z in rng.choice([2, 5, 13, 32, 64], 20)]
    shapes += [(0, 384), (1, 384), (0, 128), (1, 208), (0, 64), (0, 64)]
    order = rng.permutation(len(shapes))
    shapes = [shapes[i] for i in order]
    recs, buf, n_words, refs = build_mix(shapes, 11)
    batch = S.MixedBatch(recs, 0.5, S.QuantParams(), 8)
    assert sum(c for _, _, c in batch.items()) == len(shapes)
    use_kernel(batch, kernel)
    check(batch, buf, n_words, refs)


def test_mixed_batch_reporting_every_variable():
    """Codewords reporting hard decisions past their core columns run the
    shared-memory paired kernel, whose extension decisions are in shared memory."""
    shapes = [(0, 384), (1, 384), (0, 64), (1, 26), (1, 2), (0, 160)] * 2
    recs, buf, n_words, refs = build_mix(shapes, 61, report_all=True)
    batch = S.MixedBatch(recs, 0.5, S.QuantParams(), 8)
    assert not batch.set_kernel("auto")
    check(batch, buf, n_words, refs)


def test_mixed_batch_one_codeword_per_thread_kernel():
    """app_clamp below 7874 selects the one-codeword-per-thread mixed kernel."""
    rng = np.random.default_rng(8)
    shapes = [(int(rng.integers(0, 2)), int(z)) for z in rng.choice([4, 26, 96, 384], 16)]
    recs, buf, n_words, refs = build_mix(shapes, 41, clamp=1000)
    batch = S.MixedBatch(recs, 0.5, S.QuantParams().with_app_clamp(1000), 8)
    check(batch, buf, n_words, refs)


@pytest.mark.parametrize("kernel", ["auto", "pair_smem"])
def test_mixed_batch_odd_counts_per_shape(kernel):
    """Paired items with an odd codeword count leave one lane empty; items of small Z
    leave the threads past their pairs idle."""
    shapes = [(0, 384)] * 3 + [(1, 384)] * 5 + [(0, 7)] * 9 + [(1, 2)] * 1 + [(0, 240)] * 3 + [(1, 176)] * 2
    recs, buf, n_words, refs = build_mix(shapes, 57)
    batch = S.MixedBatch(recs, 0.5, S.QuantParams(), 8)
    use_kernel(batch, kernel)
    check(batch, buf, n_words, refs)


@pytest.mark.parametrize("kernel", ["auto", "pair_smem"])
def test_mixed_batch_graph_replay_and_tiles(kernel):
    shapes = [(1, 13)] * 30 + [(0, 16)] * 20 + [(1, 52)] * 7
    recs, buf, n_words, refs = build_mix(shapes, 23)
    batch = S.MixedBatch(recs, 0.5, S.QuantParams(), 8, tile_hints={(1, 13): 4, (0, 16): 1})
    items = batch.items()
    assert all(c <= 4 for bg, z, c in items if (bg, z) == (1, 13))
    assert all(c == 1 for bg, z, c in items if (bg, z) == (0, 16))
    use_kernel(batch, kernel)
    check(batch, buf, n_words, refs, use_graph=True, reps=3)
    # switching the kernel drops the captured graph; the other kernel replays the same
    use_kernel(batch, "pair_smem" if kernel == "auto" else "auto")
    check(batch, buf, n_words, refs, use_graph=True, reps=2)


def test_mixed_batch_rejects_unknown_kernel():
    recs, _, _, _ = build_mix([(1, 13)], 3)
    batch = S.MixedBatch(recs)
    with pytest.raises(ValueError):
        batch.set_kernel("tmem")
