"""The persistent f32 decode of mixed 802.11 batches (WifiMixedBatch) against the
oracle's decode_layered_offset_min_sum (src/qc_ldpc.rs:962-1221), codeword by
codeword: iteration counts and hard decisions bit-identical.

The batches mix all twelve matrices of src/wifi_ldpc_tables.rs:339-453 with a
per-codeword Eb/N0 drawn from [0.5, 4] dB and up to 20 iterations, so iteration
counts range from 1 to the limit inside every chunk; small chunks make CTAs switch
matrices often and take many chunks each."""
import numpy as np
import pytest

import _oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402


def build(count, seed, report="k"):
    rng = np.random.default_rng(seed)
    shapes = [S.WIFI_SHAPES[i % 12] for i in rng.permutation(count)]
    recs, rows, codes = [], [], {}
    off, out = 0, 0
    for i, (z, rn, rd) in enumerate(shapes):
        code = codes.setdefault((z, rn, rd), O.Code.wifi(z, rn, rd))
        info = rng.integers(0, 2, size=(1, code.k), dtype=np.uint8)
        ebno = float(rng.uniform(0.5, 4.0))
        row = O.batch_channel_f32(code, info, ebno, code.k / code.n, [seed * 7919 + i])[0]
        hard_bits = code.k if report == "k" else code.n
        recs.append((z, rn, rd, hard_bits, off, out))
        rows.append(row)
        off += code.n + (i % 3)  # odd gaps between codewords
        out += (hard_bits + 31) // 32
    buf = np.zeros(off, np.float32)
    for r, row in zip(recs, rows):
        buf[r[4]: r[4] + row.size] = row
    return np.array(recs, dtype=S.WIFI_CODEWORD_DTYPE), buf, out, codes, rows


def oracle(recs, rows, codes, beta, iterations):
    its, words = [], []
    for r, row in zip(recs, rows):
        code = codes[(int(r["z"]), int(r["rate_num"]), int(r["rate_den"]))]
        ref = O.decode_f32_batch(code, row[None], beta, iterations, hard_bits=int(r["hard_bits"]))
        its.append(int(ref["iters"][0]))
        words.append(ref["packed"][0])
    return its, words


def run(batch, buf, n_words, count, use_graph=False, reps=1):
    llr = torch.from_numpy(buf).cuda()
    out = torch.zeros(max(n_words, 1), dtype=torch.int32, device="cuda")
    iters = torch.full((count,), -1, dtype=torch.int32, device="cuda")
    for _ in range(reps):
        out.zero_()
        iters.fill_(-1)
        batch.decode(llr, out, iters, use_graph=use_graph)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32), iters.cpu().numpy()


def check(recs, words, it, ref_its, ref_words):
    for i, r in enumerate(recs):
        assert it[i] == ref_its[i], f"codeword {i} {tuple(r)}: iterations {it[i]} != {ref_its[i]}"
        w = words[r["out_offset"]: r["out_offset"] + len(ref_words[i])]
        assert np.array_equal(w, ref_words[i]), f"codeword {i} {tuple(r)}: hard decisions differ"


@pytest.mark.parametrize("chunk", [0, 2])
def test_wifi_mixed_matches_oracle(chunk):
    recs, buf, n_words, codes, rows = build(720, 31 + chunk, report="n" if chunk else "k")
    batch = S.WifiMixedBatch(recs, 0.5, 20, chunk=chunk)
    n_chunks, ctas = batch.chunks()
    if chunk:
        assert n_chunks > ctas, "the small-chunk case must give CTAs several chunks each"
    words, it = run(batch, buf, n_words, len(recs))
    ref_its, ref_words = oracle(recs, rows, codes, 0.5, 20)
    assert min(ref_its) <= 2 and max(ref_its) == 20, "the batch must mix fast and slow codewords"
    check(recs, words, it, ref_its, ref_words)


def test_wifi_mixed_graph_replay_and_beta():
    recs, buf, n_words, codes, rows = build(150, 77)
    batch = S.WifiMixedBatch(recs, 0.25, 12, chunk=5)
    words, it = run(batch, buf, n_words, len(recs), use_graph=True, reps=3)
    check(recs, words, it, *oracle(recs, rows, codes, 0.25, 12))


def test_wifi_mixed_zero_iterations_and_one_shape():
    recs, buf, n_words, codes, rows = build(40, 5)
    batch = S.WifiMixedBatch(recs, 0.5, 0)
    words, it = run(batch, buf, n_words, len(recs))
    assert (it == 0).all()
    check(recs, words, it, *oracle(recs, rows, codes, 0.5, 0))
    one = recs[recs["z"] == recs["z"][0]]
    one = one[(one["rate_num"] == one["rate_num"][0])]
    batch = S.WifiMixedBatch(one, 0.5, 20)
    words, it = run(batch, buf, n_words, len(one))
    sel = [i for i, r in enumerate(recs) if tuple(r) in {tuple(x) for x in one}]
    ref_its, ref_words = oracle(one, [rows[i] for i in sel], codes, 0.5, 20)
    check(one, words, it, ref_its, ref_words)


def test_wifi_mixed_rejects_bad_plans_and_buffers():
    bad = np.array([(27, 1, 3, 10, 0, 0)], dtype=S.WIFI_CODEWORD_DTYPE)
    with pytest.raises(S.FecError):
        S.WifiMixedBatch(bad)
    recs, buf, n_words, _, _ = build(12, 9)
    batch = S.WifiMixedBatch(recs)
    with pytest.raises(S.FecError):
        batch.decode(torch.zeros(10, dtype=torch.float32, device="cuda"),
                     torch.zeros(n_words, dtype=torch.int32, device="cuda"))
