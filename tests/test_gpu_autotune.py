"""Autotuner on the GPU: the chosen item size of each shape is one of its candidates,
and decoding with the tuned sizes (mixed batches and the serving engine) gives the
same results as with the defaults -- the tuning changes only the time."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import syndrome_b200 as S  # noqa: E402
from syndrome_b200 import autotune as A  # noqa: E402
from syndrome_b200.mixed import CODEWORD_DTYPE, code_dims  # noqa: E402

SHAPES = [(1, 13), (0, 64), (1, 384)]


def mixed_case(seed):
    cws, parts, off, out = [], [], 0, 0
    for i, (bg, z) in enumerate(SHAPES):
        n, k, _ = code_dims(bg, z)
        llr = A.synthetic_llrs(bg, z, 40, 1.0 + 0.3 * i, seed + i).reshape(-1)
        for j in range(40):
            cws.append((bg, z, 0, k, off + j * (n - 2 * z), out))
            out += (k + 31) // 32
        off += llr.numel()
        parts.append(llr)
    return np.array(cws, dtype=CODEWORD_DTYPE), torch.cat(parts), out


def test_tune_tiles_and_same_results():
    log = []
    tiles = A.tune_tiles(SHAPES, codewords=64, repeats=1, log=log)
    for shape, t in tiles.items():
        assert t in A.tile_candidates(*shape)
    assert len(log) == sum(len(A.tile_candidates(*s)) for s in SHAPES)
    cws, llr, words = mixed_case(5)
    res = []
    for hints in (None, tiles, {s: 2 for s in SHAPES}):
        plan = S.MixedBatch(cws, tile_hints=hints)
        out = torch.zeros(words, dtype=torch.int32, device="cuda")
        it = torch.zeros(len(cws), dtype=torch.int32, device="cuda")
        plan.decode(llr, out, it)
        torch.cuda.synchronize()
        res.append((out.cpu().numpy(), it.cpu().numpy()))
    for o, i in res[1:]:
        assert np.array_equal(o, res[0][0]) and np.array_equal(i, res[0][1])


def test_tune_kernel_picks_a_serving_kernel():
    log = []
    name = A.tune_kernel(0, 64, batch=300, repeats=1, log=log)
    names = {"pair", "nr", "generic", "generic_global"}
    assert name in names and {r[2] for r in log} == names


def test_serving_with_tuned_tiles_gives_the_same_results():
    def run(tiles):
        s = S.Server(max_step_code_blocks=64)
        if tiles:
            s.set_tiles(tiles)
        reports = []
        for i, (a, r, qm, g, eb) in enumerate([(3000, 0.7, 2, 4288, 1.5), (20000, 0.6, 2, 33334, 1.0),
                                               (500, 0.5, 1, 1000, 2.0)]):
            rng = np.random.default_rng(70 + i)
            tb = rng.integers(0, 2, a, dtype=np.uint8)
            llr = S.AwgnChannel(eb, r, 80 + i).transmit(S.DlSchEncoder(a, r, qm, g).encode(tb, 0))
            s.submit(i, a, r, qm, g, 0, llr)
        got = {}
        while len(got) < 3:
            for res in s.wait(1):
                res.pop("latency_us", None)
                res.pop("queue_us", None)
                res.pop("step_us", None)
                got[res["tb_id"]] = res
        s.close()
        return got

    base = run(None)
    seg = [S.compute_segmentation(a, r) for a, r in [(3000, 0.7), (20000, 0.6), (500, 0.5)]]
    assert run({(p.bg, p.z): 2 for p in seg}) == base
