"""Autotuner results on the host: candidate item sizes and the JSON round trip."""
import syndrome_b200 as S  # noqa: F401
from syndrome_b200 import autotune as A
from syndrome_b200.mixed import tile_capacity


def test_tile_candidates_are_halvings_of_the_capacity():
    for bg, z in [(0, 2), (0, 384), (1, 13), (1, 96)]:
        c = A.tile_candidates(bg, z)
        cap = tile_capacity(bg, z)
        assert c[0] == cap and all(t >= 2 for t in c) or c == [cap]
        assert all(a == 2 * b or a == 2 * b + 1 for a, b in zip(c, c[1:]))


def test_save_load_round_trip(tmp_path):
    tiles = {(0, 384): 2, (1, 13): 24, (0, 64): 6}
    kernels = {(0, 384): "pair", (1, 2): "generic"}
    p = tmp_path / "tune.json"
    A.save(tiles, str(p), kernels)
    assert A.load(str(p)) == (tiles, kernels)
