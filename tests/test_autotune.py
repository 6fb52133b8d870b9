"""The tile-shape autotuner's host logic (no GPU): candidate enumeration, cache keys
and the cache round trip, with a stand-in context that times nothing."""
import json

from imau_ice_b200 import autotune, diva


def test_candidates_cover_every_assignment_of_the_tiled_levels():
    c = list(autotune.candidates([32, 16, 0, 0]))
    assert len(c) == 4 and [16, 16, 0, 0] in c and [32, 32, 0, 0] in c
    assert list(autotune.candidates([0, 0, 0])) == [[0, 0, 0]]


class FakeCtx:
    """Times a V-cycle as 1 ms per level of edge 16 and 2 ms per level of edge 32."""

    def __init__(self):
        self.grid = diva.Grid(321, 561, 5e3)
        self.cfg = type("Cfg", (), {"precision": 0, "choice_ice_margin": 0})()
        self.edges, self.calls = [], 0

    def nonlinear_residual(self):
        return 0.0

    def set_tile_edges(self, e):
        self.edges = list(e)

    def get_tile_edges(self):
        return [32, 16, 0, 0] if not any(self.edges) else list(self.edges)

    def profile_kernel(self, which, reps):
        assert which == 3
        self.calls += 1
        return sum(1.0 if e == 16 else 2.0 if e == 32 else 0.0 for e in self.edges), 0.0


def test_tuner_picks_the_fastest_and_caches_it(tmp_path):
    ctx = FakeCtx()
    cache = str(tmp_path / "tiles.json")
    best, t = autotune.tune_tile_edges(ctx, reps=1, trials=1, cache=cache)
    assert best == [16, 16, 0, 0] and ctx.edges == best and len(t) == 4
    assert json.load(open(cache)) == {autotune.cache_key(ctx): best}
    ctx2 = FakeCtx()
    best2, t2 = autotune.tune_tile_edges(ctx2, cache=cache)
    assert best2 == best and ctx2.calls == 0 and ctx2.edges == best


def test_other_backends_are_left_alone():
    ctx = FakeCtx()
    ctx.backend = type("B", (), {"name": "oracle"})()
    assert autotune.tune_tile_edges(ctx) == ([], {}) and ctx.calls == 0 and ctx.edges == []
