"""The autotuner's search (xbtrav.autotune), on the CPU: a fake context and a
fake timer stand in for the engine, so the tests see which configurations the
staged and the full search time and which one they keep."""
import pytest

from xbtrav import autotune


class FakeCtx:
    device = 0

    def __init__(self):
        self.t = dict(word_bits=64, words=4, pull_alpha=256.0, heavy_degree=256, timing=0, chains=4, level_cap=0,
                      tile=0, workspace_cap=0, push_beta=0.0, source_order=0)

    def tuning(self):
        return dict(self.t)

    def set_tuning(self, **kw):
        self.t.update(kw)


# the cost surface: a separable bowl with its minimum at one point of the space
BEST = dict(word_bits=64, words=2, heavy_degree=512, pull_alpha=1024.0, push_beta=24.0, tile=1, source_order=1,
            chains=8)


def _cost(cfg):
    c = 10.0
    for k, v in BEST.items():
        c += 0.0 if cfg.get(k) == v else 1.0
    return c


@pytest.fixture
def timed(monkeypatch):
    calls = []

    def fake(ctx, graph, sources, cfg, reps, path):
        calls.append((dict(cfg), path))
        return _cost(cfg)

    monkeypatch.setattr(autotune, "_time_config", fake)
    return calls


def test_staged_search_finds_a_separable_optimum(timed):
    ctx = FakeCtx()
    best, table = autotune.autotune(ctx, None, [0], path="batched")
    assert best == {k: BEST[k] for k in autotune.KEYS}
    assert {k: ctx.tuning()[k] for k in best} == best  # the context keeps the winner
    sp = autotune.DEFAULT_SPACE
    stages = (len(sp["word_bits"]) * len(sp["words"]) + len(sp["heavy_degree"]) * len(sp["pull_alpha"])
              + len(sp["push_beta"]) + len(sp["tile"]) + len(sp["source_order"]) + len(sp["chains"]))
    assert len(table) == stages == len(timed)


def test_plain_path_keeps_the_chain_count(timed):
    ctx = FakeCtx()
    best, _ = autotune.autotune(ctx, None, [0], path="plain")
    assert best["chains"] == 4  # chains only matter to the batched path
    assert all(p == "plain" for _, p in timed)
    assert {c["chains"] for c, _ in timed} == {4}


def test_full_grid_times_every_point(timed):
    ctx = FakeCtx()
    space = dict(word_bits=[64], words=[2, 4], heavy_degree=[256, 512], pull_alpha=[1024.0], push_beta=[0.0],
                 tile=[0, 1], source_order=[0, 1], chains=[8])
    best, table = autotune.autotune(ctx, None, [0], space=space, staged=False, path="batched")
    assert len(table) == 2 * 2 * 2 * 2
    assert best["words"] == 2 and best["heavy_degree"] == 512 and best["tile"] == 1 and best["source_order"] == 1


def test_save_and_load_round_trip(tmp_path, timed):
    ctx = FakeCtx()
    best, _ = autotune.autotune(ctx, None, [0], path="batched")
    p = tmp_path / "t.json"
    autotune.save(best, str(p))
    assert autotune.load(str(p)) == best
