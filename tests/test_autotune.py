"""The autotuner's search and its stored tunings, on synthetic cost
functions (no GPU): coordinate descent reaches the minimum of a separable
cost over every axis, skips invalid combinations, times each candidate
once; the batched search adds the path budget as an axis; tunings survive a
save / load round trip, and the package's tuned configurations load."""
import json

import pytest

from renderingengine_b200 import autotune as AT


class FakeRenderer:
    def __init__(self):
        self.calls = []

    def set_tuning(self, **kw):
        self.calls.append(kw)
        self.tuning = kw


def _cost(t: AT.Tuning) -> float:
    # Separable: traversal 5, block 256, shade 3, 4 CTAs per SM are best.
    return (abs(t.traversal - 5) + abs(t.block - 256) / 128 + abs(t.shade_variant - 3)
            + (0 if t.blocks_per_sm == 4 else 0.5) + (1 if t.fuse else 0) + t.refill / 8)


def test_coordinate_descent_finds_separable_minimum():
    timed = []

    def measure(t):
        timed.append(t)
        return _cost(t)

    best, results = AT.coordinate_descent(measure, AT.Tuning(), AT.DEFAULT_SPACE, passes=3)
    assert (best.traversal, best.block, best.shade_variant, best.blocks_per_sm) == (5, 256, 3, 4)
    assert not best.fuse and best.refill == 0
    assert best.ms_per_frame == pytest.approx(0.0)
    assert len(results) == len(timed)          # every candidate timed once
    assert all(AT.valid(t) for t in timed)


def test_validity_rules():
    assert AT.valid(AT.Tuning(fuse=True, traversal=0))
    assert not AT.valid(AT.Tuning(fuse=True, traversal=3))
    assert not AT.valid(AT.Tuning(fuse=True, traversal=0, refill=8))
    assert AT.valid(AT.Tuning(refill=8, traversal=4))
    assert AT.valid(AT.Tuning(refill=8, traversal=1))
    assert not AT.valid(AT.Tuning(refill=8, traversal=5))


def test_batched_search_sweeps_the_path_budget(tmp_path):
    r = FakeRenderer()
    seen = []

    def step(budget):
        t = r.tuning
        seen.append((budget, t["traversal"]))
        return abs(budget - (16 << 20)) / (1 << 20) + abs(t["traversal"] - 4)

    best, budget, results = AT.autotune_batched(r, step, (4 << 20, 8 << 20, 16 << 20, 32 << 20),
                                                {"traversal": (1, 3, 4, 5)}, store=tmp_path / "b.json")
    assert budget == 16 << 20 and best.traversal == 4
    stored = json.loads((tmp_path / "b.json").read_text())
    assert stored["budget"] == 16 << 20 and stored["workload"] == "batched"
    assert AT.load(tmp_path / "b.json") == AT.Tuning(**{k: v for k, v in stored["best"].items()})
    assert r.calls[-1]["traversal"] == 4       # the renderer is left at the best tuning


def test_save_load_round_trip(tmp_path):
    t = AT.Tuning(traversal=6, block=512, shade_variant=5, blocks_per_sm=4, ms_per_frame=7.0)
    AT.save(tmp_path / "t.json", t, "frame")
    assert AT.load(tmp_path / "t.json") == t
    bad = json.loads((tmp_path / "t.json").read_text())
    bad["best"]["fuse"] = True
    (tmp_path / "bad.json").write_text(json.dumps(bad))
    with pytest.raises(ValueError):
        AT.load(tmp_path / "bad.json")


def test_packaged_tunings_load():
    files = sorted(AT.TUNED_DIR.glob("*.json"))
    assert files, "no tuned configurations shipped"
    for f in files:
        t = AT.load(f.stem)
        assert AT.valid(t)
        r = FakeRenderer()
        AT.apply(r, t)
        assert r.calls[-1]["traversal"] == t.traversal
