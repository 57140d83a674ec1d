"""The autotuner's search and cache logic, on the host: a stand-in solver
scores each launch configuration with a synthetic cost, and the tuner must
find its minimum with the documented search (joint face-path search, joint
face-state search, then one knob at a time), record every trial, and serve
the result from its cache on the next call without measuring."""
import json

import pytest

from zoomy_dmplex_b200 import autotune
from zoomy_dmplex_b200.solver import LAUNCH_DEFAULTS


class FakeSolver:
    """Holds a launch configuration; a profiled step costs cost(config)."""

    def __init__(self, cost):
        self.h = object()
        self.cfg = dict(LAUNCH_DEFAULTS)
        self.cost = cost
        self.profiling = False
        self.steps = 0
        self.acc = 0.0

    def set_profiling(self, on):
        self.profiling = on
        self.acc = 0.0

    def step(self, n):
        self.steps += n
        if self.profiling:
            self.acc += n * self.cost(self.cfg)

    def read_profile(self):
        return {"prep": (0.6 * self.acc, 1), "flux": (0.4 * self.acc, 1)}


@pytest.fixture
def fake_launch(monkeypatch):
    def set_launch(h, cfg):
        fake_launch.solver.cfg = dict(cfg)

    def get_launch(h):
        return dict(fake_launch.solver.cfg)

    monkeypatch.setattr(autotune, "set_launch", set_launch)
    monkeypatch.setattr(autotune, "get_launch", get_launch)
    return fake_launch


# separable synthetic cost with its minimum away from the defaults
BEST = {"tile_faces": 128, "face": 64, "face_occ": 3, "prep_lean": 4, "prep": 64, "prep_occ": 8, "gather": 64,
        "finalize": 64, "finalize_occ": 4, "fuse_final": 1}


def cost(cfg):
    c = 1.0
    for k, v in BEST.items():
        vals = dict(autotune.KNOBS)[k]
        c += 0.1 * abs(vals.index(cfg[k]) - vals.index(v)) ** 2 + (0.01 if cfg[k] != v else 0.0)
    # a joint term: the face cap only pays at the best tile size
    if cfg["tile_faces"] == 128 and cfg["face_occ"] == 3:
        c -= 0.05
    return c


def test_tune_finds_the_minimum_and_caches(fake_launch, tmp_path):
    s = FakeSolver(cost)
    fake_launch.solver = s
    cache = str(tmp_path / "tuned.json")
    cfg = autotune.tune(s, "sme2d_l4", 3914402, steps=2, cache=cache)
    for k, v in BEST.items():
        assert cfg[k] == v, (k, cfg[k], v)
    assert s.cfg == cfg                       # applied to the solver
    knobs = dict(autotune.KNOBS)
    n_joint = len(knobs["tile_faces"]) * len(knobs["face"]) * len(knobs["face_occ"])
    n_prep = len(knobs["prep_lean"]) * len(knobs["prep_occ"])
    n_rest = sum(len(v) for k, v in autotune.KNOBS if k not in autotune.JOINT and k not in autotune.JOINT_PREP)
    assert len(autotune.last_trace) == n_joint + n_prep + n_rest
    assert all(t > 0 for _, _, t in autotune.last_trace)
    db = json.load(open(cache))
    key = autotune.cache_key("sme2d_l4", 3914402)
    assert db[key]["config"] == cfg and len(db[key]["trace"]) == len(autotune.last_trace)
    # a second call reads the cache and measures nothing
    s2 = FakeSolver(lambda c: pytest.fail("measured despite the cache"))
    fake_launch.solver = s2
    assert autotune.tune(s2, "sme2d_l4", 3914402, steps=2, cache=cache) == cfg
    assert s2.steps == 0 and s2.cfg == cfg
    # another size class is tuned afresh
    s3 = FakeSolver(cost)
    fake_launch.solver = s3
    autotune.tune(s3, "sme2d_l4", 114242, steps=1, cache=cache, write_cache=False)
    assert s3.steps > 0
    assert autotune.cache_key("sme2d_l4", 114242) not in json.load(open(cache))


def test_cache_key_buckets_sizes_by_powers_of_two():
    k = autotune.cache_key
    assert k("m", 65536) == k("m", 131071) != k("m", 131072)
    assert k("a", 1000) != k("b", 1000)


def test_knobs_cover_the_launch_keys():
    from zoomy_dmplex_b200.solver import LAUNCH_KEYS

    assert set(dict(autotune.KNOBS)) == set(LAUNCH_KEYS)
    for k, vals in autotune.KNOBS:
        assert LAUNCH_DEFAULTS[k] in vals


def test_unreadable_cache_is_retuned_and_rewritten(fake_launch, tmp_path):
    cache = tmp_path / "tuned.json"
    for junk in ("{not json", "[1, 2]"):
        cache.write_text(junk)
        assert autotune.load_cache(str(cache)) == {}
        s = FakeSolver(cost)
        fake_launch.solver = s
        cfg = autotune.tune(s, "sme2d_l2", 114242, steps=1, cache=str(cache))
        assert s.steps > 0
        assert json.load(open(cache))[autotune.cache_key("sme2d_l2", 114242)]["config"] == cfg
