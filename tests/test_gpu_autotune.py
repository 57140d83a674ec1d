"""The launch configuration changes scheduling and register allocation, not
arithmetic: the step is bit-identical under register caps 1, 4 and 8, block
sizes 64 and 128, the separate face + gather kernels and the fused tile
kernel at several tile sizes; the autotuner returns a configuration drawn
from its knobs, and the tuned step is bit-identical too."""
import numpy as np
import pytest

from zoomy_dmplex_b200 import autotune, cases, models
from zoomy_dmplex_b200.solver import BatchSolver, Solver, get_launch, set_launch

pytestmark = pytest.mark.gpu

CONFIGS = [
    {"prep": 128, "face": 128, "gather": 128, "finalize": 128, "prep_occ": 1, "face_occ": 1, "finalize_occ": 1,
     "tile_faces": 0},
    {"prep": 64, "face": 64, "gather": 64, "finalize": 64, "prep_occ": 4, "face_occ": 3, "finalize_occ": 3,
     "tile_faces": 0},
    {"prep": 128, "face": 128, "gather": 64, "finalize": 64, "prep_occ": 8, "face_occ": 4, "finalize_occ": 4,
     "tile_faces": 64},
    {"prep": 64, "face": 64, "gather": 128, "finalize": 128, "prep_occ": 4, "face_occ": 2, "finalize_occ": 2,
     "tile_faces": 128},
    {"prep": 128, "face": 128, "gather": 128, "finalize": 64, "prep_occ": 2, "face_occ": 3, "finalize_occ": 1,
     "tile_faces": 512},
    {"prep": 128, "face": 128, "gather": 128, "finalize": 64, "prep_occ": 8, "face_occ": 3, "finalize_occ": 4,
     "tile_faces": 0, "fuse_final": 1, "prep_lean": 4},
]


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


def _run(c, cfg, steps=12):
    g = Solver(c.model, c.mesh, c.settings, _params(c))
    if cfg is not None:
        set_launch(g.h, cfg)
    g.set_state(c.q0)
    g.step(steps)
    out = g.get_state(), g.time()
    g.close()
    return out


@pytest.mark.parametrize("make", [lambda: cases.level2(60), lambda: cases.roofline_l4(50),
                                  lambda: cases.mixed_level2(20), lambda: cases.plain_l0(40)])
def test_step_bit_identical_across_launch_configurations(make):
    c = make()
    ref_q, ref_t = _run(c, None)
    for cfg in CONFIGS:
        q, t = _run(c, cfg)
        assert np.array_equal(q, ref_q), cfg
        assert t == ref_t, cfg


def test_batch_bit_identical_fused_and_split():
    members = cases.ensemble(5, seed=11, side_range=(12, 40), processes=1)
    st = members[0].settings
    outs = []
    for tf in (0, 64, 256):
        b = BatchSolver(members[0].model, [c.mesh for c in members], st, [_params(c) for c in members])
        set_launch(b.h, dict(CONFIGS[1], tile_faces=tf))
        for i, c in enumerate(members):
            b.set_state(i, c.q0)
        b.step(15)
        outs.append([b.get_state(i) for i in range(len(members))])
        b.close()
    for o in outs[1:]:
        for a, r in zip(o, outs[0]):
            assert np.array_equal(a, r)


def test_autotune_returns_a_configuration_of_its_knobs():
    c = cases.level2(60)
    g = Solver(c.model, c.mesh, c.settings, _params(c))
    g.set_state(c.q0)
    cfg = autotune.tune(g, c.model, c.mesh.n_cells, steps=1, use_cache=False, write_cache=False)
    knobs = dict(autotune.KNOBS)
    for k, v in cfg.items():
        if k in knobs:
            assert v in knobs[k], (k, v)
    assert get_launch(g.h) == cfg
    g.set_state(c.q0)
    g.step(12)
    q = g.get_state()
    g.close()
    ref_q, _ = _run(c, None)
    assert np.array_equal(q, ref_q)
