"""Launch-configuration autotuner.

The knobs are the threads per block of the step kernels, the register caps
(resident blocks per SM) of the register-heavy ones, and the tile size of
the fused face + gather kernel (tile_faces; 0 runs the separate face and
gather kernels).  Each trial runs a few profiled steps (zsme_set_profiling,
one CUDA-event pair per launch) and is scored by the summed time of all the
step's kernels.  The tile size, the face block size and the face register
cap are searched together first (they decide which kernels the others act
on, and each other's occupancy); the other knobs are then set one at a time
(coordinate descent).  Results are cached in a JSON file keyed by GPU, model
and mesh size.

Tuning advances the solver's state: call it right after set_state and load
the initial state again afterwards (``reset``).  Every configuration gives
the same results bit for bit (tests/test_gpu_autotune.py): the knobs change
scheduling and register allocation, not arithmetic.
"""
from __future__ import annotations

import json
import os

from . import native
from .solver import LAUNCH_KEYS, get_launch, set_launch

KNOBS = (("tile_faces", (0, 64, 128, 256, 512)), ("face", (64, 128)), ("face_occ", (1, 2, 3, 4)),
         ("prep_lean", (0, 1, 2, 3, 4)), ("prep", (64, 128)), ("prep_occ", (1, 2, 3, 4, 6, 8)), ("gather", (64, 128)),
         ("finalize", (64, 128)), ("finalize_occ", (1, 2, 3, 4)), ("fuse_final", (0, 1)))
# searched together first: which face path, its block size and its register cap
# decide each other's worth (the fused kernel's shared memory per block is fixed
# by its tile size, so its occupancy depends on all three)
JOINT = ("tile_faces", "face", "face_occ")
# then the face-state kernel's form with its register cap (a split form runs
# more threads per cell with fewer registers each, so the cap worth having
# depends on the form)
JOINT_PREP = ("prep_lean", "prep_occ")
DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_launch.json")


def _gpu_name():
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def cache_key(model, n_cells):
    bucket = 1 << max(0, int(n_cells).bit_length() - 1)   # power-of-two size class
    return "%s|%s|%d" % (_gpu_name(), model, bucket)


def load_cache(path=DEFAULT_CACHE):
    """The cached tunings ({} when the file is missing, unreadable or not a
    JSON object: the tuner then measures afresh and rewrites it)."""
    try:
        with open(path) as f:
            db = json.load(f)
    except (OSError, ValueError):
        return {}
    return db if isinstance(db, dict) else {}


def _measure(solver, cfg, steps):
    """Summed device time (ms) of every kernel over `steps` profiled steps."""
    set_launch(solver.h, cfg)
    solver.set_profiling(True)
    solver.step(steps)
    prof = solver.read_profile() if hasattr(solver, "read_profile") else _read(solver)
    solver.set_profiling(False)
    return sum(ms for ms, n in prof.values())


def _read(solver):
    import ctypes as ct
    import numpy as np
    k = len(native.KERNEL_KINDS)
    ms = np.zeros(k)
    n = (ct.c_int64 * k)()
    native.check(solver.lib.zsme_read_profile(solver.h, ms.ctypes.data_as(ct.POINTER(ct.c_double)), n))
    return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(native.KERNEL_KINDS)}


last_trace = []   # (knob, value, summed kernel ms) of the last tuning run


def tune(solver, model, n_cells, steps=2, cache=DEFAULT_CACHE, use_cache=True, write_cache=True):
    """Pick and apply the fastest launch configuration; returns it (dict).
    The trials of the run are left in last_trace."""
    global last_trace
    key = cache_key(model, n_cells)
    db = load_cache(cache) if use_cache else {}
    if key in db:
        cfg = db[key]["config"]
        set_launch(solver.h, cfg)
        return cfg
    cfg = get_launch(solver.h)
    _measure(solver, cfg, 1)                       # warm-up
    trace = []
    values = dict(KNOBS)
    best, best_t = None, None
    for tf in values["tile_faces"]:                # tile size outermost: the tiles are rebuilt per size
        for fb in values["face"]:
            for fo in values["face_occ"]:
                trial = dict(cfg, tile_faces=tf, face=fb, face_occ=fo)
                t = _measure(solver, trial, steps)
                trace.append(("tile_faces/face/face_occ", (tf, fb, fo), t))
                if best_t is None or t < best_t:
                    best, best_t = (tf, fb, fo), t
    cfg.update(dict(zip(JOINT, best)))
    best, best_t = None, None
    for pl in values["prep_lean"]:
        for po in values["prep_occ"]:
            trial = dict(cfg, prep_lean=pl, prep_occ=po)
            t = _measure(solver, trial, steps)
            trace.append(("prep_lean/prep_occ", (pl, po), t))
            if best_t is None or t < best_t:
                best, best_t = (pl, po), t
    cfg.update(dict(zip(JOINT_PREP, best)))
    for knob, values in KNOBS:
        if knob in JOINT or knob in JOINT_PREP:
            continue
        best_v, best_t = cfg[knob], None
        for v in values:
            trial = dict(cfg)
            trial[knob] = v
            t = _measure(solver, trial, steps)
            trace.append((knob, v, t))
            if best_t is None or t < best_t:
                best_v, best_t = v, t
        cfg[knob] = best_v
    last_trace = trace
    set_launch(solver.h, cfg)
    if write_cache:
        db = load_cache(cache)
        db[key] = {"config": cfg, "trace": trace}
        try:
            with open(cache, "w") as f:
                json.dump(db, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return cfg
