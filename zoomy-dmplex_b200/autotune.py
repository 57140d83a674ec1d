"""Launch-configuration autotuner.

The knobs are the threads per block of the four step kernels and register
caps (resident blocks per SM) of the two register-heavy ones; every kernel
is timed with the library's CUDA-event profiling (zsme_set_profiling), so
each knob is tuned against the time of the kernel it affects (coordinate
descent, one knob at a time).  Results are cached in a JSON file keyed by
GPU, model and mesh size.

Tuning advances the solver's state: call it right after set_state and load
the initial state again afterwards (``reset``).
"""
from __future__ import annotations

import json
import os

from . import native
from .solver import LAUNCH_KEYS, get_launch, set_launch

KNOBS = (("prep", (64, 128)), ("prep_occ", (1, 2, 3, 4, 6, 8)), ("face", (64, 128)), ("face_occ", (1, 2, 3, 4)),
         ("gather", (64, 128)), ("finalize", (64, 128)), ("finalize_occ", (1, 2, 3, 4)))
KERNEL_OF = {"prep": "prep", "prep_occ": "prep", "face": "flux", "face_occ": "flux", "gather": "gather",
             "finalize": "finalize", "finalize_occ": "finalize"}
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
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _measure(solver, cfg, steps):
    set_launch(solver.h, cfg)
    solver.set_profiling(True)
    solver.step(steps)
    prof = solver.read_profile() if hasattr(solver, "read_profile") else _read(solver)
    solver.set_profiling(False)
    return {k: (ms / n if n else float("inf")) for k, (ms, n) in prof.items()}


def _read(solver):
    import ctypes as ct
    import numpy as np
    k = len(native.KERNEL_KINDS)
    ms = np.zeros(k)
    n = (ct.c_int64 * k)()
    native.check(solver.lib.zsme_read_profile(solver.h, ms.ctypes.data_as(ct.POINTER(ct.c_double)), n))
    return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(native.KERNEL_KINDS)}


def tune(solver, model, n_cells, steps=2, cache=DEFAULT_CACHE, use_cache=True, write_cache=True):
    """Pick and apply the fastest launch configuration; returns it (dict)."""
    key = cache_key(model, n_cells)
    db = load_cache(cache) if use_cache else {}
    if key in db:
        cfg = db[key]["config"]
        set_launch(solver.h, cfg)
        return cfg
    cfg = get_launch(solver.h)
    _measure(solver, cfg, 1)                       # warm-up
    trace = []
    for knob, values in KNOBS:
        best_v, best_t = cfg[knob], None
        for v in values:
            trial = dict(cfg)
            trial[knob] = v
            t = _measure(solver, trial, steps)[KERNEL_OF[knob]]
            trace.append((knob, v, t))
            if best_t is None or t < best_t:
                best_v, best_t = v, t
        cfg[knob] = best_v
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
