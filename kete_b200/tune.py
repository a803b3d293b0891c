"""Launch-configuration autotuner for the N-body kernels.

The node-parallel Radau kernel comes in three register budgets (no cap, 168 registers for
3 blocks/SM, 128 registers for 4 blocks/SM: more resident lane groups against spills to
local memory), each with or without the step-end lane (variants 3-5: the eighth lane
evaluates the step end during every corrector iteration instead of a separate round;
variants 6-8 add warp-synchronous step starts with the bodies' positions cached across a
step's corrector iterations; variants 9 and 10, at 168 and 128 registers, keep the cache but
let the warp's four objects step independently and share every round's ephemeris-record
evaluations across all 32 lanes) and in two grid forms (one lane group per object, or a
persistent grid whose groups take the next object from a queue).  Which is fastest depends on the object
count and the spread of their step counts, so it is measured: ``autotune`` times every
configuration on the caller's own inputs (device arrays) and installs the fastest.
"""
from __future__ import annotations

import ctypes
import itertools
import json
import os

from . import _lib
from .propagation import propagate_n_body_arrays

CONFIGS = [dict(mode=_lib.MODE_NODES, variant=v, refill=r) for v, r in
           itertools.product((0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10), (0, 1))] + [
               dict(mode=_lib.MODE_THREAD, variant=0, refill=0)]
_current = dict(mode=_lib.MODE_NODES, variant=7, refill=0, thread_block=128)


def set_config(mode=_lib.MODE_NODES, variant=7, refill=0, thread_block=128):
    L = _lib.lib()
    L.kete_b200_set_launch_config.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    _lib.check(L.kete_b200_set_launch_config(int(variant), int(refill), int(thread_block)))
    _current.update(mode=mode, variant=variant, refill=refill, thread_block=thread_block)


def set_step_limit(max_steps: int = 0):
    """Bound each object's Radau step loop (kete_b200_set_step_limit): an object that has not
    reached its target epoch after ``max_steps`` step attempts gets the Timeout status and a
    NaN state.  0 restores the default bound."""
    L = _lib.lib()
    L.kete_b200_set_step_limit.argtypes = [ctypes.c_int64]
    _lib.check(L.kete_b200_set_step_limit(int(max_steps)))


def current():
    return dict(_current)


def _time_config(cfg, pos, vel, jd0, jd1, nongrav, reps):
    import torch

    set_config(**cfg)
    propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=nongrav, mode=cfg["mode"])  # warm
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=nongrav, mode=cfg["mode"])
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _label(cfg):
    return f"mode{cfg['mode']}_v{cfg['variant']}_r{cfg['refill']}"


def autotune(pos, vel, jd0, jd1, nongrav=None, reps=2, cache_path=None, key=None,
             full=None, finalists=3, within=0.05):
    """Time each configuration on these (torch CUDA) inputs; install and return the best.

    ``full``: when the inputs are a sample of a larger population, that population's
    (pos, vel, jd0, jd1, nongrav).  The configurations within ``within`` of the sample's best
    (at most ``finalists`` of them) are then timed again on it and the fastest there wins:
    on a persistent grid the sample's tail of last objects weighs more than in the full
    launch, which favours the variants with fewer resident lane groups.

    Returns (best_config, {label: ms}); the re-timed finalists appear as ``<label>_full``."""

    if cache_path and key and os.path.exists(cache_path):
        with open(cache_path) as f:
            cached = json.load(f).get(key)
        if cached:
            set_config(**cached["best"])
            return cached["best"], cached["times"]
    times = {}
    best, best_ms = None, float("inf")
    for cfg in CONFIGS:
        ms = _time_config(cfg, pos, vel, jd0, jd1, nongrav, reps)
        times[_label(cfg)] = ms
        if ms < best_ms:
            best, best_ms = dict(cfg), ms
    if full is not None:
        ranked = sorted(CONFIGS, key=lambda c: times[_label(c)])
        close = [c for c in ranked if times[_label(c)] <= best_ms * (1.0 + within)][:finalists]
        if len(close) > 1:
            best_ms = float("inf")
            for cfg in close:
                ms = _time_config(cfg, *full, reps)
                times[_label(cfg) + "_full"] = ms
                if ms < best_ms:
                    best, best_ms = dict(cfg), ms
    set_config(**best)
    if cache_path and key:
        data = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                data = json.load(f)
        data[key] = {"best": best, "times": times}
        with open(cache_path, "w") as f:
            json.dump(data, f, indent=1)
    return best, times
