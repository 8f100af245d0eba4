"""Schedule autotuner.

Searches the engine's schedule knobs (glu_tuning: work threshold that sends a
level to its own launch, cluster size of the narrow-level kernel, lanes per
update item, smallest dense trailing block) by timing real factorizations on
the device, and caches the winner per (pattern hash, GPU name) in a JSON file.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os

import numpy as np

from . import _capi

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "glu_b200", "tune.json")


def _pattern_key(an):
    h = hashlib.sha1()
    h.update(np.asarray(an.pap).tobytes())
    h.update(np.asarray(an.pai).tobytes())
    return h.hexdigest()[:16]


def _gpu_name():
    try:
        import torch

        return torch.cuda.get_device_name(0)
    except Exception:  # pragma: no cover
        return "unknown"


def _get(handle):
    t = _capi.Tuning()
    _capi.check(_capi.engine().glu_get_tuning(handle, _capi.C.byref(t)), "get tuning")
    return t


def _set(handle, cfg):
    t = _get(handle)
    for k, v in cfg.items():
        setattr(t, k, v)
    _capi.check(_capi.engine().glu_set_tuning(handle, _capi.C.byref(t)), "set tuning")


def candidates():
    """The search space (small grid)."""
    grid = dict(wide_work=[50_000, 200_000, 1_000_000], chain_cluster=[8, 16], group_lanes=[0, 8, 32])
    keys = list(grid)
    for vals in itertools.product(*(grid[k] for k in keys)):
        yield dict(zip(keys, vals))


def tune(lu, data=None, repeats=3, cache=DEFAULT_CACHE, space=None, use_cache=True):
    """Pick the fastest schedule for ``lu`` (a GLUFactorization or BatchedGLU).

    ``data`` are the values to factor while timing (default: the analysed
    ones).  Returns (best_config, best_ms).  The handle keeps the winner.
    """
    an = lu._an
    h = lu.handle
    key = f"{_pattern_key(an)}:{_gpu_name()}:{getattr(lu, 'batch', 1)}"
    if use_cache and cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                db = json.load(f)
            if key in db:
                _set(h, db[key]["config"])
                lu.refactor(an.data if data is None else data) if getattr(lu, "batch", 1) == 1 else None
                return db[key]["config"], db[key]["ms"]
        except (OSError, ValueError):
            pass
    values = an.data if data is None else data
    best, best_ms = None, float("inf")
    for cfg in (space if space is not None else candidates()):
        try:
            _set(h, cfg)
        except ValueError:
            continue
        times = []
        for _ in range(repeats):
            if getattr(lu, "batch", 1) == 1:
                lu.refactor(values)
            else:
                lu.refactor(values)
            times.append(lu.stats["last_factor_ms"])
        ms = float(np.median(times))
        if ms < best_ms:
            best, best_ms = cfg, ms
    _set(h, best)
    if getattr(lu, "batch", 1) == 1:
        lu.refactor(values)
    else:
        lu.refactor(values)
    if cache:
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            db = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    db = json.load(f)
            db[key] = dict(config=best, ms=best_ms)
            with open(cache, "w") as f:
                json.dump(db, f, indent=1)
        except (OSError, ValueError):
            pass
    return best, best_ms
