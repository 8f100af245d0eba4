"""Schedule autotuner.

The reference fixes its schedule in code: a level's columns go to blocks of
2, 4 or 32 warps by level size (896 / 448 / 16 thresholds) and narrow levels
spread over 16 streams (src/numeric.cu:390, 557-565).  Here the engine's
schedule knobs (glu_tuning) are chosen per pattern by timing real
factorizations on the device, and the winner is cached per (pattern, GPU,
batch) in a JSON file.

Search: coordinate descent from the engine's defaults over the knobs the
factorization path in use reads --

* supernodal path (sn_width > 0, the default): widest supernode, grouping of
  small supernodes into warps, the split between sparse part and dense
  trailing block (the cost model's dense rate and the largest buffered
  block), the width from which the dense block takes its panels in
  look-ahead groups and the panels per group, the width from which it
  updates on the tensor cores,
  how many of the sparse part's updates of the dense block are deferred to
  tensor-core products after the sparse part;
* column path (sn_width = 0): lanes per update, the cluster size of the
  narrow-level kernel, the work that sends a level to its own launch;
* batched handles, in addition: the batch tile, the number of value sets one
  supernode-update block applies its tile to.

Each knob takes its values in turn with the others held; the fastest
refactorization (median of ``repeats``) is kept; two passes.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from . import _capi

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "glu_b200", "tune.json")

# values tried per knob (the engine's default is always tried first)
SUPERNODAL_SPACE = {
    "sn_width": [16, 32, 64],
    "sn_small": [0, 1],
    "dense_rate": [0, 15_000, 60_000, 250_000],
    "dense_tail_max": [2048, 4096, 8192],
    "dense_lookahead": [0, 1024, 3072],
    "dense_tc_min": [0, 512, 1024, 2048],
    "defer_tail": [0, 1, 4],
    "dense_group": [2, 3, 4],
}
COLUMN_SPACE = {
    "group_lanes": [0, 8, 32],
    "chain_cluster": [8, 16],
    "wide_work": [50_000, 200_000, 1_000_000],
}


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


def current(handle):
    """The handle's schedule knobs as a dict."""
    t = _get(handle)
    return {k: getattr(t, k) for k, _ in _capi.Tuning._fields_}


def _time(lu, values, repeats):
    times = []
    for _ in range(repeats):
        lu.refactor(values)
        times.append(lu.stats["last_factor_ms"])
    return float(np.median(times))


# the batch tile (value sets per supernode-update block), for batched handles
BATCH_SPACE = {"batch_tile": [0, 1, 2, 4, 8, 16]}


def _space_for(cfg, space, batch=1):
    if space is not None:
        return space
    base = SUPERNODAL_SPACE if cfg.get("sn_width", 1) else COLUMN_SPACE
    return {**base, **BATCH_SPACE} if batch > 1 else base


def tune(lu, data=None, repeats=3, cache=DEFAULT_CACHE, space=None, use_cache=True, passes=2):
    """Pick the fastest schedule for ``lu`` (a GLUFactorization or BatchedGLU).

    ``data`` are the values to factor while timing (default: the analysed
    ones; for a batch, its value array).  ``space`` overrides the knob grid
    (a dict knob -> list of values).  Returns (best_config, best_ms,
    report) where report holds the default's time and every trial; the handle
    keeps the winner and is left factored with ``data``.
    """
    an = lu._an
    h = lu.handle
    batch = getattr(lu, "batch", 1)
    values = (an.data if data is None else data) if batch == 1 else data
    if values is None:
        raise ValueError("a batch needs its value sets to time")
    key = f"{_pattern_key(an)}:{_gpu_name()}:{batch}"
    if use_cache and cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                db = json.load(f)
            if key in db:
                _set(h, db[key]["config"])
                lu.refactor(values)
                return db[key]["config"], db[key]["ms"], {"cached": True}
        except (OSError, ValueError):
            pass
    base = current(h)
    best = dict(base)
    best_ms = _time(lu, values, repeats)
    report = {"default_ms": best_ms, "trials": [], "cached": False}
    grid = _space_for(base, space, batch)
    for _ in range(passes):
        improved = False
        for knob, choices in grid.items():
            for v in choices:
                if v == best.get(knob):
                    continue
                cfg = dict(best)
                cfg[knob] = v
                try:
                    _set(h, cfg)
                except (ValueError, _capi.GLUError):
                    continue
                ms = _time(lu, values, repeats)
                report["trials"].append((knob, v, ms))
                if ms < best_ms:
                    best, best_ms, improved = cfg, ms, True
        if not improved:
            break
    _set(h, best)
    lu.refactor(values)
    changed = {k: v for k, v in best.items() if base.get(k) != v}
    report["changed"] = changed
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
    return best, best_ms, report
