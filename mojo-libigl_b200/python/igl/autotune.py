"""Autotuner for the batched launch: queries per thread, work-item size,
persistent CTAs per SM and the refinement radius kappa.

``tune(meshes, queries)`` times every candidate on a query subsample of the
batch (at most ``sample_queries`` per mesh, so a candidate costs tens of ms),
forward + backward by default, with CUDA events after a warm-up, and returns
the fastest configuration. Results are cached in a JSON file keyed by GPU name,
mesh count and size buckets: ``$WN_AUTOTUNE_CACHE`` or
``~/.cache/wn_b200/autotune.json``. kappa only ranges over values whose error
bound holds (>= 3; see wn_mixed.cu), so the choice trades speed, not accuracy
beyond the tested bound.
"""

from __future__ import annotations

import itertools
import json
import math
import os

import numpy as np
import torch

from .batched import Batch

DEFAULT_SPACE = {
    "qpt": (1, 2, 4),
    "target_pairs": (1 << 21, 1 << 23),
    "ctas_per_sm": (0,),
    "kappa": (3.0, 4.0),
}


def cache_path() -> str:
    return os.environ.get("WN_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "wn_b200", "autotune.json")


def _bucket(x: float) -> int:
    return int(round(math.log2(max(x, 1.0))))


def cache_key(meshes, queries) -> str:
    nf = np.array([len(F) for _, F in meshes], dtype=np.float64)
    nq = np.array([len(O) for O in queries], dtype=np.float64)
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return (f"{name}|meshes={len(meshes)}|faces~2^{_bucket(nf.sum())}|"
            f"queries~2^{_bucket(nq.sum())}|pairs~2^{_bucket((nf * nq).sum())}")


def _time(batch: Batch, backward: bool, reps: int) -> float:
    batch.step(backward)
    torch.cuda.synchronize()
    best = math.inf
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.step(backward)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune(meshes, queries, space=None, backward: bool = True, sample_queries: int = 16384,
         reps: int = 3, use_cache: bool = True, seed: int = 0) -> dict:
    """Return {"config": {...}, "ms": ..., "trials": [...], "cached": bool}."""
    key = cache_key(meshes, queries) + f"|bwd={int(backward)}"
    path = cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except (OSError, ValueError):
            cache = {}
        if key in cache:
            return dict(cache[key], cached=True)
    rng = np.random.default_rng(seed)
    sample = [O if len(O) <= sample_queries else O[rng.choice(len(O), sample_queries,
                                                               replace=False)]
              for O in queries]
    space = space or DEFAULT_SPACE
    trials = []
    for values in itertools.product(*space.values()):
        cfg = dict(zip(space.keys(), values))
        batch = Batch(meshes, sample, **cfg)
        try:
            batch.gW.normal_()
            ms = _time(batch, backward, reps)
        finally:
            batch.close()
        trials.append({"config": cfg, "ms": ms})
    best = min(trials, key=lambda t: t["ms"])
    result = {"config": best["config"], "ms": best["ms"], "trials": trials, "key": key}
    if use_cache:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        cache[key] = result
        tmp = f"{path}.{os.getpid()}.tmp"  # one per process: ranks may tune at once
        with open(tmp, "w") as fh:
            json.dump(cache, fh, indent=1)
        os.replace(tmp, path)
    return dict(result, cached=False)
