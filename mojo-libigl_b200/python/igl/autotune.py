"""Autotuner for the batched launch: the tile shape (faces per tile, queries per
thread), the work-item size, persistent CTAs per SM and the refinement radius
kappa.

``tune(meshes, queries)`` times candidates on a query subsample of the batch
(at most ``sample_queries`` per mesh, so a candidate costs tens of ms),
forward + backward by default, with CUDA events after a warm-up, and returns
the fastest configuration. The search is a coordinate descent from the default
configuration: each dimension in turn is swept with the others fixed at the
best so far, and the sweep repeats until a full pass changes nothing (at most
``passes`` times); ``search="grid"`` times the whole product instead. Results
are cached in a JSON file keyed by GPU name, mesh count, size buckets and the
search space: ``$WN_AUTOTUNE_CACHE`` or ``~/.cache/wn_b200/autotune.json``.
kappa only ranges over values whose error bound holds (>= 3; see wn_mixed.cu),
and 32- and 64-face tiles keep the same bound, so the choice trades speed, not
accuracy beyond the tested bound.
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
    "tile_faces": (64, 32),
    "qpt": (2, 1, 4),
    "target_pairs": (1 << 23, 1 << 21),
    "ctas_per_sm": (0, 2),
    "kappa": (4.0, 3.0),
}
# The first value of each dimension is the starting point of the descent.


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
         reps: int = 3, use_cache: bool = True, seed: int = 0, search: str = "descent",
         passes: int = 2) -> dict:
    """Return {"config": {...}, "ms": ..., "trials": [...], "cached": bool}."""
    if search not in ("descent", "grid"):
        raise ValueError("search must be 'descent' or 'grid'")
    space = space or DEFAULT_SPACE
    key = (cache_key(meshes, queries) + f"|bwd={int(backward)}|{search}|" +
           ",".join(f"{k}={list(v)}" for k, v in space.items()))
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
    trials = []
    timed = {}

    def measure(cfg: dict) -> float:
        k = tuple(sorted(cfg.items()))
        if k not in timed:
            batch = Batch(meshes, sample, **cfg)
            try:
                batch.gW.normal_()
                timed[k] = _time(batch, backward, reps)
            finally:
                batch.close()
            trials.append({"config": dict(cfg), "ms": timed[k]})
        return timed[k]

    if search == "grid":
        for values in itertools.product(*space.values()):
            measure(dict(zip(space.keys(), values)))
    else:
        cfg = {k: v[0] for k, v in space.items()}
        best = measure(cfg)
        for _ in range(max(1, passes)):
            changed = False
            for dim, values in space.items():
                for v in values:
                    cand = dict(cfg, **{dim: v})
                    ms = measure(cand)
                    if ms < best:
                        best, cfg, changed = ms, cand, True
            if not changed:
                break
    best_trial = min(trials, key=lambda t: t["ms"])
    result = {"config": best_trial["config"], "ms": best_trial["ms"], "trials": trials,
              "key": key, "search": search}
    if use_cache:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        cache[key] = result
        tmp = f"{path}.{os.getpid()}.tmp"  # one per process: ranks may tune at once
        with open(tmp, "w") as fh:
            json.dump(cache, fh, indent=1)
        os.replace(tmp, path)
    return dict(result, cached=False)
