"""Autotuner of the batched launch's tile size.

The tile (samples per work tile) sets how many consecutive samples of a
detector a CTA takes at a time: tile 1 spreads neighbouring samples over all
CTAs (they share the sky region in L2), larger tiles keep runs of samples on
one CTA (they share it in L1).  ``choose_tile`` times each
candidate on the actual batch with CUDA events (two launches each, best
kept) and caches the winner in a JSON file keyed by GPU, nside, map type,
interpolation mode, detector count and sample/beam-pixel scale, so later runs
with the same shape reuse it.  The cache lives at ``$TODGPU_AUTOTUNE_CACHE``
(default ``~/.cache/todgpu/autotune.json``).
"""

from __future__ import annotations

import json
import math
import os

import torch

CANDIDATES = (1, 4, 16, 64, 256)


def cache_path():
    return os.environ.get("TODGPU_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "todgpu", "autotune.json"))


def _key(batch):
    name = torch.cuda.get_device_name(torch.cuda.current_device()).replace(" ", "_")
    mt = getattr(batch.map, "kind", None) or str(batch.map.dtype).replace("torch.", "")
    s_mean = batch.n_evals / max(1, batch.n_samples)
    return (f"{name}|nside{batch.nside}|{mt}|interp{batch.interp}|qu{int(batch.c_q >= 0)}|"
            f"det{len(batch.vec)}|n2^{round(math.log2(max(1, batch.n_samples)))}|"
            f"S2^{round(math.log2(max(1.0, s_mean)))}")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only disables the cache


def choose_tile(batch, candidates=CANDIDATES, use_cache=True, timing_batch=None):
    """Tile size with the shortest launch for ``batch`` (cached under the
    batch's key).  ``timing_batch`` (e.g. ``batch.truncated(1 / 16)``) is
    timed instead of the batch itself when given."""
    key = _key(batch)
    cache = _load() if use_cache else {}
    if key in cache:
        return int(cache[key]["tile"])
    if timing_batch is not None:
        batch = timing_batch
    stream = torch.cuda.current_stream()
    timings = {}
    for t in candidates:
        best = float("inf")
        for _ in range(2):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.launch(t)
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        timings[t] = best
    tile = min(timings, key=timings.get)
    if use_cache:
        cache[key] = {"tile": tile, "ms": {str(k): round(v, 3) for k, v in timings.items()}}
        _store(cache)
    return tile
