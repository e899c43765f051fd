"""Autotuner for the batched form's tile shape.

For a planned-able Batch, every compiled tile configuration that fits the
batch's widest taps is planned and timed (CUDA events, a few launches after a
warm-up); the fastest is chosen and cached in a JSON file keyed by the GPU
name, the storage type and a signature of the batch (instance count and the
histogram of (rank, tap widths)).  A later batch with the same key reuses the
cached choice without timing.

    cfg = best_tile_config(batch)     # plans the batch with the winner
"""
from __future__ import annotations

import hashlib
import json
import os

import torch

from . import abi
from .batch import tile_configs

CACHE = os.environ.get("NDLGPU_AUTOTUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "ndlgpu", "batch_tiles.json"))


def _key(batch):
    hist = {}
    for rank, _ext, taps, border, adj, dt in batch.signature:
        k = "%d:%s:%d:%d:%s" % (rank, ",".join(str(t) for t in taps), border, int(adj), dt)
        hist[k] = hist.get(k, 0) + 1
    sig = json.dumps(sorted(hist.items()))
    name = torch.cuda.get_device_name()
    return "%s|%d|%s" % (name, len(batch.signature), hashlib.sha1(sig.encode()).hexdigest()[:16])


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except Exception:
        return {}


def _save(db):
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        tmp = CACHE + ".tmp"
        with open(tmp, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE)
    except OSError:
        pass


def time_config(batch, cfg, iters=5, warm=2):
    batch.plan(cfg)
    for _ in range(warm):
        batch.launch()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(iters):
        batch.launch()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / iters


def best_tile_config(batch, use_cache=True, iters=5):
    """Plans `batch` with the fastest tile configuration; returns
    (config index, {config: ms})."""
    key = _key(batch)
    db = _load() if use_cache else {}
    if key in db:
        cfg = int(db[key]["config"])
        batch.plan(cfg)
        return cfg, db[key].get("times", {})
    times = {}
    for cfg in range(len(tile_configs())):
        try:
            times[cfg] = time_config(batch, cfg, iters)
        except abi.NdlGpuError:
            continue          # does not fit this batch's widest taps
    if not times:
        raise RuntimeError("no tile configuration fits this batch")
    best = min(times, key=times.get)
    batch.plan(best)
    if use_cache:
        db[key] = {"config": best, "times": {str(k): v for k, v in times.items()}}
        _save(db)
    return best, times
