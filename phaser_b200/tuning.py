"""Persistent cache of autotuned launch parameters (phgpu_autotune) per shape
and device model.

The cache is a JSON file (PHGPU_TUNING_CACHE, or ~/.cache/phaser_b200/
tuning.json) mapping a shape key -- device name, library build, bandwidth,
spherical zero padding, voxels, precision -- to the parameters and the
registration time the search measured under them.  The build is part of the
key because a kernel change can move the best parameters.  `tuned(params,
clouds)` returns the cached entry or runs the search on the given pair and
stores it.
"""
from __future__ import annotations

import json
import os
import tempfile


def cache_path() -> str:
    return os.environ.get("PHGPU_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "phaser_b200", "tuning.json"))


def shape_key(params, device_name: str, build: str = "") -> str:
    return (f"{device_name}|{build}|B{params.spherical_bandwidth}+{params.spherical_zero_padding}|"
            f"N{params.spatial_n_voxels}|P{params.precision}")


def _read(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def load(params, device_name: str, path: str | None = None, build: str = ""):
    return _read(path or cache_path()).get(shape_key(params, device_name, build))


def save(params, device_name: str, tuning: dict, ms_per_pair: float, path: str | None = None, build: str = ""):
    path = path or cache_path()
    d = _read(path)
    d[shape_key(params, device_name, build)] = {"tuning": tuning, "ms_per_pair": ms_per_pair}
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path) or ".", suffix=".json")
    with os.fdopen(fd, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tuned(params, target, source, reps: int = 3, force: bool = False, path: str | None = None) -> dict:
    """The cached entry of params' shape on this device, or a new search on the
    pair (target, source as accepted by Context.register_pair), stored."""
    import torch
    from . import native
    dev = torch.cuda.get_device_name(params.device)
    build = native.build_id()
    if not force:
        hit = load(params, dev, path, build)
        if hit is not None:
            return dict(hit, cached=True)
    ctx = native.Context(params)
    try:
        t, ms = ctx.autotune(target, source, reps=reps)
    finally:
        ctx.close()
    save(params, dev, t, ms, path, build)
    return {"tuning": t, "ms_per_pair": ms, "cached": False}
