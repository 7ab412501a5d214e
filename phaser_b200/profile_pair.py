"""Registers a few pairs of a workload through the C ABI and prints the per-stage
device time -- the small, self-contained program the committed ncu summaries
under profiles/ were captured on:

    python -m phaser_b200.profile_pair --workload 1 --pairs 2
    ncu --metrics gpu__time_duration.sum --clock-control none --csv \
        --log-file launches.csv python -m phaser_b200.profile_pair --workload 1 --pairs 2
"""
from __future__ import annotations

import argparse
import json

from . import native, scene


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", type=int, default=1)
    ap.add_argument("--pairs", type=int, default=2)
    ap.add_argument("--stages", action="store_true", help="print per-stage CUDA-event times")
    a = ap.parse_args()
    w = scene.WORKLOADS[a.workload]
    p = scene.workload_pair(a.workload, 0)
    ctx = native.Context(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"],
                         spatial_discretize_lower=w["lo"], spatial_discretize_upper=w["hi"],
                         max_points=max(1 << 18, p.target.xyzi.shape[0], p.source.xyzi.shape[0]))
    if a.stages:
        ctx.profile(True)
    pose = None
    for _ in range(a.pairs):
        pose = ctx.register_pair((p.target.xyzi, p.target.reflectivity), (p.source.xyzi, p.source.reflectivity))
    out = {"workload": a.workload, "rot_bin": pose.rot_bin, "voxel": pose.voxel}
    if a.stages:
        out["stage_ms_total"] = ctx.profile_read()
    print(json.dumps(out))
    ctx.close()


if __name__ == "__main__":
    main()
