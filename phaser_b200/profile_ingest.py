"""Ingest timing: one scan of a workload written as a binary PLY, read back
into pinned host buffers (phgpu_ply_read) and downsampled on the GPU
(phgpu_voxel_grid_filter, leaf 0.25 as VoxelGridCmd).  The small program
the committed voxel-grid ncu summaries under profiles/ were captured on:

    python -m phaser_b200.profile_ingest --workload 1 --calls 4
    ncu --metrics gpu__time_duration.sum --clock-control none --csv \\
        --log-file launches.csv python -m phaser_b200.profile_ingest --workload 1 --calls 4
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import native, scene


def write_ply(path, xyzi, reflectivity=None):
    cols = [("x", 0), ("y", 1), ("z", 2), ("intensity", 3)]
    head = ["ply", "format binary_little_endian 1.0", f"element vertex {len(xyzi)}"]
    head += [f"property float {n}" for n, _ in cols]
    data = [np.asarray(xyzi, np.float32)]
    if reflectivity is not None:
        head.append("property float reflectivity")
        data.append(np.asarray(reflectivity, np.float32)[:, None])
    head.append("end_header")
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode())
        f.write(np.concatenate(data, axis=1).astype("<f4").tobytes())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", type=int, default=1)
    ap.add_argument("--calls", type=int, default=4)
    ap.add_argument("--leaf", type=float, default=0.25)
    a = ap.parse_args()
    import torch
    cl = scene.workload_pair(a.workload, 0).target
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "scan.ply")
        write_ply(path, cl.xyzi, cl.reflectivity)
        t0 = time.perf_counter()
        ply = native.ply_read(path, pinned=True)
        t_ply = time.perf_counter() - t0
    vg = native.VoxelGrid(max(1 << 18, len(cl.xyzi)))
    dev = torch.from_numpy(cl.xyzi).cuda()
    out = None
    t0 = time.perf_counter()
    for _ in range(a.calls):
        out, _, _ = vg.filter(dev, (a.leaf,) * 3, out_device=True)
    t_dev = (time.perf_counter() - t0) / a.calls
    t0 = time.perf_counter()
    for _ in range(a.calls):
        vg.filter(ply["xyzi"], (a.leaf,) * 3, reflectivity=ply["reflectivity"])
    t_host = (time.perf_counter() - t0) / a.calls
    vg.close()
    print(json.dumps({"workload": a.workload, "points": len(cl.xyzi), "leaves": int(out.shape[0]),
                      "ply_read_pinned_ms": round(1e3 * t_ply, 3), "voxel_grid_device_ms": round(1e3 * t_dev, 3),
                      "voxel_grid_host_ms": round(1e3 * t_host, 3)}))


if __name__ == "__main__":
    main()
