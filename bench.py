#!/usr/bin/env python
"""Registration throughput and latency of the B200 hot path.

Metric: registrations/s & p50/p99 latency at B=100, N=200 (served vs plain GPU
vs CPU).  A step registers `--pairs-per-step` pairs of the B=100 / N=200
workload (seeded synthetic room scans, 128 beams x 1024 columns, ~130k points,
3 channels); every pair's working set (~1 GB of grids and spectra) is far
larger than the 126 MB L2, so no flush is needed between iterations.

  value      served pipeline, clouds already resident in HBM
  e2e        served pipeline through the public API from pinned host memory
             (host->device copies and the pose read-back inside the timed region)
  plain_gpu  one pair at a time through phgpu_register_pair
  mixed_arrivals  open-loop Poisson arrivals of a three-shape mix through one server
  config2    256 pairs over twelve (B, N) shapes through one server (reg/s, waves/s)
  --impl reference  the reference's CPU path (SOFT sources + restated glue,
             oracle/_ref) on the host cores

Multi-GPU: one process per GPU (torchrun), each rank registers its own pairs
(no collective on the data path), value = all pairs / max over ranks of the
device-timed window.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "registrations/s & p50/p99 latency at B=100,N=200: served vs plain GPU vs CPU"
UNIT = "registrations/s"
WORKLOAD = 1


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--pairs-per-step", type=int, default=512)
    ap.add_argument("--max-wave", type=int, default=16, help="pairs per wave of the server")
    ap.add_argument("--lanes", type=int, default=2, help="waves in flight at once")
    ap.add_argument("--pool", type=int, default=4, help="distinct synthetic pairs per rank")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", choices=["pair", "served", "ingest"], default=None,
                    help="run a small program for an ncu capture and exit: `pair` registers --pairs pairs of "
                         "--workload one at a time (plain), `served` runs --pairs pairs through the server in "
                         "waves, `ingest` reads one scan from a PLY and voxel-grid filters it --calls times")
    ap.add_argument("--workload", type=int, default=WORKLOAD)
    ap.add_argument("--pairs", type=int, default=2)
    ap.add_argument("--calls", type=int, default=4)
    ap.add_argument("--precision", type=int, default=0, help="--profile pair: PHGPU_PRECISION_* of the context")
    ap.add_argument("--no-config2", action="store_true", help="skip the 256-pair, 12-shape batched workload leg")
    ap.add_argument("--no-cpu-throughput", action="store_true",
                    help="reference arm: skip the nproc single-threaded processes leg")
    return ap.parse_args()


def pct(v, q):
    if not v:
        return None
    return float(np.percentile(np.asarray(v), q))


def workload_desc():
    from phaser_b200 import scene
    w = scene.WORKLOADS[WORKLOAD]
    return w, (f"B={w['bw']} (200x200 S2, 200^3 SO(3)), N={w['n_voxels']} voxels over "
               f"[{w['lo']},{w['hi']}]^3 m, {w['beams']}x{w['cols']} LiDAR (~130k points), "
               "channels range/intensity/reflectivity")


def pool_seeds(rank, n):
    """Pair seeds of one rank: disjoint across ranks (the pairs are sharded,
    each rank registers its own)."""
    return [rank * 1000 + j for j in range(n)]


def make_pool(rank, n):
    from phaser_b200 import scene
    return [scene.workload_pair(WORKLOAD, k) for k in pool_seeds(rank, n)]


def max_over_ranks(x, dist=None, device="cuda"):
    """Largest value of x over the ranks (the job's time is its slowest
    rank's); x itself without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, steps, pairs_per_step, max_ms):
    """Whole-job registrations/s: every rank registers steps x pairs_per_step
    pairs within the slowest rank's window."""
    return world * steps * pairs_per_step / (max_ms * 1e-3)


# ------------------------------------------------------------------ clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_id):
        self.dev_id = dev_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.dev_id), "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def physical_gpu_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local < len(ids):
            return ids[local]
    return local


# ------------------------------------------------------------------ roofline

def stage_bytes(stage, bw, N, C, P):
    """Algorithmic HBM bytes of one call of a stage (per cloud where a stage
    runs per cloud: sampling, voxelisation, the forward spatial transform), after the per-unit figures of the survey's
    measurement section: FP32 data, complex64 spectra, the minimum each stage
    moves with its inputs and outputs in HBM."""
    nv = N ** 3
    H = N * N * (N // 2 + 1)
    n = 2 * bw
    return {
        "s2_sample": P * 20 + 4 * n * n * 4,                 # points in, 4 sample channels out
        "sht": 2 * (C * n * n * 4 + C * bw * bw * 8),        # both sides: C grids in, C coefficient sets out
        "fuse_s2": 2 * C * bw * bw * 8 + 2 * bw * bw * 8,    # both sides' coefficients in, fused out
        "so3_synth": n * n * bw * 8,                         # half spectrum S written (m2 >= 0)
        "so3_fft": 3 * n * n * bw * 8,                       # S read + write (alpha), read (gamma)
        "voxelize": P * 20,                                  # points in (voxel updates are scattered)
        "spatial_fwd": C * (nv * 4 + H * 8),                 # R2C of C grids: read + write
        "fuse_z": 2 * C * H * 8 + H * 8,                     # both sides' spectra in, product out
        "spatial_inv": H * 8,                                # product in (argmax fused, no volume)
    }.get(stage)


def pair_bytes(bw, N, C, P):
    """Algorithmic bytes of one served registration (the survey's per-pair
    total: rotation + translation subtotals)."""
    n = 2 * bw
    nv = N ** 3
    H = N * N * (N // 2 + 1)
    rot = (2 * P * 20 + 2 * C * n * n * 4 + 2 * C * bw * bw * 8 + (4 * bw ** 3 // 3) * 8 + n ** 3 * 8
           + 2 * n ** 3 * 8 + n ** 3 * 8)
    trans = P * 20 + 2 * C * nv * 4 + 2 * C * (nv * 4 + H * 8) + (2 * C * H * 8 + H * 8) + (H * 8 + nv * 4) + nv * 4
    return rot + trans


# Kernels of each profiled stage (one launch of each per stage call).
STAGE_KERNELS = {
    "s2_sample": ("k_project", "k_bin_scan", "k_bin_scatter", "k_nn_rows"),
    "sht": ("k_sht_phi", "k_sht_leg", "k_sht_leg_tc"),
    "fuse_s2": ("k_fuse_s2",),
    "so3_synth": ("k_so3_synth", "k_so3_synth_tc"),
    "so3_fft": ("k_so3_fft_a", "k_so3_c2r_tail"),
    "voxelize": ("k_voxelize",),
    "spatial_fwd": ("k_slab_fwd",),
    "fuse_z": ("k_fuse_z",),
    "spatial_inv": ("k_slab_inv",),
}

TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "traffic_register_pair_B100_N200.md")


def ncu_traffic(path=TRAFFIC_PROFILE):
    """DRAM read + write bytes per stage call at B = 100 / N = 200, summed over
    the stage's kernels, from the committed table of one-kernel ncu captures
    (`dram__bytes_read.sum + dram__bytes_write.sum` per launch of the current
    kernels; the file gives the capture command).  A stage is left out when
    one of the kernels it launched has no row (variant kernels of a stage,
    e.g. the CUDA-core and tensor-core synthesis, count whichever has one)."""
    per_kernel = {}
    try:
        lines = open(path).read().splitlines()
    except OSError:
        return {}
    for ln in lines:
        if not ln.startswith("| `"):
            continue
        cells = [c.strip() for c in ln.strip().strip("|").split("|")]
        if len(cells) != 5:  # the first table: kernel, launches, us, read MB, write MB
            continue
        name = re.sub(r"<.*", "", cells[0].strip("`").replace("void ", "")).strip()
        try:
            per_kernel[name] = (float(cells[3]) + float(cells[4])) * 1e6
        except ValueError:
            continue
    out = {}
    for stage, kernels in STAGE_KERNELS.items():
        have = [per_kernel[k] for k in kernels if k in per_kernel]
        if have:
            out[stage] = int(sum(have))
    return out


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def roofline(nat, pool, params, tuning, served_value):
    """Per-stage device time from CUDA events recorded on each stage's stream
    while both halves of a registration run on one stream (so no two stages'
    events overlap), on a context of the served form (tensor-core synthesis,
    its tuning) registering the bench pairs one at a time.  Each stage is rated
    by its algorithmic bytes (frac) and, where an ncu capture measured it, by
    its DRAM traffic (frac_actual); the top-level entry is the stage with the
    largest device time.  The whole pipeline is rated with the per-pair
    algorithmic bytes at the served rate."""
    ctx = nat.Context(params)
    ctx.set_tuning(tuning)
    ctx.profile(True, serial=True)
    import torch
    dev = [((torch.from_numpy(p.target.xyzi).cuda(), torch.from_numpy(p.target.reflectivity).cuda()),
            (torch.from_numpy(p.source.xyzi).cuda(), torch.from_numpy(p.source.reflectivity).cuda()))
           for p in pool]
    for i in range(2):
        ctx.register_pair(*dev[i % len(dev)])
    ctx.profile_read()
    nrep = 8
    for i in range(nrep):
        ctx.register_pair(*dev[i % len(dev)])
    st = ctx.profile_read()
    ctx.close()
    bw, N, C = params.spherical_bandwidth, params.spatial_n_voxels, 3
    P = int(np.mean([p.target.xyzi.shape[0] for p in pool]))
    peak, src = measured_peak()
    tot = {k: v for k, v in st.items() if v[1] > 0 and k != "upload"}
    workload_is_bench = (bw, N) == (100, 200)
    traffic = ncu_traffic()
    stages = {}
    for k, (ms, calls) in tot.items():
        nb = stage_bytes(k, bw, N, C, P)
        per = ms / calls
        e = {"ms_per_call": round(per, 4), "calls_per_pair": round(calls / nrep, 2),
             "ms_per_pair": round(ms / nrep, 4)}
        if nb:
            gbs = nb / (per * 1e-3) / 1e9
            e.update({"algorithmic_bytes": nb, "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)})
        tr = traffic.get(k) if workload_is_bench else None
        if tr:
            e.update({"traffic": tr, "traffic_gbs": round(tr / (per * 1e-3) / 1e9, 1),
                      "frac_actual": round(tr / (per * 1e-3) / 1e9 / peak, 4)})
        stages[k] = e
    top = max(stages, key=lambda k: stages[k]["ms_per_pair"])
    e = stages[top]
    roof = {"kernel": top, "bound": "hbm", "achieved": e.get("achieved_gbs"), "peak": peak, "unit": "GB/s",
            "frac": e.get("frac"), "traffic": e.get("traffic"), "frac_actual": e.get("frac_actual"),
            "peak_source": src, "algorithmic_bytes_per_launch": e.get("algorithmic_bytes"),
            "avg_launch_ms": e["ms_per_call"], "timing": "CUDA events, stages serialised on one stream",
            "stages": stages}
    pb = pair_bytes(bw, N, C, P)
    roof["pipeline"] = {"algorithmic_bytes_per_pair": pb, "achieved_gbs": round(served_value * pb / 1e9, 1),
                        "frac": round(served_value * pb / 1e9 / peak, 4),
                        "device_ms_per_pair_serialised": round(sum(v["ms_per_pair"] for v in stages.values()), 4),
                        "basis": "served registrations/s x per-pair algorithmic bytes"}
    return roof


def ingest(nat, pool, cpu_ok, reps=20):
    """Ingest (PLY read + VoxelGridCmd) of one bench scan: the scan written as
    a binary PLY and read into pinned host buffers (phgpu_ply_read), then
    downsampled with leaf 0.25 (phgpu_voxel_grid_filter).  The filter is
    synchronous (it returns the leaf count), so its time is the wall time per
    call: host buffers in and out (copies included) and device-resident
    buffers.  Algorithmic bytes: 16 per point in (x, y, z, intensity) and 16
    per leaf out.  CPU: the oracle's single-thread restatement of
    pcl::VoxelGrid on the same scan."""
    import tempfile
    import torch
    from phaser_b200.scene import write_ply
    cl = pool[0].target
    n = int(cl.xyzi.shape[0])
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "scan.ply")
        write_ply(path, cl.xyzi, cl.reflectivity)
        nat.ply_read(path, pinned=True)
        t0 = time.perf_counter()
        for _ in range(3):
            ply = nat.ply_read(path, pinned=True)
        t_ply = (time.perf_counter() - t0) / 3
    vg = nat.VoxelGrid(max(1 << 18, n))
    dev = torch.from_numpy(cl.xyzi).cuda()
    for _ in range(3):
        out, _, _ = vg.filter(dev, (0.25,) * 3, out_device=True)
        vg.filter(ply["xyzi"], (0.25,) * 3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        out, _, _ = vg.filter(dev, (0.25,) * 3, out_device=True)
    t_dev = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        vg.filter(ply["xyzi"], (0.25,) * 3)
    t_host = (time.perf_counter() - t0) / reps
    vg.close()
    leaves = int(out.shape[0])
    nb = 16 * n + 16 * leaves
    peak, src = measured_peak()
    res = {"workload": f"voxel grid (leaf 0.25 m) of one {n}-point bench scan, read from a binary PLY",
           "points": n, "leaves": leaves, "ply_read_pinned_ms": round(1e3 * t_ply, 3),
           "voxel_grid_ms": round(1e3 * t_host, 4), "voxel_grid_device_ms": round(1e3 * t_dev, 4),
           "points_per_s": round(n / t_host, 1),
           "roofline": {"bound": "hbm", "achieved": round(nb / t_dev / 1e9, 2), "peak": peak, "unit": "GB/s",
                        "frac": round(nb / t_dev / 1e9 / peak, 5), "algorithmic_bytes": nb,
                        "basis": "device-resident call wall time (launch-latency bound at this size)"}}
    if cpu_ok:
        from oracle import oracle as O
        t0 = time.perf_counter()
        for _ in range(3):
            O.voxel_grid(cl.xyzi, 0.25)
        res["cpu_baseline"] = {"ms": round(1e3 * (time.perf_counter() - t0) / 3, 3), "cores": 1, "kind": "port",
                               "sample": "the same scan, oracle restatement of pcl::VoxelGrid"}
    return res


def config3(nat, local, rates=(50, 200, 500, 1000, 2000), seconds=1.0, cap=600):
    """Open-loop Poisson arrivals of a shape mix through one server (50 %
    B=64/N=128, 35 % B=100/N=200, 15 % B=128/N=256; HBM budget 150 GB; clouds
    resident in HBM): per arrival rate, the requests' p50 / p99 latency from
    submission to completion and the completed rate."""
    import torch
    from phaser_b200 import scene
    rng = np.random.default_rng(3)
    shapes = []
    for i, (weight, sh) in enumerate(scene.CONFIG3_MIX):
        params = nat.default_params(spherical_bandwidth=sh["bw"], spatial_n_voxels=sh["n_voxels"],
                                    spatial_discretize_lower=sh["lo"], spatial_discretize_upper=sh["hi"],
                                    max_points=1 << 18, device=local, precision=nat.PHGPU_PRECISION_TF32X3)
        pairs = [scene.make_pair(3, 10 * i + k, sh["beams"]) for k in range(2 if i == 0 else 1)]
        dev = [((torch.from_numpy(p.target.xyzi).cuda(), torch.from_numpy(p.target.reflectivity).cuda()),
                (torch.from_numpy(p.source.xyzi).cuda(), torch.from_numpy(p.source.reflectivity).cuda()))
               for p in pairs]
        shapes.append((weight, params, dev))
    probs = [w for w, _, _ in shapes]
    lanes, max_wave = 2, 16
    srv = nat.Server(max_wave=max_wave, lanes=lanes, hbm_budget_bytes=150 << 30, device=local)
    warm = [srv.submit(params, *dev[j % len(dev)]) for _, params, dev in shapes for j in range(2 * max_wave)]
    srv.drain()
    for t in warm:
        srv.poll(t)
    out = []
    for rate in rates:
        n = int(min(max(rate * seconds, 50), cap))
        gaps = rng.exponential(1.0 / rate, size=n)
        kinds = rng.choice(len(shapes), size=n, p=probs)
        tick = []
        t0 = due = time.perf_counter()
        for g, kd in zip(gaps, kinds):
            due += g
            while time.perf_counter() < due:
                time.sleep(0.0001)
            _, params, dev = shapes[kd]
            tick.append((int(kd), srv.submit(params, *dev[len(tick) % len(dev)])))
        srv.drain()
        span = time.perf_counter() - t0
        lat = [(kd, srv.poll(t)[1]) for kd, t in tick]
        by = {f"B{shapes[i][1].spherical_bandwidth}/N{shapes[i][1].spatial_n_voxels}":
              round(pct([v for k, v in lat if k == i], 99), 3) for i in range(len(shapes))
              if any(k == i for k, _ in lat)}
        out.append({"rate_per_s": rate, "requests": n, "completed_per_s": round(n / span, 1),
                    "p50_ms": round(pct([v for _, v in lat], 50), 3),
                    "p99_ms": round(pct([v for _, v in lat], 99), 3), "p99_ms_by_shape": by})
    srv.close()
    return {"mix": "50% B64/N128, 35% B100/N200, 15% B128/N256 (64/128/128-beam scans)",
            "hbm_budget_gb": 150, "server_lanes": lanes, "max_wave": max_wave, "inputs": "clouds resident in HBM",
            "rates": out}


def config2(nat, local, n=256, max_wave=8):
    """The batched workload: n independent pairs over twelve (B, N) shapes
    (beams {32, 64, 128} x 1024, B {32, 64, 100, 128}, N {64, 128, 200},
    seeded per pair) through one server in size-grouped waves, tf32x3, clouds
    resident in HBM, default launch parameters.  The batch runs twice (the
    first pass creates the executors and captures their graphs); the second
    is reported: registrations/s and waves/s over the wall time from the first
    submit to the drain, and the per-request latency."""
    import torch
    from phaser_b200 import scene
    specs = scene.config2_specs(n)
    pairs = scene.config2_pairs(specs)

    def dev(a):
        return None if a is None else torch.from_numpy(a).cuda()

    clouds = [((dev(p.target.xyzi), dev(p.target.reflectivity)), (dev(p.source.xyzi), dev(p.source.reflectivity)))
              for p in pairs]
    prms = [nat.default_params(spherical_bandwidth=sp["bw"], spatial_n_voxels=sp["n_voxels"],
                               spatial_discretize_lower=sp["lo"], spatial_discretize_upper=sp["hi"],
                               precision=nat.PHGPU_PRECISION_TF32X3, device=local) for sp in specs]
    srv = nat.Server(max_wave=max_wave, lanes=2, device=local)

    def batch():
        w0 = srv.stats()["waves"]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tickets = [srv.submit(prms[i], *clouds[i]) for i in range(n)]
        srv.drain()
        wall = time.perf_counter() - t0
        lat = [srv.poll(t)[1] for t in tickets]
        return wall, lat, srv.stats()["waves"] - w0

    batch()
    wall, lat, waves = batch()
    st = srv.stats()
    srv.close()
    return {"workload": f"{n} pairs, 12 (B, N) shapes, beams 32/64/128 x 1024", "max_wave": max_wave,
            "server_lanes": 2, "precision": "tf32x3", "registrations_per_s": round(n / wall, 1),
            "waves_per_s": round(waves / wall, 1), "waves": waves, "wall_s": round(wall, 4),
            "p50_ms": round(pct(lat, 50), 3), "p99_ms": round(pct(lat, 99), 3),
            "executors": st["executors"], "graph_captures": st["graph_captures"]}


def run_script_config(nat, pool, local, reps=10):
    """One pair at a time with the configuration of the reference's run script
    (phaser_share/run_phaser_core_driver: B = 150 with spherical zero padding
    10, N = 201 voxels over [-50, 50]^3 m) on the bench scans, clouds resident
    in HBM: registrations/s and the latency of one pair."""
    import torch
    params = nat.default_params(spherical_bandwidth=150, spherical_zero_padding=10, spatial_n_voxels=201,
                                spatial_discretize_lower=-50, spatial_discretize_upper=50, max_points=1 << 18,
                                device=local)
    ctx = nat.Context(params)
    dev = [((torch.from_numpy(p.target.xyzi).cuda(), torch.from_numpy(p.target.reflectivity).cuda()),
            (torch.from_numpy(p.source.xyzi).cuda(), torch.from_numpy(p.source.reflectivity).cuda()))
           for p in pool]
    for i in range(3):
        ctx.register_pair(*dev[i % len(dev)])
    lat = []
    for i in range(reps):
        t0 = time.perf_counter()
        ctx.register_pair(*dev[i % len(dev)])
        lat.append(1e3 * (time.perf_counter() - t0))
    ctx.close()
    return {"config": "B=150 + spherical zero padding 10 (SO(3) on 320^3), N=201 over [-50,50]^3 m",
            "plain_gpu_per_s": round(1e3 / float(np.mean(lat)), 2), "p50_ms": round(pct(lat, 50), 3),
            "p99_ms": round(pct(lat, 99), 3)}


# ------------------------------------------------------------------ CPU

# FFTW threads the reference registration plans with
# (phaser_core/src/backend/registration/sph-opt-registration.cc:29-30).
REF_FFT_THREADS = 12

CPU_PATH = ("SOFT 2.0 sources of the reference (unmodified) + project FP64 FFTW-API shim (no FFTW3 library in "
            "the image) + restated phaser_core glue, kd-tree NN")


def config_desc(desc, world):
    """The `config` both arms print (identical, so the two arms' lines pair up)."""
    return {"workload": desc, "l2": "per-pair working set ~1 GB > 126 MB L2 (no flush needed)",
            "parallelism": f"replicas x{world}, pairs sharded per rank"}


def cpu_reference(pair, w, threads=REF_FFT_THREADS):
    """One registration on the host cores through the reference path (the
    oracle port when oracle/_ref is absent): seconds, kind, (bin, voxel)."""
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    t0 = time.perf_counter()
    if kind == "reference":
        rb, vx, _ = O.ref_register_pair(pair.target.xyzi, pair.target.reflectivity, pair.source.xyzi,
                                        pair.source.reflectivity, w["bw"], w["n_voxels"], w["lo"], w["hi"],
                                        threads=threads)
    else:
        pose = O.register_pair(pair.target.xyzi, pair.target.reflectivity, pair.source.xyzi,
                               pair.source.reflectivity, w["bw"], w["n_voxels"], w["lo"], w["hi"])
        rb, vx = pose.rot_bin, pose.voxel
    return time.perf_counter() - t0, kind, (int(rb), int(vx))


def _throughput_worker(k):
    """One single-threaded reference registration of pair k (spawned process):
    wall-clock start and end of the registration alone."""
    sys.path.insert(0, ROOT)
    from phaser_b200 import scene
    w = scene.WORKLOADS[WORKLOAD]
    pair = scene.workload_pair(WORKLOAD, k)
    t0 = time.time()
    cpu_reference(pair, w, threads=1)
    return t0, time.time()


def cpu_throughput(n_proc):
    """nproc independent single-threaded registrations of distinct pairs at
    once: the aggregate rate over the span from the first start to the last
    end."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(n_proc) as pool:
        spans = pool.map(_throughput_worker, list(range(100, 100 + n_proc)))
    wall = max(b for _, b in spans) - min(a for a, _ in spans)
    return {"value": round(n_proc / wall, 4), "unit": UNIT, "processes": n_proc, "threads_per_process": 1,
            "wall_s": round(wall, 2), "sample": f"{n_proc} distinct pairs of the workload, one per process"}


def run_reference(a, world, rank):
    if rank != 0:
        return 0
    w, desc = workload_desc()
    pool = make_pool(0, 1)
    lat = []
    kind = "reference"
    bins = None
    for i in range(a.warmup + a.steps):
        dt, kind, bins = cpu_reference(pool[0], w)
        if i >= a.warmup:
            lat.append(dt)
    T = sum(lat)
    v = a.steps / T
    cores = os.cpu_count()
    thr = cpu_throughput(cores) if not a.no_cpu_throughput else None
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(1e3 * T / a.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded room scans)", "config": config_desc(desc, world), "pairs_per_step": 1,
        "path": CPU_PATH,
        "latency_ms": {"p50": round(1e3 * pct(lat, 50), 2), "p99": round(1e3 * pct(lat, 99), 2),
                       "threads": REF_FFT_THREADS},
        "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": REF_FFT_THREADS, "kind": kind,
                         "sample": f"1 pair of the workload per step (seed {pool_seeds(0, 1)[0]}), FFTs on "
                                   f"{REF_FFT_THREADS} threads as the reference plans them, {cores} host threads"},
        "cpu_throughput": thr,
        "parity": {"pair_seed": pool_seeds(0, 1)[0], "rot_bin": bins[0], "voxel": bins[1]},
        "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ profiling programs

def run_profile(a):
    """The small programs the committed ncu summaries are captured on (one GPU,
    a few launches of each kernel): prints one JSON line."""
    import torch
    from phaser_b200 import native as nat, scene
    nat.load()
    w = scene.WORKLOADS[a.workload]
    p = scene.workload_pair(a.workload, 0)
    cap = max(1 << 18, p.target.xyzi.shape[0], p.source.xyzi.shape[0])
    params = nat.default_params(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"],
                                spatial_discretize_lower=w["lo"], spatial_discretize_upper=w["hi"], max_points=cap,
                                precision=a.precision)
    clouds = ((p.target.xyzi, p.target.reflectivity), (p.source.xyzi, p.source.reflectivity))
    out = {"profile": a.profile, "workload": a.workload}
    if a.profile == "pair":
        ctx = nat.Context(params)
        pose = None
        for _ in range(a.pairs):
            pose = ctx.register_pair(*clouds)
        out.update({"rot_bin": pose.rot_bin, "voxel": pose.voxel, "pairs": a.pairs})
        ctx.close()
    elif a.profile == "served":
        params.precision = nat.PHGPU_PRECISION_TF32X3
        dev = tuple((torch.from_numpy(x).cuda(), torch.from_numpy(r).cuda()) for x, r in clouds)
        srv = nat.Server(max_wave=a.max_wave, lanes=1, max_points=cap)
        tickets = [srv.submit(params, *dev) for _ in range(a.pairs)]
        srv.drain()
        poses = [srv.poll(t)[0] for t in tickets]
        out.update({"rot_bin": poses[0].rot_bin, "voxel": poses[0].voxel, "pairs": a.pairs, "server": srv.stats()})
        srv.close()
    else:
        import tempfile
        cl = p.target
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "scan.ply")
            scene.write_ply(path, cl.xyzi, cl.reflectivity)
            ply = nat.ply_read(path, pinned=True)
        vg = nat.VoxelGrid(max(1 << 18, len(cl.xyzi)))
        dv = torch.from_numpy(cl.xyzi).cuda()
        leaves = 0
        for _ in range(a.calls):
            o, _, _ = vg.filter(dv, (0.25,) * 3, out_device=True)
            vg.filter(ply["xyzi"], (0.25,) * 3, reflectivity=ply["reflectivity"])
            leaves = int(o.shape[0])
        vg.close()
        out.update({"points": len(cl.xyzi), "leaves": leaves, "calls": 2 * a.calls})
    torch.cuda.synchronize()
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------ GPU

def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference(a, world, rank)
    if a.profile:
        return run_profile(a)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from phaser_b200 import native as nat
    nat.load()
    w, desc = workload_desc()
    params = nat.default_params(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"],
                                spatial_discretize_lower=w["lo"], spatial_discretize_upper=w["hi"],
                                max_points=1 << 18, device=local)
    pool = make_pool(rank, a.pool)
    dev = [((torch.from_numpy(p.target.xyzi).cuda(), torch.from_numpy(p.target.reflectivity).cuda()),
            (torch.from_numpy(p.source.xyzi).cuda(), torch.from_numpy(p.source.reflectivity).cuda()))
           for p in pool]
    pinned = [((torch.from_numpy(p.target.xyzi).pin_memory(), torch.from_numpy(p.target.reflectivity).pin_memory()),
               (torch.from_numpy(p.source.xyzi).pin_memory(), torch.from_numpy(p.source.reflectivity).pin_memory()))
              for p in pool]
    pinned_np = [((t[0].numpy(), t[1].numpy()), (s[0].numpy(), s[1].numpy())) for t, s in pinned]
    h2d_per_pair = int(np.mean([p.target.xyzi.nbytes + p.target.reflectivity.nbytes + p.source.xyzi.nbytes +
                                p.source.reflectivity.nbytes for p in pool]))
    K, W, S = a.steps, a.warmup, a.pairs_per_step

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # ---------------- autotuned launch parameters of both forms (cached per
    # shape and device; the search times candidates on one pool pair)
    from phaser_b200 import tuning as tuning_cache
    sparams = nat.default_params(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"],
                                 spatial_discretize_lower=w["lo"], spatial_discretize_upper=w["hi"],
                                 max_points=1 << 18, device=local, precision=nat.PHGPU_PRECISION_TF32X3)
    tuned_plain = tuning_cache.tuned(params, *dev[0])
    tuned_served = tuning_cache.tuned(sparams, *dev[0])

    # ---------------- plain GPU pipeline (one pair at a time)
    ctx = nat.Context(params)
    ctx.set_tuning(tuned_plain["tuning"])
    for i in range(W * S):
        ctx.register_pair(*dev[i % len(dev)])
    barrier()
    plain_lat = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(K * S):
        t = time.perf_counter()
        ctx.register_pair(*dev[i % len(dev)])
        plain_lat.append(1e3 * (time.perf_counter() - t))
    e1.record()
    e1.synchronize()
    plain_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    plain_value = job_rate(world, K, S, plain_ms)
    plain_pose0 = ctx.register_pair(*dev[0])
    ctx.close()

    # ---------------- served pipeline, device-resident inputs (value)
    # host inputs are borrowed (pinned, copied to the device inside each request)
    srv = nat.Server(max_wave=a.max_wave, lanes=a.lanes, hbm_budget_bytes=150 << 30, device=local,
                     flags=nat.PHGPU_SERVER_BORROW_HOST)
    # the served form: tensor-core (split-TF32) Wigner-d synthesis, batched per wave
    srv.set_tuning(sparams, tuned_served["tuning"])

    def served_round(inputs, n):
        tickets = [srv.submit(sparams, *inputs[i % len(inputs)]) for i in range(n)]
        srv.drain()
        lats = []
        for t in tickets:
            r = srv.poll(t)
            lats.append(r[1])
        return lats

    served_round(dev, W * S)
    barrier()
    sampler = ClockSampler(physical_gpu_index(local))
    sampler.start()
    time.sleep(0.3)
    l0 = nat.launch_count()
    e0.record()
    served_lat = []
    for _ in range(K):
        served_lat += served_round(dev, S)
    e1.record()
    e1.synchronize()
    launches = nat.launch_count() - l0
    time.sleep(0.2)
    clocks = sampler.stop()
    served_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    value = job_rate(world, K, S, served_ms)

    # ---------------- e2e: served, pinned host inputs through the public API
    served_round(pinned_np, S)
    barrier()
    e0.record()
    for _ in range(K):
        served_round(pinned_np, S)
    e1.record()
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    e2e_value = job_rate(world, K, S, e2e_ms)

    # ---------------- open-loop Poisson arrivals at 80% of the served rate
    rate = 0.8 * value / world
    n_req = int(min(max(2.0 * rate, 50), 400))
    rng = np.random.default_rng(rank)
    gaps = rng.exponential(1.0 / rate, size=n_req)
    tick = []
    t_start = time.perf_counter()
    due = t_start
    for i in range(n_req):
        due += gaps[i]
        while time.perf_counter() < due:
            time.sleep(0.0001)
        tick.append(srv.submit(sparams, *dev[i % len(dev)]))
    srv.drain()
    open_lat = [srv.poll(t)[1] for t in tick]
    t0 = srv.submit(sparams, *dev[0])
    srv.drain()
    served_pose0 = srv.poll(t0)[0]
    server_stats = srv.stats()
    srv.close()
    barrier()

    # ---------------- roofline of the dominant stage (rank 0 context, profiled)
    roof = roofline(nat, pool, sparams, tuned_served["tuning"], value / world)

    # ---------------- mixed shapes under Poisson arrivals (rank 0)
    mix = None
    if rank == 0:
        try:
            mix = config3(nat, local)
        except Exception as exc:  # the headline line is printed regardless
            mix = {"error": f"{type(exc).__name__}: {exc}"}

    # ---------------- the batched 256-pair, 12-shape workload (rank 0)
    c2 = None
    if rank == 0 and world == 1 and not a.no_config2:
        try:
            c2 = config2(nat, local)
        except Exception as exc:  # the headline line is printed regardless
            c2 = {"error": f"{type(exc).__name__}: {exc}"}

    # ---------------- the reference run script's configuration (rank 0)
    rsc = None
    if rank == 0:
        try:
            rsc = run_script_config(nat, pool, local)
        except Exception as exc:  # the headline line is printed regardless
            rsc = {"error": f"{type(exc).__name__}: {exc}"}

    # ---------------- ingest: PLY read + voxel-grid downsample (rank 0)
    ing = None
    if rank == 0:
        try:
            ing = ingest(nat, pool, world == 1 and not a.no_cpu_baseline)
        except Exception as exc:  # the headline line is printed regardless
            ing = {"error": f"{type(exc).__name__}: {exc}"}

    # ---------------- CPU baseline and reference parity (rank 0, N = 1): the
    # reference path on the first pool pair; the GPU's plain and served poses
    # of that pair must equal its bin and voxel
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        dt, kind, bins = cpu_reference(pool[0], w)
        cpu = {"value": round(1.0 / dt, 4), "unit": UNIT, "cores": REF_FFT_THREADS, "kind": kind,
               "sample": f"1 pair of the workload (seed {pool_seeds(rank, 1)[0]}), FFTs on {REF_FFT_THREADS} threads "
                         f"as the reference plans them; {CPU_PATH}"}
        gp = [(q.rot_bin, q.voxel) for q in (plain_pose0, served_pose0)]
        parity = {"pair_seed": pool_seeds(rank, 1)[0], "reference": {"rot_bin": bins[0], "voxel": bins[1]},
                  "plain": {"rot_bin": gp[0][0], "voxel": gp[0][1]},
                  "served": {"rot_bin": gp[1][0], "voxel": gp[1][1]},
                  "equal": all(g == bins for g in gp)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": round(served_ms / K, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded room scans, 128x1024 LiDAR)",
            "config": config_desc(desc, world), "pairs_per_step": S, "pairs_per_rank": K * S,
            "server": {"max_wave": a.max_wave, "lanes": a.lanes}, "distinct_pairs": a.pool,
            "served": {"value": round(value, 2), "precision": "tf32x3 tensor-core Wigner-d synthesis",
                       "server_stats": server_stats, "p50_ms": round(pct(served_lat, 50), 3),
                       "p99_ms": round(pct(served_lat, 99), 3), "latency": "closed-loop batches of pairs_per_step",
                       "open_loop": {"rate_per_s": round(rate, 1), "requests": n_req,
                                     "p50_ms": round(pct(open_lat, 50), 3), "p99_ms": round(pct(open_lat, 99), 3)}},
            "plain_gpu": {"value": round(plain_value, 2), "precision": "fp32", "p50_ms": round(pct(plain_lat, 50), 3),
                          "p99_ms": round(pct(plain_lat, 99), 3)},
            "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": h2d_per_pair * S,
                    "d2h_bytes_per_step": 16 * S},
            "roofline": roof,
            "cpu_baseline": cpu,
            "reference_parity": parity,
            "clocks": clocks,
            "gpu_launches": int(launches),
            "tuning": {"plain": tuned_plain, "served": tuned_served},
            "ingest": ing,
            "mixed_arrivals": mix,
            "config2": c2,
            "run_script_config": rsc,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if parity is not None and not parity["equal"]:
        print("GPU poses differ from the reference path on the checked pair", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
