"""Seeded synthetic scenes and spinning-LiDAR scans for the registration
workloads (the reference's PLY test clouds are not available, so seeded
synthetic clouds with the same shapes stand in for them).

Scene: a 20 x 12 x 4 m box room (floor, ceiling, four walls) with 40
axis-aligned boxes (sides U[0.3, 2] m, standing on the floor) and 20
floor-to-ceiling cylinders (radius U[0.1, 0.5] m), placed uniformly but
outside the square |x|, |y| <= 2.6 m that holds the sensor positions.

Scan: `beams` elevations uniform in [-22.5, 22.5] deg x `cols` azimuth
columns, ray-cast against the scene, Gaussian range noise sigma = 0.01 m,
intensity clip(0.5 + 0.3 cos(incidence) + N(0, 0.05), 0, 1), optional
reflectivity = intensity * range^2 normalised to [0, 1].  Points are returned
in the sensor frame as float32 (x, y, z, intensity).

A pair is (target, source): the source is scanned at the origin with the
identity orientation; the target is scanned from a pose with rotation uniform
on SO(3) and translation U[-2, 2]^3 m, and expressed in its own frame.  Seeds:
workload c, pair k -> seed 1000 c + k, with scene and pose drawn from separate
streams.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

ROOM_LO = np.array([-10.0, -6.0, -2.0])
ROOM_HI = np.array([10.0, 6.0, 2.0])


@dataclass
class Scene:
    box_lo: np.ndarray  # [nb, 3]
    box_hi: np.ndarray
    cyl_xy: np.ndarray  # [nc, 2]
    cyl_r: np.ndarray   # [nc]


@dataclass
class Cloud:
    xyzi: np.ndarray          # float32 [P, 4]
    reflectivity: np.ndarray | None  # float32 [P] or None


def make_scene(rng: np.random.Generator, n_boxes=40, n_cyl=20) -> Scene:
    def place(n, margin):
        out = []
        while len(out) < n:
            x = rng.uniform(ROOM_LO[0] + margin, ROOM_HI[0] - margin)
            y = rng.uniform(ROOM_LO[1] + margin, ROOM_HI[1] - margin)
            if abs(x) <= 2.6 + margin and abs(y) <= 2.6 + margin:
                continue
            out.append((x, y))
        return np.array(out)

    sides = rng.uniform(0.3, 2.0, size=(n_boxes, 3))
    centers = place(n_boxes, 1.0)
    box_lo = np.stack([centers[:, 0] - sides[:, 0] / 2, centers[:, 1] - sides[:, 1] / 2,
                       np.full(n_boxes, ROOM_LO[2])], 1)
    box_hi = np.stack([centers[:, 0] + sides[:, 0] / 2, centers[:, 1] + sides[:, 1] / 2,
                       ROOM_LO[2] + sides[:, 2]], 1)
    cyl_r = rng.uniform(0.1, 0.5, size=n_cyl)
    cyl_xy = place(n_cyl, 0.5)
    return Scene(box_lo, box_hi, cyl_xy, cyl_r)


def uniform_rotation(rng: np.random.Generator) -> np.ndarray:
    # uniform unit quaternion (Shoemake)
    u1, u2, u3 = rng.random(3)
    q = np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)])
    w, x, y, z = q[3], q[0], q[1], q[2]
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def _ray_cast(scene: Scene, origin: np.ndarray, d: np.ndarray):
    """Nearest hit distance and unit normal per ray (world frame)."""
    n = d.shape[0]
    inv = 1.0 / np.where(np.abs(d) < 1e-12, np.copysign(1e-12, d), d)
    # room interior: exit distance of the slab box
    t1 = (ROOM_LO - origin) * inv
    t2 = (ROOM_HI - origin) * inv
    tfar = np.maximum(t1, t2)
    t_best = tfar.min(1)
    ax = tfar.argmin(1)
    normal = np.zeros((n, 3))
    normal[np.arange(n), ax] = -np.sign(d[np.arange(n), ax])
    # boxes: entry distance
    for lo, hi in zip(scene.box_lo, scene.box_hi):
        a = (lo - origin) * inv
        b = (hi - origin) * inv
        tn = np.minimum(a, b)
        tf = np.maximum(a, b)
        tent = tn.max(1)
        texit = tf.min(1)
        hit = (tent <= texit) & (tent > 1e-6) & (tent < t_best)
        if hit.any():
            t_best = np.where(hit, tent, t_best)
            axe = tn.argmax(1)
            nn = np.zeros((n, 3))
            nn[np.arange(n), axe] = -np.sign(d[np.arange(n), axe])
            normal = np.where(hit[:, None], nn, normal)
    # cylinders (vertical, floor to ceiling)
    dx, dy = d[:, 0], d[:, 1]
    A = dx * dx + dy * dy
    for (cx, cy), r in zip(scene.cyl_xy, scene.cyl_r):
        ox, oy = origin[0] - cx, origin[1] - cy
        Bq = 2 * (ox * dx + oy * dy)
        Cq = ox * ox + oy * oy - r * r
        disc = Bq * Bq - 4 * A * Cq
        ok = (disc > 0) & (A > 1e-12)
        t = np.where(ok, (-Bq - np.sqrt(np.maximum(disc, 0))) / (2 * np.maximum(A, 1e-12)), np.inf)
        z = origin[2] + t * d[:, 2]
        hit = ok & (t > 1e-6) & (t < t_best) & (z >= ROOM_LO[2]) & (z <= ROOM_HI[2])
        if hit.any():
            t_best = np.where(hit, t, t_best)
            px = ox + t * dx
            py = oy + t * dy
            nn = np.stack([px / r, py / r, np.zeros(n)], 1)
            normal = np.where(hit[:, None], nn, normal)
    return t_best, normal


def scan(scene: Scene, rng: np.random.Generator, R: np.ndarray, t: np.ndarray, beams: int,
         cols: int, with_reflectivity: bool) -> Cloud:
    el = np.deg2rad(np.linspace(-22.5, 22.5, beams))
    az = 2 * np.pi * np.arange(cols) / cols
    E, A = np.meshgrid(el, az, indexing="ij")
    d_s = np.stack([np.cos(E) * np.cos(A), np.cos(E) * np.sin(A), np.sin(E)], -1).reshape(-1, 3)
    d_w = d_s @ R.T
    with np.errstate(invalid="ignore", over="ignore"):
        rng_true, normal = _ray_cast(scene, t, d_w)
    ok = np.isfinite(rng_true) & (rng_true > 0.05)
    r = rng_true + rng.normal(0.0, 0.01, size=rng_true.shape)
    cosinc = np.abs(np.sum(normal * d_w, 1))
    inten = np.clip(0.5 + 0.3 * cosinc + rng.normal(0.0, 0.05, size=cosinc.shape), 0.0, 1.0)
    pts = d_s * r[:, None]
    pts = pts[ok]
    inten = inten[ok]
    r = r[ok]
    xyzi = np.concatenate([pts, inten[:, None]], 1).astype(np.float32)
    refl = None
    if with_reflectivity:
        rf = inten * r * r
        refl = (rf / max(rf.max(), 1e-12)).astype(np.float32)
    return Cloud(xyzi, refl)


@dataclass
class Pair:
    target: Cloud
    source: Cloud
    R: np.ndarray
    t: np.ndarray


def make_pair(workload: int, k: int, beams: int, cols: int = 1024,
              with_reflectivity: bool = True) -> Pair:
    seed = 1000 * workload + k
    scene_rng = np.random.default_rng([seed, 0])
    pose_rng = np.random.default_rng([seed, 1])
    scene = make_scene(scene_rng)
    R = uniform_rotation(pose_rng)
    t = pose_rng.uniform(-2.0, 2.0, size=3)
    noise_rng = np.random.default_rng([seed, 2])
    src = scan(scene, noise_rng, np.eye(3), np.zeros(3), beams, cols, with_reflectivity)
    tgt = scan(scene, noise_rng, R, t, beams, cols, with_reflectivity)
    return Pair(tgt, src, R, t)


# Workload shapes (beams, columns, B, N, lo, hi, reflectivity)
WORKLOADS = {
    0: dict(beams=64, cols=1024, bw=32, n_voxels=64, lo=-10, hi=10, reflectivity=False),
    1: dict(beams=128, cols=1024, bw=100, n_voxels=200, lo=-10, hi=10, reflectivity=True),
    4: dict(beams=256, cols=4096, bw=256, n_voxels=512, lo=-20, hi=20, reflectivity=True),
}


# Served mix of arrivals (weight, shape): 50 % B = 64 / N = 128, 35 % B = 100 /
# N = 200, 15 % B = 128 / N = 256, all over [-10, 10]^3 m; scans of the
# given beam count x 1024 columns, seeds 1000 * 3 + k.
CONFIG3_MIX = [
    (0.50, dict(beams=64, bw=64, n_voxels=128, lo=-10, hi=10)),
    (0.35, dict(beams=128, bw=100, n_voxels=200, lo=-10, hi=10)),
    (0.15, dict(beams=128, bw=128, n_voxels=256, lo=-10, hi=10)),
]


# Batched workload: independent pairs of the room generator, pair k with its
# own seed (1000 * 2 + k), a beam count from {32, 64, 128} x 1024 columns, B
# from {32, 64, 100, 128} and N from {64, 128, 200} over [-10, 10]^3 m, all
# drawn uniformly from a stream of its own per pair.
CONFIG2_BEAMS = (32, 64, 128)
CONFIG2_B = (32, 64, 100, 128)
CONFIG2_N = (64, 128, 200)


def config2_specs(n: int = 256) -> list[dict]:
    out = []
    for k in range(n):
        rng = np.random.default_rng([2000 + k, 7])
        out.append(dict(k=k, beams=int(rng.choice(CONFIG2_BEAMS)), bw=int(rng.choice(CONFIG2_B)),
                        n_voxels=int(rng.choice(CONFIG2_N)), lo=-10, hi=10))
    return out


def _config2_pair(spec):
    return make_pair(2, spec["k"], spec["beams"])


def config2_pairs(specs, processes: int | None = None) -> list[Pair]:
    """The pairs of config2_specs, generated in spawned processes (safe in a
    process that already uses the GPU)."""
    import multiprocessing as mp
    import os
    n = processes or min(len(specs), os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(n) as pool:
        return pool.map(_config2_pair, specs)


def workload_pair(workload: int, k: int = 0) -> Pair:
    w = WORKLOADS[workload]
    return make_pair(workload, k, w["beams"], w["cols"], w["reflectivity"])


def write_ply(path, xyzi, reflectivity=None):
    """A scan as a binary little-endian PLY with the reference reader's field
    names (x, y, z, intensity[, reflectivity]), float32."""
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
