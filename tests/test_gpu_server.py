"""Request server (phgpu_server_*): waves of same-shape pairs replayed as CUDA
graphs.  Served poses equal those of the plain context -- bins and voxels --
for host (copied or borrowed) and device inputs, FP32 and tensor-core
precision, and requests of different shapes in flight together; each request's
full correlation volumes are the same alone and in a mixed wave; admission
under a budget below two shapes' working sets evicts and never stalls."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / np.linalg.norm(b))


def _pairs():
    from phaser_b200 import scene
    return [scene.workload_pair(0, k) for k in range(3)]


def _reference_poses(nat, params, pairs):
    c = nat.Context(params)
    out = [c.register_pair((p.target.xyzi, None), (p.source.xyzi, None)) for p in pairs]
    c.close()
    return [(q.rot_bin, q.voxel) for q in out]


@pytest.mark.parametrize("flags,precision", [(0, 0), (1, 0), (0, 1)])
def test_server_matches_context(flags, precision):
    import torch
    from phaser_b200 import native as nat, scene
    w = scene.WORKLOADS[0]
    params = nat.default_params(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"],
                                spatial_discretize_lower=w["lo"], spatial_discretize_upper=w["hi"],
                                precision=precision)
    small = nat.default_params(spherical_bandwidth=16, spatial_n_voxels=32, spatial_discretize_lower=w["lo"],
                               spatial_discretize_upper=w["hi"], precision=precision)
    pairs = _pairs()
    want = _reference_poses(nat, params, pairs)
    want_small = _reference_poses(nat, small, pairs)
    srv = nat.Server(max_wave=4, lanes=2, device=0, flags=flags)
    dev = [((torch.from_numpy(p.target.xyzi).cuda(), None), (torch.from_numpy(p.source.xyzi).cuda(), None))
           for p in pairs]
    tickets = []
    for rep in range(2):
        for i, p in enumerate(pairs):
            tickets.append(("host", i, srv.submit(params, (p.target.xyzi, None), (p.source.xyzi, None))))
            tickets.append(("dev", i, srv.submit(params, *dev[i])))
            tickets.append(("small", i, srv.submit(small, (p.target.xyzi, None), (p.source.xyzi, None))))
    srv.drain()
    for kind, i, t in tickets:
        pose, lat = srv.poll(t)
        expect = want_small[i] if kind == "small" else want[i]
        assert (pose.rot_bin, pose.voxel) == expect, (kind, i)
        assert lat > 0
    st = srv.stats()
    assert st["requests"] == len(tickets)
    assert st["waves"] < len(tickets)  # requests of one shape were batched
    assert st["graph_captures"] >= 1
    srv.close()


def test_alone_vs_mix_volumes():
    """A B=100/N=200 request (bench workload, tensor-core synthesis) gives the
    same bin, voxel and full correlation volumes served alone as in waves
    mixed with other requests of its shape and of two other shapes."""
    from phaser_b200 import native as nat, scene
    w = scene.WORKLOADS[1]
    main = nat.default_params(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"],
                              spatial_discretize_lower=w["lo"], spatial_discretize_upper=w["hi"],
                              flags=nat.PHGPU_FLAG_KEEP_VOLUMES, precision=nat.PHGPU_PRECISION_TF32X3)
    others = [nat.default_params(spherical_bandwidth=b, spatial_n_voxels=n, spatial_discretize_lower=-10,
                                 spatial_discretize_upper=10, precision=nat.PHGPU_PRECISION_TF32X3)
              for b, n in ((64, 128), (32, 64))]
    pairs = [scene.workload_pair(1, k) for k in range(2)]
    clouds = [((p.target.xyzi, p.target.reflectivity), (p.source.xyzi, p.source.reflectivity)) for p in pairs]
    srv = nat.Server(max_wave=8, lanes=2, device=0)
    alone = []
    for c in clouds:
        t = srv.submit(main, *c)
        srv.drain()
        alone.append(srv.poll(t, volumes=True))
    mixed = []
    for rep in range(3):
        for j, c in enumerate(clouds):
            mixed.append((j, srv.submit(main, *c)))
            srv.submit(others[rep % 2], *clouds[1 - j])
    srv.drain()
    for j, t in mixed:
        pose, _, rv, tv = srv.poll(t, volumes=True)
        p0, _, rv0, tv0 = alone[j]
        assert (pose.rot_bin, pose.voxel) == (p0.rot_bin, p0.voxel)
        assert rel_l2(rv, rv0) <= REL_L2
        assert rel_l2(tv, tv0) <= REL_L2
    srv.close()


@pytest.mark.timeout(300)
def test_budget_below_two_shapes_drains():
    """With an HBM budget that holds one executor but not two, requests of two
    shapes alternate: executors are evicted and every request completes."""
    from phaser_b200 import native as nat, scene
    pairs = _pairs()
    shapes = [nat.default_params(spherical_bandwidth=b, spatial_n_voxels=n, spatial_discretize_lower=-10,
                                 spatial_discretize_upper=10) for b, n in ((32, 64), (16, 32))]
    probe = nat.Server(max_wave=2, lanes=1, device=0)
    t = probe.submit(shapes[0], (pairs[0].target.xyzi, None), (pairs[0].source.xyzi, None))
    probe.drain()
    probe.poll(t)
    one = probe.stats()["bytes_in_use"]
    probe.close()
    srv = nat.Server(max_wave=2, lanes=2, device=0, hbm_budget_bytes=int(one * 1.5))
    tickets = []
    for rep in range(6):
        for s in shapes:
            p = pairs[rep % len(pairs)]
            tickets.append(srv.submit(s, (p.target.xyzi, None), (p.source.xyzi, None)))
    srv.drain()
    for t in tickets:
        assert srv.poll(t) is not None
    st = srv.stats()
    assert st["evictions"] >= 1
    assert st["bytes_in_use"] <= int(one * 1.5)
    srv.close()


def test_server_reports_bad_request():
    from phaser_b200 import native as nat
    srv = nat.Server(max_wave=2, lanes=1, device=0)
    bad = nat.default_params(spherical_bandwidth=4, spatial_n_voxels=131)  # prime factor above 128
    pts = np.zeros((8, 4), np.float32)
    pts[:, 0] = np.arange(1, 9)
    t = srv.submit(bad, (pts, None), (pts, None))
    srv.drain()
    with pytest.raises(nat.PhgpuError):
        srv.poll(t)
    srv.close()
