"""Request server (phgpu_server_*): poses of served requests equal those of the
plain context -- bins, voxels and the correlation values at the peaks -- for
host (copied or borrowed) and device inputs and for requests of different
shapes in flight together."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pairs():
    from phaser_b200 import scene
    return [scene.workload_pair(0, k) for k in range(3)]


def _reference_poses(nat, params, pairs):
    c = nat.Context(params)
    out = [c.register_pair((p.target.xyzi, None), (p.source.xyzi, None)) for p in pairs]
    c.close()
    return [(q.rot_bin, q.voxel, q.rot_peak, q.trans_peak) for q in out]


@pytest.mark.parametrize("flags", [0, 1])
def test_server_matches_context(flags):
    import torch
    from phaser_b200 import native as nat, scene
    w = scene.WORKLOADS[0]
    params = nat.default_params(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"],
                                spatial_discretize_lower=w["lo"], spatial_discretize_upper=w["hi"])
    small = nat.default_params(spherical_bandwidth=16, spatial_n_voxels=32, spatial_discretize_lower=w["lo"],
                               spatial_discretize_upper=w["hi"])
    pairs = _pairs()
    want = _reference_poses(nat, params, pairs)
    want_small = _reference_poses(nat, small, pairs)
    srv = nat.Server(workers=3, device=0, flags=flags)
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
        assert (pose.rot_bin, pose.voxel) == expect[:2], (kind, i)
        # the correlation values at the peaks: the same volumes alone and in a
        # mixed wave (voxel sums are float atomics: equal within 1e-5)
        assert pose.rot_peak == pytest.approx(expect[2], rel=1e-5), (kind, i)
        assert pose.trans_peak == pytest.approx(expect[3], rel=1e-5), (kind, i)
        assert lat > 0
    srv.close()


def test_server_reports_bad_request():
    from phaser_b200 import native as nat
    srv = nat.Server(workers=1, device=0)
    bad = nat.default_params(spherical_bandwidth=4, spatial_n_voxels=131)  # prime factor above 128
    pts = np.zeros((8, 4), np.float32)
    pts[:, 0] = np.arange(1, 9)
    t = srv.submit(bad, (pts, None), (pts, None))
    srv.drain()
    with pytest.raises(nat.PhgpuError):
        srv.poll(t)
    srv.close()
