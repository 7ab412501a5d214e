"""The batched workload: 256 independent pairs (beams {32, 64, 128} x 1024,
B {32, 64, 100, 128}, N {64, 128, 200}: twelve shapes) through the server in
size-grouped waves with the tensor-core synthesis and autotuned launch
parameters.  Every served pose equals the plain (FP32, one pair at a time)
GPU path's; a seeded subset of one pair per shape equals the FP64 oracle."""
import concurrent.futures as cf

import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    from phaser_b200 import scene
    specs = scene.config2_specs(256)
    return specs, scene.config2_pairs(specs)


def test_config2_waves_match_plain_and_oracle(batch, tmp_path):
    from phaser_b200 import native as nat, tuning
    specs, pairs = batch
    nat.load()
    shapes = sorted({(s["bw"], s["n_voxels"]) for s in specs})
    assert len(shapes) == 12

    def params(b, n, prec):
        return nat.default_params(spherical_bandwidth=b, spatial_n_voxels=n, spatial_discretize_lower=-10,
                                  spatial_discretize_upper=10, precision=prec)

    clouds = [((p.target.xyzi, p.target.reflectivity), (p.source.xyzi, p.source.reflectivity)) for p in pairs]
    first = {}
    for i, s in enumerate(specs):
        first.setdefault((s["bw"], s["n_voxels"]), i)
    srv = nat.Server(max_wave=16, lanes=2, flags=nat.PHGPU_SERVER_BORROW_HOST)
    for sh in shapes:
        sp = params(*sh, nat.PHGPU_PRECISION_TF32X3)
        t = tuning.tuned(sp, *clouds[first[sh]], reps=2, path=str(tmp_path / "tuning.json"))
        srv.set_tuning(sp, t["tuning"])
    tickets = [srv.submit(params(s["bw"], s["n_voxels"], nat.PHGPU_PRECISION_TF32X3), *clouds[i])
               for i, s in enumerate(specs)]
    srv.drain()
    served = [srv.poll(t)[0] for t in tickets]
    st = srv.stats()
    srv.close()
    print(f"\n256 pairs, 12 shapes: {st['waves']} waves, {st['graph_captures']} graph captures, "
          f"{st['pose_reruns']} pose reruns")
    assert st["requests"] == 256 and st["waves"] < 256
    plain = [None] * len(specs)
    for sh in shapes:
        c = nat.Context(params(*sh, nat.PHGPU_PRECISION_FP32), max_points=1 << 18)
        for i, s in enumerate(specs):
            if (s["bw"], s["n_voxels"]) == sh:
                plain[i] = c.register_pair(*clouds[i])
        c.close()
    diff = [(i, specs[i]["bw"], specs[i]["n_voxels"], (served[i].rot_bin, served[i].voxel),
             (plain[i].rot_bin, plain[i].voxel)) for i in range(len(specs))
            if (served[i].rot_bin, served[i].voxel) != (plain[i].rot_bin, plain[i].voxel)]
    for d in diff:
        print("served != plain:", d)
    assert diff == []

    def oracle(i):
        s, p = specs[i], pairs[i]
        return O.register_pair(p.target.xyzi, p.target.reflectivity, p.source.xyzi, p.source.reflectivity,
                               s["bw"], s["n_voxels"], -10, 10)

    subset = [first[sh] for sh in shapes]
    with cf.ThreadPoolExecutor(max_workers=6) as ex:
        want = list(ex.map(oracle, subset))
    for i, w in zip(subset, want):
        assert (served[i].rot_bin, served[i].voxel) == (w.rot_bin, w.voxel), specs[i]
