"""phgpu_sample_s2_noalloc: the sampler without device allocation, against the
context entry point (phgpu_sample_s2 + phgpu_get_samples) on the same device
clouds.  Tolerance: none -- both run the same kernels, so nearest-neighbour
indices and sampled values must be identical.  This file is collected last so
that the check also covers a process whose device already ran every other
test."""
import numpy as np
import pytest

from phaser_b200 import scene


def _clouds():
    pair = scene.make_pair(0, 3, beams=32, cols=512)
    return [pair.target, pair.source]


def _run_noalloc(native, torch, params, cl, values_dev, nn_dev):
    x = torch.from_numpy(np.ascontiguousarray(cl.xyzi, np.float32)).cuda()
    r = None if cl.reflectivity is None else torch.from_numpy(np.ascontiguousarray(cl.reflectivity, np.float32)).cuda()
    values_dev.fill_(float("nan"))
    nn_dev.fill_(-7)
    rc = native.sample_s2_noalloc(params, x, r, None, values_dev, nn_dev, torch.cuda.current_stream())
    assert rc == native.PHGPU_OK
    torch.cuda.synchronize()
    return x, r


def _run_context(native, params, x, r):
    c = native.Context(params)
    try:
        c.sample_s2(x, r, side=0)
        return c.samples(0)
    finally:
        c.close()


@pytest.mark.gpu
def test_noalloc_matches_context_two_calls():
    import torch
    from phaser_b200 import native
    bw = 32
    params = native.default_params(spherical_bandwidth=bw)
    nq = 4 * bw * bw
    values_dev = torch.empty(4 * nq, dtype=torch.float32, device="cuda")
    nn_dev = torch.empty(nq, dtype=torch.int32, device="cuda")
    clouds = _clouds()
    assert clouds[0].xyzi.shape[0] != clouds[1].xyzi.shape[0] or not np.array_equal(clouds[0].xyzi, clouds[1].xyzi)
    for cl in clouds:  # two calls in a row on different clouds
        x, r = _run_noalloc(native, torch, params, cl, values_dev, nn_dev)
        ref_vals, ref_idx = _run_context(native, params, x, r)
        assert np.array_equal(nn_dev.cpu().numpy(), ref_idx)
        np.testing.assert_array_equal(values_dev.cpu().numpy().astype(np.float64).reshape(4, nq), ref_vals)
        assert (ref_idx >= 0).any()


@pytest.mark.gpu
def test_noalloc_bandwidth_change():
    import torch
    from phaser_b200 import native
    cl = _clouds()[0]
    for bw in (16, 24):
        params = native.default_params(spherical_bandwidth=bw)
        nq = 4 * bw * bw
        values_dev = torch.empty(4 * nq, dtype=torch.float32, device="cuda")
        nn_dev = torch.empty(nq, dtype=torch.int32, device="cuda")
        x, r = _run_noalloc(native, torch, params, cl, values_dev, nn_dev)
        ref_vals, ref_idx = _run_context(native, params, x, r)
        assert np.array_equal(nn_dev.cpu().numpy(), ref_idx)
        np.testing.assert_array_equal(values_dev.cpu().numpy().astype(np.float64).reshape(4, nq), ref_vals)


def test_noalloc_rejections():
    """Argument checks happen on the host before any CUDA call."""
    import ctypes as C
    from phaser_b200 import native
    lib = native.load()
    dummy = np.zeros(16, np.float32)  # never dereferenced: every call below is rejected first
    addr = dummy.ctypes.data
    p = native.default_params(spherical_bandwidth=native.NOALLOC_MAX_BANDWIDTH + 1)
    dev_cloud = native.Cloud(addr, None, None, 4, 1)
    assert lib.phgpu_sample_s2_noalloc(C.byref(p), C.byref(dev_cloud), addr, None, None) == native.PHGPU_ERR_LIMIT
    p = native.default_params(spherical_bandwidth=8)
    big = native.Cloud(addr, None, None, native.NOALLOC_MAX_POINTS + 1, 1)
    assert lib.phgpu_sample_s2_noalloc(C.byref(p), C.byref(big), addr, None, None) == native.PHGPU_ERR_LIMIT
    host_cloud = native.Cloud(addr, None, None, 4, 0)
    assert lib.phgpu_sample_s2_noalloc(C.byref(p), C.byref(host_cloud), addr, None, None) == native.PHGPU_ERR_INVALID
    assert lib.phgpu_sample_s2_noalloc(C.byref(p), C.byref(dev_cloud), None, None, None) == native.PHGPU_ERR_INVALID
    assert lib.phgpu_sample_s2_noalloc(None, C.byref(dev_cloud), addr, None, None) == native.PHGPU_ERR_INVALID


@pytest.mark.gpu
def test_noalloc_new_bandwidth_refused_under_capture():
    """A bandwidth change needs a pageable host-to-device copy, which cannot be
    captured: under stream capture the call returns PHGPU_ERR_INVALID and
    enqueues nothing; outside capture the same call then succeeds."""
    import torch
    from phaser_b200 import native
    cl = _clouds()[0]
    x = torch.from_numpy(np.ascontiguousarray(cl.xyzi, np.float32)).cuda()
    bw_a, bw_b = 16, 20
    vals = {bw: torch.empty(16 * bw * bw, dtype=torch.float32, device="cuda") for bw in (bw_a, bw_b)}
    p_a = native.default_params(spherical_bandwidth=bw_a)
    p_b = native.default_params(spherical_bandwidth=bw_b)
    assert native.sample_s2_noalloc(p_a, x, None, None, vals[bw_a], None, torch.cuda.current_stream()) == native.PHGPU_OK
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rc = native.sample_s2_noalloc(p_b, x, None, None, vals[bw_b], None, torch.cuda.current_stream())
    assert rc == native.PHGPU_ERR_INVALID
    del g
    assert native.sample_s2_noalloc(p_b, x, None, None, vals[bw_b], None, torch.cuda.current_stream()) == native.PHGPU_OK
    torch.cuda.synchronize()
    ref_vals, _ = _run_context(native, p_b, x, None)
    np.testing.assert_array_equal(vals[bw_b].cpu().numpy().astype(np.float64).reshape(4, -1), ref_vals)
