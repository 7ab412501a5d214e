"""The Python binding checks CUDA tensors before handing their pointers to the
C ABI: wrong shapes, dtypes, layouts, devices or sizes raise ValueError and
no kernel runs on them."""
import pytest

pytestmark = pytest.mark.gpu


def test_device_cloud_and_output_checks():
    import torch
    from phaser_b200 import native
    native.load()
    dev = torch.device("cuda:0")
    x = torch.zeros(100, 4, device=dev)
    p = native.default_params(spherical_bandwidth=8)
    nq = 4 * 8 * 8
    out = torch.zeros(4 * nq, device=dev)
    bad_clouds = [
        (torch.zeros(100, 3, device=dev), None),                    # (n, 3)
        (torch.zeros(100, 4, device=dev, dtype=torch.float64), None),  # float64
        (torch.zeros(4, 100, device=dev).t(), None),                # not contiguous
        (x, torch.zeros(100)),                                      # reflectivity on the host
        (x, torch.zeros(50, device=dev)),                           # reflectivity too short
    ]
    for xyzi, refl in bad_clouds:
        with pytest.raises(ValueError):
            native.make_cloud(xyzi, refl)
    with pytest.raises(ValueError):
        native.sample_s2_noalloc(p, x, None, None, torch.zeros(4 * nq - 1, device=dev))
    with pytest.raises(ValueError):
        native.sample_s2_noalloc(p, x, None, None, torch.zeros(4 * nq))  # output on the host
    with pytest.raises(ValueError):
        native.sample_s2_noalloc(p, x, None, None, out, torch.zeros(nq, device=dev))  # float32 indices
    assert native.sample_s2_noalloc(p, x, None, None, out, torch.zeros(nq, device=dev, dtype=torch.int32)) == 0
