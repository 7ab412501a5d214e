"""ctypes binding of the C ABI in include/phaser_gpu.h.

Loads phaser_b200/_lib/libphaser_gpu.so (built by ``python -m phaser_b200.build``).
There is no CPU fallback: if the library or a CUDA device is missing, every
entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libphaser_gpu.so")

PHGPU_OK = 0
PHGPU_ERR_INVALID = -1
PHGPU_ERR_LIMIT = -5
NOALLOC_MAX_POINTS = 1 << 18
NOALLOC_MAX_BANDWIDTH = 128
PHGPU_FUSION_LAPLACE = 0
PHGPU_FUSION_NONE = 1
PHGPU_FUSION_LOW_PASS = 2
PHGPU_FLAG_KEEP_VOLUMES = 1
PHGPU_SERVER_BORROW_HOST = 1
PHGPU_FUSION_MIX = 3
PHGPU_PRECISION_FP32 = 0
PHGPU_PRECISION_TF32X3 = 1
PHGPU_PRECISION_BF16X3 = 2


class PhgpuError(RuntimeError):
    pass


class Params(C.Structure):
    _fields_ = [
        ("spherical_bandwidth", C.c_uint32),
        ("spherical_zero_padding", C.c_uint32),
        ("spatial_n_voxels", C.c_uint32),
        ("spatial_discretize_lower", C.c_int32),
        ("spatial_discretize_upper", C.c_int32),
        ("spatial_zero_padding", C.c_uint32),
        ("spatial_low_pass_lower", C.c_float),
        ("spatial_low_pass_upper", C.c_float),
        ("n_channels", C.c_uint32),
        ("fusion_levels", C.c_uint32),
        ("spherical_fusion", C.c_uint32),
        ("spatial_fusion", C.c_uint32),
        ("max_points", C.c_uint32),
        ("flags", C.c_uint32),
        ("device", C.c_int32),
        ("rot_peak_neighbors", C.c_uint32),
        ("trans_peak_neighbors", C.c_uint32),
        ("spherical_low_pass_lower", C.c_uint32),
        ("spherical_low_pass_upper", C.c_uint32),
        ("precision", C.c_uint32),
    ]


class Cloud(C.Structure):
    _fields_ = [
        ("xyzi", C.c_void_p),
        ("reflectivity", C.c_void_p),
        ("ambient", C.c_void_p),
        ("n_points", C.c_uint32),
        ("on_device", C.c_int32),
    ]


class Pose(C.Structure):
    _fields_ = [
        ("rot_bin", C.c_uint32),
        ("rot_peak", C.c_float),
        ("zyz", C.c_double * 3),
        ("quat", C.c_double * 4),
        ("xyz", C.c_double * 3),
        ("voxel", C.c_uint32),
        ("trans_peak", C.c_float),
        ("trans", C.c_double * 3),
        ("rot_omega", C.c_double * 4),
        ("trans_cov", C.c_double * 9),
    ]

    def as_dict(self):
        return dict(rot_bin=self.rot_bin, rot_peak=self.rot_peak, zyz=list(self.zyz),
                    quat=list(self.quat), xyz=list(self.xyz), voxel=self.voxel,
                    trans_peak=self.trans_peak, trans=list(self.trans), rot_omega=list(self.rot_omega),
                    trans_cov=list(self.trans_cov))


class ServerParams(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64),
        ("max_wave", C.c_uint32),
        ("max_points", C.c_uint32),
        ("device", C.c_int32),
        ("flags", C.c_uint32),
        ("lanes", C.c_uint32),
        ("max_delay_us", C.c_uint32),
    ]


class Tuning(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("fuse_z_tile", "so3_beta_tile", "tc_chunk", "radix_order")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}

    @classmethod
    def from_dict(cls, d):
        return cls(*[int(d.get(n, 0)) for n, _ in cls._fields_])


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("waves", "requests", "graph_captures", "direct_waves", "evictions", "pose_reruns",
                                          "executors", "bytes_in_use")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


# every symbol the header declares (checked by the CPU tests)
EXPORTED = [
    "phgpu_params_default", "phgpu_ctx_create", "phgpu_ctx_destroy", "phgpu_last_error",
    "phgpu_stream", "phgpu_sample_s2", "phgpu_get_samples", "phgpu_sph_correlate",
    "phgpu_sph_correlate_sampled", "phgpu_sph_result", "phgpu_sph_bandwidth", "phgpu_voxelize",
    "phgpu_get_voxel_index", "phgpu_spatial_correlate", "phgpu_spatial_correlate_voxelized",
    "phgpu_spatial_result", "phgpu_register_pair", "phgpu_pose_from_bin",
    "phgpu_translation_from_index", "phgpu_server_create", "phgpu_server_destroy",
    "phgpu_server_submit", "phgpu_server_poll", "phgpu_server_drain", "phgpu_server_last_error",
    "phgpu_profile_enable", "phgpu_profile_read", "phgpu_profile_stage_count",
    "phgpu_profile_stage_name", "phgpu_launch_count",
    "phgpu_sample_s2_noalloc", "phgpu_bingham_peak", "phgpu_gaussian_peak", "phgpu_peak_window",
    "phgpu_ply_info", "phgpu_ply_read", "phgpu_ply_last_error", "phgpu_voxel_grid_create",
    "phgpu_voxel_grid_destroy", "phgpu_voxel_grid_filter", "phgpu_voxel_grid_last_error",
    "phgpu_spatial_correlation_size", "phgpu_pose_reruns", "phgpu_server_poll_volumes",
    "phgpu_server_get_stats", "phgpu_tuning_get", "phgpu_tuning_set", "phgpu_autotune",
    "phgpu_server_set_tuning", "phgpu_zscore_params_default", "phgpu_zscore_peaks",
]

_LIB = None
_LIB_FILE = None
_BUILD_ID = None


def load(path: str = LIB_PATH):
    """Load the library (no GPU needed just to load it)."""
    global _LIB, _LIB_FILE
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise PhgpuError(f"CUDA library not built: {path} (run python -m phaser_b200.build)")
    lib = C.CDLL(path)
    _LIB_FILE = path
    vp = C.c_void_p
    lib.phgpu_params_default.argtypes = [C.POINTER(Params)]
    lib.phgpu_ctx_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
    lib.phgpu_ctx_destroy.argtypes = [vp]
    lib.phgpu_last_error.restype = C.c_char_p
    lib.phgpu_last_error.argtypes = [vp]
    lib.phgpu_stream.restype = vp
    lib.phgpu_stream.argtypes = [vp]
    lib.phgpu_sample_s2.argtypes = [vp, C.POINTER(Cloud), C.c_int]
    lib.phgpu_get_samples.argtypes = [vp, C.c_int, vp, vp]
    lib.phgpu_sph_correlate.argtypes = [vp, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_uint32]
    lib.phgpu_sph_correlate_sampled.argtypes = [vp]
    lib.phgpu_sph_result.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_float), vp]
    lib.phgpu_sph_bandwidth.restype = C.c_uint32
    lib.phgpu_sph_bandwidth.argtypes = [vp]
    lib.phgpu_spatial_correlation_size.restype = C.c_uint32
    lib.phgpu_spatial_correlation_size.argtypes = [vp]
    lib.phgpu_voxelize.argtypes = [vp, C.POINTER(Cloud), C.c_int, vp]
    lib.phgpu_get_voxel_index.argtypes = [vp, C.c_int, vp, C.c_uint32]
    lib.phgpu_spatial_correlate.argtypes = [vp, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_uint32]
    lib.phgpu_spatial_correlate_voxelized.argtypes = [vp]
    lib.phgpu_spatial_result.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_float), vp]
    lib.phgpu_register_pair.argtypes = [vp, C.POINTER(Cloud), C.POINTER(Cloud), C.POINTER(Pose)]
    lib.phgpu_pose_from_bin.argtypes = [C.c_uint32, C.c_uint32, vp, vp, vp, vp]
    lib.phgpu_translation_from_index.restype = C.c_double
    lib.phgpu_translation_from_index.argtypes = [C.c_double, C.c_uint32, C.c_int32, C.c_int32]
    lib.phgpu_server_create.argtypes = [C.POINTER(ServerParams), C.POINTER(vp)]
    lib.phgpu_server_destroy.argtypes = [vp]
    lib.phgpu_server_submit.argtypes = [vp, C.POINTER(Params), C.POINTER(Cloud), C.POINTER(Cloud),
                                        C.POINTER(C.c_uint64)]
    lib.phgpu_server_poll.argtypes = [vp, C.c_uint64, C.POINTER(Pose), C.POINTER(C.c_double)]
    lib.phgpu_server_drain.argtypes = [vp]
    lib.phgpu_server_poll_volumes.argtypes = [vp, C.c_uint64, C.POINTER(Pose), C.POINTER(C.c_double), vp, vp]
    lib.phgpu_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
    lib.phgpu_tuning_get.argtypes = [vp, C.POINTER(Tuning)]
    lib.phgpu_tuning_set.argtypes = [vp, C.POINTER(Tuning)]
    lib.phgpu_autotune.argtypes = [vp, C.POINTER(Cloud), C.POINTER(Cloud), C.c_uint32, C.POINTER(Tuning),
                                   C.POINTER(C.c_double)]
    lib.phgpu_server_set_tuning.argtypes = [vp, C.POINTER(Params), C.POINTER(Tuning)]
    lib.phgpu_server_last_error.restype = C.c_char_p
    lib.phgpu_server_last_error.argtypes = [vp]
    lib.phgpu_profile_enable.argtypes = [vp, C.c_int]
    lib.phgpu_profile_read.argtypes = [vp, vp, vp, C.c_int]
    lib.phgpu_profile_stage_count.restype = C.c_int
    lib.phgpu_profile_stage_name.restype = C.c_char_p
    lib.phgpu_profile_stage_name.argtypes = [C.c_int]
    lib.phgpu_launch_count.restype = C.c_ulonglong
    lib.phgpu_pose_reruns.restype = C.c_ulonglong
    lib.phgpu_pose_reruns.argtypes = [vp]
    lib.phgpu_bingham_peak.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
    lib.phgpu_gaussian_peak.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32, C.c_int32,
                                        C.c_void_p, C.c_void_p]
    lib.phgpu_peak_window.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32)]
    lib.phgpu_peak_window.restype = None
    lib.phgpu_zscore_params_default.argtypes = [C.POINTER(ZScoreParams)]
    lib.phgpu_zscore_peaks.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(ZScoreParams), C.c_void_p, C.c_uint64,
                                       C.POINTER(C.c_uint64)]
    lib.phgpu_sample_s2_noalloc.argtypes = [C.POINTER(Params), C.POINTER(Cloud), C.c_void_p, C.c_void_p,
                                            C.c_void_p]
    lib.phgpu_ply_info.argtypes = [C.c_char_p, C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    lib.phgpu_ply_read.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_uint32, C.POINTER(C.c_uint32)]
    lib.phgpu_ply_last_error.restype = C.c_char_p
    lib.phgpu_ply_last_error.argtypes = []
    lib.phgpu_voxel_grid_create.argtypes = [C.c_uint32, C.c_int32, C.POINTER(vp)]
    lib.phgpu_voxel_grid_destroy.argtypes = [vp]
    lib.phgpu_voxel_grid_filter.argtypes = [vp, C.POINTER(Cloud), C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_int, C.POINTER(C.c_uint32)]
    lib.phgpu_voxel_grid_last_error.restype = C.c_char_p
    lib.phgpu_voxel_grid_last_error.argtypes = [vp]
    _LIB = lib
    return lib



def build_id() -> str:
    """Identity of the loaded library build: the first 12 hex digits of the
    SHA-1 of its file (autotuned parameters are kept per build, since a
    kernel change can move the best launch parameters)."""
    global _BUILD_ID
    if _BUILD_ID is None:
        import hashlib
        load()
        h = hashlib.sha1()
        with open(_LIB_FILE, "rb") as f:
            for chunk in iter(lambda: f.read(1 << 20), b""):
                h.update(chunk)
        _BUILD_ID = h.hexdigest()[:12]
    return _BUILD_ID

def default_params(**kw) -> Params:
    p = Params()
    load().phgpu_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _addr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    # torch tensor
    return a.data_ptr()


def _check_device_tensor(name, t, dtype, min_numel, device):
    """A CUDA tensor the C ABI may write or read `min_numel` elements of."""
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name}: expected a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name}: expected dtype {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")
    if t.numel() < min_numel:
        raise ValueError(f"{name}: {t.numel()} elements, at least {min_numel} needed")
    if device is not None and t.device != device:
        raise ValueError(f"{name}: on {t.device}, expected {device}")


def make_cloud(xyzi, reflectivity=None, ambient=None) -> tuple[Cloud, list]:
    """Build a phgpu_cloud from numpy arrays (host) or torch tensors.

    CUDA tensors are passed to the device code as they are, so they are
    checked first: xyzi float32 contiguous of shape (n, 4), reflectivity /
    ambient None or float32 contiguous with at least n elements on the same
    device (ValueError otherwise).  Host inputs are converted to contiguous
    float32 and must have shape (n, 4) too."""
    keep = []
    on_dev = 0
    host_tensor = False
    try:
        import torch
        if isinstance(xyzi, torch.Tensor):
            on_dev = 1 if xyzi.is_cuda else 0
            # float32 contiguous host tensors (pinned ones included) are read in place
            host_tensor = not on_dev and all(
                t is None or (isinstance(t, torch.Tensor) and not t.is_cuda and t.dtype == torch.float32
                              and t.is_contiguous()) for t in (xyzi, reflectivity, ambient))
    except Exception:  # pragma: no cover - torch is always present here
        pass
    if on_dev:
        import torch
        if xyzi.dim() != 2 or xyzi.shape[1] != 4:
            raise ValueError(f"xyzi: expected shape (n, 4), got {tuple(xyzi.shape)}")
        _check_device_tensor("xyzi", xyzi, torch.float32, 4 * xyzi.shape[0], None)
        for name, t in (("reflectivity", reflectivity), ("ambient", ambient)):
            if t is not None:
                _check_device_tensor(name, t, torch.float32, xyzi.shape[0], xyzi.device)
    elif not host_tensor:
        xyzi = np.ascontiguousarray(xyzi, np.float32)
        reflectivity = None if reflectivity is None else np.ascontiguousarray(reflectivity, np.float32)
        ambient = None if ambient is None else np.ascontiguousarray(ambient, np.float32)
    if not on_dev:
        if xyzi.ndim != 2 or xyzi.shape[1] != 4:
            raise ValueError(f"xyzi: expected shape (n, 4), got {tuple(xyzi.shape)}")
        for name, t in (("reflectivity", reflectivity), ("ambient", ambient)):
            if t is not None and (t.ndim != 1 or t.shape[0] < xyzi.shape[0]):
                raise ValueError(f"{name}: expected at least {xyzi.shape[0]} values")
            if t is not None and getattr(t, "is_cuda", False):
                raise ValueError(f"{name}: on the device while xyzi is on the host")
    keep += [xyzi, reflectivity, ambient]
    n = int(xyzi.shape[0])
    c = Cloud(_addr(xyzi), _addr(reflectivity), _addr(ambient), n, on_dev)
    return c, keep


def sample_s2_noalloc(params: Params, xyzi, reflectivity, ambient, values_dev, nn_index_dev=None,
                      stream=None) -> int:
    """phgpu_sample_s2_noalloc on device tensors; returns the status code.
    values_dev: float32 CUDA tensor of 4 * 4bw^2, nn_index_dev: int32 of 4bw^2
    or None; stream: a torch.cuda.Stream (None = legacy default stream).
    Every tensor is checked before the call (ValueError): the cloud as in
    make_cloud and on the device, the outputs on the cloud's device with
    enough elements of the right type."""
    import torch
    if not (isinstance(xyzi, torch.Tensor) and xyzi.is_cuda):
        raise ValueError("xyzi: phgpu_sample_s2_noalloc reads a CUDA tensor")
    c, keep = make_cloud(xyzi, reflectivity, ambient)
    nq = 4 * params.spherical_bandwidth * params.spherical_bandwidth
    _check_device_tensor("values_dev", values_dev, torch.float32, 4 * nq, xyzi.device)
    if nn_index_dev is not None:
        _check_device_tensor("nn_index_dev", nn_index_dev, torch.int32, nq, xyzi.device)
    return load().phgpu_sample_s2_noalloc(C.byref(params), C.byref(c), _addr(values_dev), _addr(nn_index_dev),
                                          None if stream is None else stream.cuda_stream)


class ZScoreParams(C.Structure):
    """phgpu_zscore_params (the reference's z_score_* flags)."""
    _fields_ = [
        ("lag_percentile", C.c_double),
        ("lag_max", C.c_uint32),
        ("threshold", C.c_double),
        ("influence", C.c_double),
        ("filter_threshold", C.c_double),
    ]


def zscore_peaks(values, **overrides):
    """Smoothed z-score peaks of a correlation vector (ZScorePeakExtraction::
    extractPeaks): ascending indices (uint32).  Keyword overrides of the
    defaults: lag_percentile, lag_max, threshold, influence, filter_threshold."""
    lib = load()
    p = ZScoreParams()
    lib.phgpu_zscore_params_default(C.byref(p))
    for k, v in overrides.items():
        if k not in dict(ZScoreParams._fields_):
            raise ValueError(f"unknown z-score parameter {k!r}")
        setattr(p, k, v)
    v = np.ascontiguousarray(values, np.float64).reshape(-1)
    out = np.zeros(max(v.size, 1), np.uint32)
    n = C.c_uint64()
    rc = lib.phgpu_zscore_peaks(v.ctypes.data, v.size, C.byref(p), out.ctypes.data, out.size, C.byref(n))
    if rc != PHGPU_OK:
        raise PhgpuError(f"phgpu_zscore_peaks failed ({rc})")
    return out[:n.value].copy()


def peak_window(index, n, k):
    """Linear-index window (first, count) of k neighbours around an argmax."""
    f, c = C.c_uint32(), C.c_uint32()
    load().phgpu_peak_window(int(index), int(n), int(k), C.byref(f), C.byref(c))
    return f.value, c.value


def bingham_peak(values, first_bin, bw_out):
    """Mode quaternion (w, x, y, z), normalised scatter eigenvalues and XYZ
    angles of the weighted bins first_bin .. first_bin + len(values) - 1."""
    v = np.ascontiguousarray(values, np.float64)
    mode, omega, xyz = np.zeros(4), np.zeros(4), np.zeros(3)
    rc = load().phgpu_bingham_peak(v.ctypes.data, int(first_bin), len(v), int(bw_out), mode.ctypes.data,
                                   omega.ctypes.data, xyz.ctypes.data)
    if rc != PHGPU_OK:
        raise PhgpuError(f"phgpu_bingham_peak failed ({rc})")
    return mode, omega, xyz


def gaussian_peak(values, first_voxel, n_voxels, lower, upper):
    """Weighted mean and covariance (3x3) of the translations of the voxels
    first_voxel .. first_voxel + len(values) - 1."""
    v = np.ascontiguousarray(values, np.float64)
    mean, cov = np.zeros(3), np.zeros(9)
    rc = load().phgpu_gaussian_peak(v.ctypes.data, int(first_voxel), len(v), int(n_voxels), int(lower), int(upper),
                                    mean.ctypes.data, cov.ctypes.data)
    if rc != PHGPU_OK:
        raise PhgpuError(f"phgpu_gaussian_peak failed ({rc})")
    return mean, cov.reshape(3, 3)


PHGPU_PLY_REFLECTIVITY = 1
PHGPU_PLY_AMBIENT = 2
PHGPU_PLY_RANGE = 4


def _ply_names(field_names):
    if field_names is None:
        return None, None
    names = [None if f is None else f.encode() for f in field_names]
    names += [None] * (4 - len(names))
    arr = (C.c_char_p * 4)(*names[:4])
    return C.cast(arr, C.c_void_p), arr


def ply_info(path, field_names=None):
    """(vertex count, PHGPU_PLY_* bits of the optional fields present)."""
    names, keep = _ply_names(field_names)
    n, present = C.c_uint32(), C.c_uint32()
    lib = load()
    rc = lib.phgpu_ply_info(os.fsencode(path), names, C.byref(n), C.byref(present))
    if rc != PHGPU_OK:
        raise PhgpuError(f"phgpu_ply_info: {lib.phgpu_ply_last_error().decode(errors="replace")} ({rc})")
    return n.value, present.value


def ply_read(path, field_names=None, pinned=False):
    """Read a PLY file: dict with xyzi (n x 4 float32) and reflectivity,
    ambient, range (float32 arrays, or None when the field is absent).
    field_names: intensity, reflectivity, ambient, range property names
    (None entries keep "intensity", "reflectivity", "noise", "range").
    pinned=True returns page-locked torch tensors ready for an async upload."""
    n, present = ply_info(path, field_names)
    if pinned:
        import torch

        def buf(shape):
            return torch.empty(shape, dtype=torch.float32, pin_memory=True)
    else:
        def buf(shape):
            return np.empty(shape, np.float32)
    xyzi = buf((n, 4))
    opt = {k: (buf((n,)) if present & bit else None) for k, bit in
           (("reflectivity", PHGPU_PLY_REFLECTIVITY), ("ambient", PHGPU_PLY_AMBIENT), ("range", PHGPU_PLY_RANGE))}
    names, keep = _ply_names(field_names)
    got = C.c_uint32()
    lib = load()
    rc = lib.phgpu_ply_read(os.fsencode(path), names, _addr(xyzi) if n else _addr(buf((1, 4))),
                            _addr(opt["reflectivity"]), _addr(opt["ambient"]), _addr(opt["range"]), n,
                            C.byref(got))
    if rc != PHGPU_OK:
        raise PhgpuError(f"phgpu_ply_read: {lib.phgpu_ply_last_error().decode(errors="replace")} ({rc})")
    return dict(xyzi=xyzi, **opt)


class VoxelGrid:
    """GPU pcl::VoxelGrid<PointXYZI> (phgpu_voxel_grid_*): leaf centroids of
    a cloud, leaves in increasing index order."""

    def __init__(self, max_points: int, device: int = 0):
        lib = load()
        h = C.c_void_p()
        rc = lib.phgpu_voxel_grid_create(int(max_points), int(device), C.byref(h))
        if rc != PHGPU_OK:
            raise PhgpuError(f"phgpu_voxel_grid_create: {lib.phgpu_voxel_grid_last_error(None).decode(errors="replace")} ({rc})")
        self._h = h
        self.max_points = int(max_points)
        self.device = int(device)

    def filter(self, xyzi, leaf=(0.25, 0.25, 0.25), min_points_per_voxel=0, reflectivity=None, ambient=None,
               out_device=False):
        """Returns (xyzi, reflectivity, ambient) of the leaf centroids (the
        last two None unless given).  Host inputs give numpy outputs;
        out_device=True returns CUDA tensors instead."""
        lib = load()
        c, keep = make_cloud(xyzi, reflectivity, ambient)
        n = int(c.n_points)
        cap = max(n, 1)
        if out_device:
            import torch
            dev = torch.device("cuda", self.device)
            o = torch.empty((cap, 4), dtype=torch.float32, device=dev)
            orf = torch.empty(cap, dtype=torch.float32, device=dev) if reflectivity is not None else None
            oam = torch.empty(cap, dtype=torch.float32, device=dev) if ambient is not None else None
        else:
            o = np.empty((cap, 4), np.float32)
            orf = np.empty(cap, np.float32) if reflectivity is not None else None
            oam = np.empty(cap, np.float32) if ambient is not None else None
        lf = np.ascontiguousarray(np.broadcast_to(np.asarray(leaf, np.float32), (3,)))
        m = C.c_uint32()
        rc = lib.phgpu_voxel_grid_filter(self._h, C.byref(c), lf.ctypes.data, int(min_points_per_voxel), _addr(o),
                                         _addr(orf), _addr(oam), 1 if out_device else 0, C.byref(m))
        if rc != PHGPU_OK:
            raise PhgpuError(f"phgpu_voxel_grid_filter: {lib.phgpu_voxel_grid_last_error(self._h).decode(errors="replace")} ({rc})")
        k = m.value
        return o[:k], None if orf is None else orf[:k], None if oam is None else oam[:k]

    def close(self):
        if self._h:
            load().phgpu_voxel_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def launch_count() -> int:
    return int(load().phgpu_launch_count())


def translation_from_index(index, n_voxels, lower, upper) -> float:
    return load().phgpu_translation_from_index(float(index), int(n_voxels), int(lower), int(upper))


def pose_from_bin(bin_, bw_out):
    zyz = np.zeros(3)
    q = np.zeros(4)
    xyz = np.zeros(3)
    T = np.zeros(12, np.float32)
    load().phgpu_pose_from_bin(int(bin_), int(bw_out), zyz.ctypes.data, q.ctypes.data, xyz.ctypes.data,
                               T.ctypes.data)
    return zyz, q, xyz, T.reshape(3, 4)


class Context:
    """One configuration's device state (C ABI phgpu_ctx)."""

    def __init__(self, params: Params | None = None, **kw):
        lib = load()
        self.params = params if params is not None else default_params(**kw)
        if params is not None:
            for k, v in kw.items():
                setattr(self.params, k, v)
        h = C.c_void_p()
        rc = lib.phgpu_ctx_create(C.byref(self.params), C.byref(h))
        if rc != PHGPU_OK:
            raise PhgpuError(f"phgpu_ctx_create failed ({rc}): {lib.phgpu_last_error(None).decode(errors="replace")}")
        self.h = h
        self.lib = lib

    def close(self):
        if getattr(self, "h", None):
            self.lib.phgpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        if rc != PHGPU_OK:
            raise PhgpuError(f"phaser_gpu error {rc}: {self.lib.phgpu_last_error(self.h).decode(errors="replace")}")

    @property
    def bw(self):
        return self.params.spherical_bandwidth

    @property
    def bw_out(self):
        return self.params.spherical_bandwidth + self.params.spherical_zero_padding

    @property
    def n_voxels(self):
        return self.params.spatial_n_voxels

    @property
    def stream(self):
        return self.lib.phgpu_stream(self.h)

    # ---- tracing
    def profile(self, enable=True, serial=False):
        """Per-stage CUDA events; serial=True puts both halves of a
        registration on one stream so the stage times do not overlap."""
        self.check(self.lib.phgpu_profile_enable(self.h, (2 if serial else 1) if enable else 0))

    def profile_read(self):
        n = self.lib.phgpu_profile_stage_count()
        ms = np.zeros(n)
        calls = np.zeros(n, np.uint64)
        self.check(self.lib.phgpu_profile_read(self.h, ms.ctypes.data, calls.ctypes.data, n))
        names = [self.lib.phgpu_profile_stage_name(i).decode() for i in range(n)]
        return {nm: (float(ms[i]), int(calls[i])) for i, nm in enumerate(names)}

    # ---- sampling
    def sample_s2(self, xyzi, reflectivity=None, ambient=None, side=0):
        c, keep = make_cloud(xyzi, reflectivity, ambient)
        self.check(self.lib.phgpu_sample_s2(self.h, C.byref(c), side))

    def samples(self, side):
        nq = 4 * self.bw * self.bw
        v = np.zeros(4 * nq)
        idx = np.zeros(nq, np.int32)
        self.check(self.lib.phgpu_get_samples(self.h, side, v.ctypes.data, idx.ctypes.data))
        return v.reshape(4, nq), idx

    # ---- rotation
    def sph_correlate(self, f, g):
        f = [np.ascontiguousarray(x, np.float64) for x in f]
        g = [np.ascontiguousarray(x, np.float64) for x in g]
        fp = (C.c_void_p * len(f))(*[x.ctypes.data for x in f])
        gp = (C.c_void_p * len(g))(*[x.ctypes.data for x in g])
        self.check(self.lib.phgpu_sph_correlate(self.h, fp, gp, len(f)))

    def sph_correlate_sampled(self):
        self.check(self.lib.phgpu_sph_correlate_sampled(self.h))

    def sph_result(self, volume=False):
        b = C.c_uint32()
        pk = C.c_float()
        vol = np.zeros((2 * self.bw_out) ** 3) if volume else None
        self.check(self.lib.phgpu_sph_result(self.h, C.byref(b), C.byref(pk),
                                             None if vol is None else vol.ctypes.data))
        return (b.value, pk.value, vol) if volume else (b.value, pk.value)

    # ---- translation
    def voxelize(self, xyzi, reflectivity=None, ambient=None, side=0, T=None):
        c, keep = make_cloud(xyzi, reflectivity, ambient)
        Tp = None
        if T is not None:
            T = np.ascontiguousarray(T, np.float32).reshape(12)
            Tp = T.ctypes.data
        self.check(self.lib.phgpu_voxelize(self.h, C.byref(c), side, Tp))

    def voxel_index(self, side, n_points):
        out = np.zeros(n_points, np.uint32)
        self.check(self.lib.phgpu_get_voxel_index(self.h, side, out.ctypes.data, n_points))
        return out

    def spatial_correlate(self, f, g):
        f = [np.ascontiguousarray(x, np.float64) for x in f]
        g = [np.ascontiguousarray(x, np.float64) for x in g]
        fp = (C.c_void_p * len(f))(*[x.ctypes.data for x in f])
        gp = (C.c_void_p * len(g))(*[x.ctypes.data for x in g])
        self.check(self.lib.phgpu_spatial_correlate(self.h, fp, gp, len(f)))

    def spatial_correlate_voxelized(self):
        self.check(self.lib.phgpu_spatial_correlate_voxelized(self.h))

    def spatial_result(self, volume=False):
        v = C.c_uint32()
        pk = C.c_float()
        vol = np.zeros(self.lib.phgpu_spatial_correlation_size(self.h)) if volume else None
        self.check(self.lib.phgpu_spatial_result(self.h, C.byref(v), C.byref(pk),
                                                 None if vol is None else vol.ctypes.data))
        return (v.value, pk.value, vol) if volume else (v.value, pk.value)

    # ---- full pipeline
    # ---- tuning
    def tuning(self) -> dict:
        t = Tuning()
        self.check(self.lib.phgpu_tuning_get(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, tuning: dict):
        t = Tuning.from_dict(tuning)
        self.check(self.lib.phgpu_tuning_set(self.h, C.byref(t)))

    def autotune(self, target, source, reps=3):
        """Coordinate search over the launch parameters on this pair; keeps and
        returns the fastest (dict) and the registration's device ms under it."""
        ct, k1 = make_cloud(*target)
        cs, k2 = make_cloud(*source)
        t = Tuning()
        ms = C.c_double()
        self.check(self.lib.phgpu_autotune(self.h, C.byref(ct), C.byref(cs), int(reps), C.byref(t), C.byref(ms)))
        return t.as_dict(), ms.value

    def pose_reruns(self) -> int:
        """Translations register_pair redid with the host transform."""
        return int(self.lib.phgpu_pose_reruns(self.h))

    def register_pair(self, target, source) -> Pose:
        """target/source: (xyzi, reflectivity) tuples of numpy arrays or torch CUDA tensors."""
        ct, k1 = make_cloud(*target)
        cs, k2 = make_cloud(*source)
        pose = Pose()
        self.check(self.lib.phgpu_register_pair(self.h, C.byref(ct), C.byref(cs), C.byref(pose)))
        return pose


class Server:
    """Continuous-batching request server (C ABI phgpu_server_*): waves of up
    to max_wave same-shape pairs, `lanes` waves in flight."""

    def __init__(self, max_wave=16, hbm_budget_bytes=150 << 30, max_points=1 << 18, device=0, flags=0, lanes=2,
                 max_delay_us=500):
        lib = load()
        self.lib = lib
        sp = ServerParams(int(hbm_budget_bytes), int(max_wave), int(max_points), int(device), int(flags), int(lanes),
                          int(max_delay_us))
        h = C.c_void_p()
        rc = lib.phgpu_server_create(C.byref(sp), C.byref(h))
        if rc != PHGPU_OK:
            raise PhgpuError(f"phgpu_server_create failed ({rc})")
        self.h = h
        self._keep = {}
        self._vol = {}
        self._borrow = bool(int(flags) & PHGPU_SERVER_BORROW_HOST)

    def submit(self, params: Params, target, source) -> int:
        ct, k1 = make_cloud(*target)
        cs, k2 = make_cloud(*source)
        t = C.c_uint64()
        rc = self.lib.phgpu_server_submit(self.h, C.byref(params), C.byref(ct), C.byref(cs), C.byref(t))
        if rc != PHGPU_OK:
            raise PhgpuError(f"submit failed ({rc}): {self.lib.phgpu_server_last_error(self.h).decode(errors="replace")}")
        if (ct.on_device and cs.on_device) or self._borrow:
            self._keep[t.value] = (k1, k2)  # read in place until the ticket completes
        if params.flags & PHGPU_FLAG_KEEP_VOLUMES:
            bo = params.spherical_bandwidth + params.spherical_zero_padding
            self._vol[t.value] = ((2 * bo) ** 3, params.spatial_n_voxels ** 3)
        return t.value

    def poll(self, ticket, volumes=False):
        """None while running; (pose, latency_ms) when done, plus the rotation
        and translation volumes when volumes=True (submitted with
        PHGPU_FLAG_KEEP_VOLUMES)."""
        pose = Pose()
        lat = C.c_double()
        rv = tv = None
        if volumes:
            nr, nt = self._vol[ticket]
            rv = np.zeros(nr, np.float32)
            tv = np.zeros(nt, np.float32)
        rc = self.lib.phgpu_server_poll_volumes(self.h, C.c_uint64(ticket), C.byref(pose), C.byref(lat),
                                                rv.ctypes.data if volumes else None,
                                                tv.ctypes.data if volumes else None)
        if rc < 0:
            raise PhgpuError(f"request {ticket} failed ({rc}): {self.lib.phgpu_server_last_error(self.h).decode(errors="replace")}")
        if rc == 0:
            return None
        self._keep.pop(ticket, None)
        self._vol.pop(ticket, None)
        if volumes:
            return pose, lat.value, rv, tv
        return pose, lat.value

    def set_tuning(self, params: Params, tuning: dict):
        t = Tuning.from_dict(tuning)
        rc = self.lib.phgpu_server_set_tuning(self.h, C.byref(params), C.byref(t))
        if rc != PHGPU_OK:
            raise PhgpuError(f"set_tuning failed ({rc})")

    def stats(self) -> dict:
        st = ServerStats()
        rc = self.lib.phgpu_server_get_stats(self.h, C.byref(st))
        if rc != PHGPU_OK:
            raise PhgpuError(f"stats failed ({rc})")
        return st.as_dict()

    def drain(self):
        rc = self.lib.phgpu_server_drain(self.h)
        if rc != PHGPU_OK:
            raise PhgpuError(f"drain failed ({rc})")

    def close(self):
        if getattr(self, "h", None):
            self.lib.phgpu_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
