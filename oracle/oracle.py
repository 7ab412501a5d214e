"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` import this module, always as the
checker or the timed CPU baseline, never as part of the product path.

``lib()`` loads ``oracle/_build/liboracle.so`` (the FP64 restatement);
``ref_lib()`` loads ``oracle/_ref/libphaser_ref.so`` (the reference's own SOFT
sources built with the project's FFTW-API shim and the restated phaser_core
glue).  Both are built by ``oracle/Makefile``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class Pose(C.Structure):
    _fields_ = [
        ("rot_bin", C.c_uint32),
        ("rot_peak", C.c_double),
        ("zyz", C.c_double * 3),
        ("quat", C.c_double * 4),
        ("xyz", C.c_double * 3),
        ("voxel", C.c_uint32),
        ("trans_peak", C.c_double),
        ("trans", C.c_double * 3),
    ]


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree exists, oracle/_ref)."""
    targets = ["all"]
    # the reference tree beside the repository unless PHASER_REF_ROOT names it
    ref_root = os.environ.get("PHASER_REF_ROOT",
                              os.path.abspath(os.path.join(HERE, os.pardir, os.pardir, "reference")))
    if ref and os.path.isdir(os.path.join(ref_root, "phaser_core", "lib", "SOFT")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF_ROOT={ref_root}"] + targets,
                   check=True)


def _declare(lib):
    lib.orc_fft1d.argtypes = [_f64p, C.c_int, C.c_int]
    lib.orc_sub2ind.restype = C.c_uint32
    lib.orc_sub2ind.argtypes = [C.c_uint32] * 5
    lib.orc_ind2sub.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, _u32p]
    lib.orc_fftshift.argtypes = [_f64p, C.c_size_t]
    lib.orc_ifftshift.argtypes = [_f64p, C.c_size_t]
    lib.orc_pyramid_struct.argtypes = [C.c_uint32, C.c_int, C.c_float, _u32p, _u32p, _u32p]
    lib.orc_fuse_channels_literal.argtypes = [_f64p, C.c_int, C.c_uint32, C.c_int, C.c_float, _f64p]
    lib.orc_fusion_rule.restype = C.c_int
    lib.orc_fusion_rule.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.c_float]
    lib.orc_dh_grid.argtypes = [C.c_int, _f32p]
    lib.orc_dh_weights.argtypes = [C.c_int, _f64p]
    lib.orc_project.argtypes = [_f32p, C.c_size_t, C.c_size_t, _f32p, _f64p]
    lib.orc_nn.argtypes = [_f32p, C.c_size_t, _f32p, C.c_size_t, C.c_float, _i32p, _f32p]
    lib.orc_sample_cloud.argtypes = [_f32p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_float, _f64p, C.c_void_p]
    lib.orc_seanindex.restype = C.c_int
    lib.orc_seanindex.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.orc_sht.argtypes = [_f64p, C.c_int, _f64p, _f64p]
    lib.orc_wigner_column.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _f64p]
    lib.orc_so3_correlate.argtypes = [C.c_int, C.c_int, _f64p, _f64p, _f64p, _f64p, _f64p]
    lib.orc_spherical_correlation.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_int,
                                              C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_spherical_volume.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_int, _f64p]
    lib.orc_argmax.restype = C.c_uint64
    lib.orc_argmax.argtypes = [_f64p, C.c_uint64]
    lib.orc_bin_to_zyz.argtypes = [C.c_uint32, C.c_uint32, _f64p]
    lib.orc_zyz_to_quat.argtypes = [_f64p, _f64p]
    lib.orc_quat_to_xyz.argtypes = [_f64p, _f64p]
    lib.orc_rotation_xyz.argtypes = [C.c_float, C.c_float, C.c_float, _f32p]
    lib.orc_transform.argtypes = [_f32p, C.c_size_t, _f32p]
    lib.orc_edges.argtypes = [C.c_int, C.c_int, C.c_int, _f32p]
    lib.orc_voxel_index.argtypes = [_f32p, C.c_size_t, C.c_int, C.c_int, C.c_int, _u32p]
    lib.orc_discretize.argtypes = [_f32p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                   C.c_int, _f64p]
    lib.orc_spatial_correlation.argtypes = [C.c_int, C.c_int, _f64p, _f64p, C.c_int, C.c_int, _f64p]
    lib.orc_translation_from_index.restype = C.c_double
    lib.orc_translation_from_index.argtypes = [C.c_double, C.c_uint32, C.c_int, C.c_int]
    lib.orc_register_pair.argtypes = [_f32p, C.c_size_t, C.c_void_p, _f32p, C.c_size_t, C.c_void_p,
                                      C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                      C.POINTER(Pose), C.c_void_p, C.c_void_p]
    lib.orc_register_pair_k.argtypes = [_f32p, C.c_size_t, C.c_void_p, _f32p, C.c_size_t, C.c_void_p,
                                        C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint32, C.c_uint32,
                                        C.POINTER(Pose), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_so3_correlate_slices.argtypes = [C.c_int, C.c_int, _f64p, _f64p, _f64p, _f64p, C.c_int, C.c_void_p,
                                             _f64p]
    lib.orc_mix_signal.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
    lib.orc_register_pair_mode.argtypes = [_f32p, C.c_size_t, C.c_void_p, _f32p, C.c_size_t, C.c_void_p,
                                           C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint32, C.c_uint32,
                                           C.c_int, C.POINTER(Pose), C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p]
    lib.orc_spherical_correlation_lowpass.argtypes = [C.c_int, C.c_int, _f64p, _f64p, C.c_uint32, C.c_uint32,
                                                      _f64p]
    lib.orc_spatial_correlation_lowpass.argtypes = [C.c_int, _f64p, _f64p, C.c_uint32, C.c_uint32, _f64p]
    lib.orc_peak_window.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]
    lib.orc_bingham_peak.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
    lib.orc_spatial_correlation_padded.restype = C.c_uint32
    lib.orc_spatial_correlation_padded.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_int, C.c_int,
                                                   C.c_uint32, C.c_uint32, _f64p, _f64p, _f64p]
    lib.orc_voxel_grid.restype = C.c_int64
    lib.orc_voxel_grid.argtypes = [_f32p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_float, C.c_float, C.c_float,
                                   C.c_uint32, _f32p, C.c_void_p, C.c_void_p]
    lib.orc_zscore_peaks.restype = C.c_uint64
    lib.orc_zscore_peaks.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_uint32, C.c_double, C.c_double,
                                     C.c_double, C.c_void_p, C.c_uint64]
    lib.orc_gaussian_peak.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int,
                                      C.c_void_p, C.c_void_p]
    lib.orc_num_threads.restype = C.c_int


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        _LIB = C.CDLL(path)
        _declare(_LIB)
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libphaser_ref.so"))


def ref_lib():
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libphaser_ref.so")
        _REF = C.CDLL(path)
        _declare(_REF)
        _REF.ref_sht.argtypes = [C.c_int, _f64p, _f64p, _f64p]
        _REF.ref_spherical_correlation.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                                   C.c_void_p, C.c_void_p]
        _REF.ref_spatial_correlation.argtypes = [C.c_int, C.c_int, _f64p, _f64p, C.c_int, _f64p]
        _REF.ref_register_pair.restype = C.c_int
        _REF.ref_register_pair.argtypes = [_f32p, C.c_size_t, C.c_void_p, _f32p, C.c_size_t,
                                           C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_float, C.c_int, C.POINTER(C.c_uint32),
                                           C.POINTER(C.c_uint32), _f64p]
        _REF.ref_register_pair_mode.restype = C.c_int
        _REF.ref_register_pair_mode.argtypes = [_f32p, C.c_size_t, C.c_void_p, _f32p, C.c_size_t,
                                                C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.c_float, C.c_int, C.c_int, C.POINTER(C.c_uint32),
                                                C.POINTER(C.c_uint32), _f64p]
    return _REF


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- wrappers


def pyramid_struct(n, levels, div=4.0):
    lb = np.zeros(levels, np.uint32)
    ub = np.zeros(levels, np.uint32)
    co = np.zeros(levels, np.uint32)
    lib().orc_pyramid_struct(n, levels, div, lb, ub, co)
    return lb, ub, co


def fuse_literal(channels: np.ndarray, levels=5, div=4.0) -> np.ndarray:
    """channels: complex128 [C, n] (FFT-shifted) -> fused complex128 [n]."""
    ch = np.ascontiguousarray(channels.astype(np.complex128)).view(np.float64).reshape(-1)
    n = channels.shape[1]
    out = np.zeros(2 * n, np.float64)
    lib().orc_fuse_channels_literal(ch, channels.shape[0], n, levels, div, out)
    return out.view(np.complex128)


def fusion_rule(p, n, levels=5, div=4.0):
    return lib().orc_fusion_rule(p, n, levels, div)


def fftshift(x: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(x.astype(np.complex128)).view(np.float64).copy()
    lib().orc_fftshift(a, x.size)
    return a.view(np.complex128)


def ifftshift(x: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(x.astype(np.complex128)).view(np.float64).copy()
    lib().orc_ifftshift(a, x.size)
    return a.view(np.complex128)


def sub2ind(i, j, k, rows, cols):
    return lib().orc_sub2ind(i, j, k, rows, cols)


def ind2sub(lin, rows, cols):
    o = np.zeros(3, np.uint32)
    lib().orc_ind2sub(lin, rows, cols, o)
    return o


def dh_grid(bw):
    g = np.zeros(4 * bw * bw * 3, np.float32)
    lib().orc_dh_grid(bw, g)
    return g.reshape(-1, 3)


def dh_weights(bw):
    w = np.zeros(2 * bw, np.float64)
    lib().orc_dh_weights(bw, w)
    return w


def project(xyzi: np.ndarray):
    pts = np.ascontiguousarray(xyzi, np.float32)
    P = pts.shape[0]
    out = np.zeros(3 * P, np.float32)
    rng = np.zeros(P, np.float64)
    lib().orc_project(pts.reshape(-1), pts.shape[1], P, out, rng)
    return out.reshape(P, 3), rng


def nn(queries: np.ndarray, points: np.ndarray, max_sq=np.float32(np.inf)):
    q = np.ascontiguousarray(queries, np.float32).reshape(-1)
    p = np.ascontiguousarray(points, np.float32).reshape(-1)
    nq = q.size // 3
    idx = np.zeros(nq, np.int32)
    d2 = np.zeros(nq, np.float32)
    lib().orc_nn(q, nq, p, p.size // 3, float(max_sq), idx, d2)
    return idx, d2


def sample_cloud(xyzi, refl, amb, bw, max_sq=1e6):
    pts = np.ascontiguousarray(xyzi, np.float32)
    out = np.zeros(4 * 4 * bw * bw, np.float64)
    nnidx = np.zeros(4 * bw * bw, np.int32)
    r = None if refl is None else np.ascontiguousarray(refl, np.float32)
    a = None if amb is None else np.ascontiguousarray(amb, np.float32)
    lib().orc_sample_cloud(pts.reshape(-1), pts.shape[0], _ptr(r), _ptr(a), bw, max_sq, out,
                           nnidx.ctypes.data_as(C.c_void_p))
    return out.reshape(4, 4 * bw * bw), nnidx


def sht(sig: np.ndarray, bw: int) -> np.ndarray:
    s = np.ascontiguousarray(sig, np.float64).reshape(-1)
    re = np.zeros(bw * bw)
    im = np.zeros(bw * bw)
    lib().orc_sht(s, bw, re, im)
    return re + 1j * im


def seanindex(m, l, bw):
    return lib().orc_seanindex(m, l, bw)


def wigner_column(m1, m2, bw, beta):
    j0 = max(abs(m1), abs(m2))
    out = np.zeros(max(bw - j0, 1))
    lib().orc_wigner_column(m1, m2, bw, beta, out)
    return out[: max(bw - j0, 0)]


def spherical_correlation(f, g, bw, bw_out=None, levels=5, return_fused=False):
    """f, g: [C, 4 bw^2] float64.  Returns corr (2 bw_out)^3 = |z|^2."""
    bw_out = bw if bw_out is None else bw_out
    f = np.ascontiguousarray(f, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    Cn = f.shape[0]
    n = 2 * bw_out
    corr = np.zeros(n ** 3)
    ff = np.zeros(2 * bw * bw)
    gg = np.zeros(2 * bw * bw)
    lib().orc_spherical_correlation(bw, bw_out, Cn, f.reshape(-1), g.reshape(-1), levels, _ptr(corr),
                                    ff.ctypes.data_as(C.c_void_p), gg.ctypes.data_as(C.c_void_p))
    if return_fused:
        return corr, ff.view(np.complex128), gg.view(np.complex128)
    return corr


def spherical_correlation_slices(f, g, bw, ks, bw_out=None, levels=5):
    """|z|^2 of the Laplace-fused correlation at beta indices ks only:
    [len(ks)][2 bw_out (alpha)][2 bw_out (gamma)], FP64."""
    bw_out = bw if bw_out is None else bw_out
    f = np.ascontiguousarray(f, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    nc = bw * bw
    ff = np.zeros(2 * nc)
    gg = np.zeros(2 * nc)
    # the fused spectra alone (no correlation volume)
    lib().orc_spherical_correlation(bw, bw_out, f.shape[0], f.reshape(-1), g.reshape(-1), levels, None,
                                    ff.ctypes.data_as(C.c_void_p), gg.ctypes.data_as(C.c_void_p))
    ks = np.ascontiguousarray(ks, np.int32)
    n = 2 * bw_out
    out = np.zeros(len(ks) * n * n)
    lib().orc_so3_correlate_slices(bw, bw_out, np.ascontiguousarray(ff[0::2]), np.ascontiguousarray(ff[1::2]),
                                   np.ascontiguousarray(gg[0::2]), np.ascontiguousarray(gg[1::2]), len(ks),
                                   ks.ctypes.data, out)
    return out.reshape(len(ks), n, n)


def spherical_volume(f, g, bw, bw_out=None, levels=5):
    bw_out = bw if bw_out is None else bw_out
    f = np.ascontiguousarray(f, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    n = 2 * bw_out
    vol = np.zeros(2 * n ** 3)
    lib().orc_spherical_volume(bw, bw_out, f.shape[0], f.reshape(-1), g.reshape(-1), levels, vol)
    return vol.view(np.complex128)


def argmax(v):
    v = np.ascontiguousarray(v, np.float64)
    return int(lib().orc_argmax(v, v.size))


def bin_to_pose(bin_, bw):
    zyz = np.zeros(3)
    q = np.zeros(4)
    xyz = np.zeros(3)
    lib().orc_bin_to_zyz(bin_, bw, zyz)
    lib().orc_zyz_to_quat(zyz, q)
    lib().orc_quat_to_xyz(q, xyz)
    return zyz, q, xyz


def rotation_xyz(a, b, c):
    T = np.zeros(12, np.float32)
    lib().orc_rotation_xyz(np.float32(a), np.float32(b), np.float32(c), T)
    return T.reshape(3, 4)


def transform(xyzi, T):
    pts = np.ascontiguousarray(xyzi, np.float32).copy()
    lib().orc_transform(pts.reshape(-1), pts.shape[0], np.ascontiguousarray(T, np.float32).reshape(-1))
    return pts


def edges(N, lo, hi):
    e = np.zeros(N, np.float32)
    lib().orc_edges(N, lo, hi, e)
    return e


def voxel_index(xyzi, N, lo, hi):
    pts = np.ascontiguousarray(xyzi, np.float32)
    out = np.zeros(pts.shape[0], np.uint32)
    lib().orc_voxel_index(pts.reshape(-1), pts.shape[0], N, lo, hi, out)
    return out


def discretize(xyzi, refl, amb, N, lo, hi):
    pts = np.ascontiguousarray(xyzi, np.float32)
    out = np.zeros(4 * N ** 3)
    r = None if refl is None else np.ascontiguousarray(refl, np.float32)
    a = None if amb is None else np.ascontiguousarray(amb, np.float32)
    lib().orc_discretize(pts.reshape(-1), pts.shape[0], _ptr(r), _ptr(a), N, lo, hi, out)
    return out.reshape(4, N ** 3)


def spatial_correlation(f, g, N, laplace=True, levels=5):
    f = np.ascontiguousarray(f, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    Cn = f.shape[0] if f.ndim == 2 else 1
    out = np.zeros(N ** 3)
    lib().orc_spatial_correlation(N, Cn, f.reshape(-1), g.reshape(-1), 1 if laplace else 0, levels, out)
    return out


def spherical_correlation_lowpass(f0, g0, bw, lower, upper, bw_out=None):
    """Low-pass spherical correlation of channel 0 (|z|^2, (2 bw_out)^3)."""
    bw_out = bw if bw_out is None else bw_out
    corr = np.zeros((2 * bw_out) ** 3)
    lib().orc_spherical_correlation_lowpass(bw, bw_out, np.ascontiguousarray(f0, np.float64).reshape(-1),
                                            np.ascontiguousarray(g0, np.float64).reshape(-1), int(lower), int(upper),
                                            corr)
    return corr


def spatial_correlation_lowpass(f1, g1, N, lower, upper):
    """Low-pass spatial correlation of channel 1 grids (N^3 each)."""
    out = np.zeros(N ** 3)
    lib().orc_spatial_correlation_lowpass(N, np.ascontiguousarray(f1, np.float64).reshape(-1),
                                          np.ascontiguousarray(g1, np.float64).reshape(-1), int(lower), int(upper),
                                          out)
    return out


def translation_from_index(idx, n, lo, hi):
    return lib().orc_translation_from_index(float(idx), n, lo, hi)


def register_pair(tgt, tgt_refl, src, src_refl, bw, N, lo, hi, max_sq=1e6, want_volumes=False, rot_k=0,
                  trans_k=0, want_stats=False, sph_mode=0):
    """Full registration; with rot_k / trans_k > 0 the Bingham mode and the
    Gaussian mean of the peak neighbourhoods give the pose.  want_stats adds
    (omega[4], cov[3x3]) to the returned tuple.  sph_mode 1: SphRegistration's
    single 0.6 intensity + 0.4 range signal instead of the Laplace fusion."""
    tgt = np.ascontiguousarray(tgt, np.float32)
    src = np.ascontiguousarray(src, np.float32)
    tr = None if tgt_refl is None else np.ascontiguousarray(tgt_refl, np.float32)
    sr = None if src_refl is None else np.ascontiguousarray(src_refl, np.float32)
    pose = Pose()
    rc = np.zeros((2 * bw) ** 3) if want_volumes else None
    tc = np.zeros(N ** 3) if want_volumes else None
    omega, cov = np.zeros(4), np.zeros(9)
    lib().orc_register_pair_mode(tgt.reshape(-1), tgt.shape[0], _ptr(tr), src.reshape(-1), src.shape[0],
                                 _ptr(sr), bw, N, lo, hi, max_sq, int(rot_k), int(trans_k), int(sph_mode),
                                 C.byref(pose), _ptr(rc), _ptr(tc), omega.ctypes.data, cov.ctypes.data)
    out = (pose,)
    if want_volumes:
        out += (rc, tc)
    if want_stats:
        out += (omega, cov.reshape(3, 3))
    return out if len(out) > 1 else pose


def peak_window(index, n, k):
    f, c = C.c_uint32(), C.c_uint32()
    lib().orc_peak_window(int(index), int(n), int(k), C.byref(f), C.byref(c))
    return f.value, c.value


def zscore_peaks(corr, lag_percentile=0.05, lag_max=20, threshold=4.33, influence=0.05, filter_threshold=0.405):
    """ZScorePeakExtraction::extractPeaks (z-score-peak-extraction.cc:42-112): ascending signal indices."""
    v = np.ascontiguousarray(corr, np.float64)
    out = np.zeros(max(len(v), 1), np.uint32)
    k = lib().orc_zscore_peaks(v.ctypes.data, len(v), float(lag_percentile), int(lag_max), float(threshold),
                               float(influence), float(filter_threshold), out.ctypes.data, len(out))
    return out[:k].copy()


def bingham_peak(values, first, bw):
    v = np.ascontiguousarray(values, np.float64)
    mode, omega, xyz = np.zeros(4), np.zeros(4), np.zeros(3)
    if lib().orc_bingham_peak(v.ctypes.data, int(first), len(v), int(bw), mode.ctypes.data, omega.ctypes.data,
                              xyz.ctypes.data) != 0:
        raise ValueError("no positive weight")
    return mode, omega, xyz


def gaussian_peak(values, first, N, lo, hi):
    v = np.ascontiguousarray(values, np.float64)
    mean, cov = np.zeros(3), np.zeros(9)
    if lib().orc_gaussian_peak(v.ctypes.data, int(first), len(v), int(N), int(lo), int(hi), mean.ctypes.data,
                               cov.ctypes.data) != 0:
        raise ValueError("no positive weight sum")
    return mean, cov.reshape(3, 3)


# ------------------------------------------------------ reference (SOFT) side


def ref_sht(sig, bw):
    s = np.ascontiguousarray(sig, np.float64).reshape(-1)
    re = np.zeros(bw * bw)
    im = np.zeros(bw * bw)
    ref_lib().ref_sht(bw, s, re, im)
    return re + 1j * im


def ref_spherical_correlation(f, g, bw, bw_out=None, volume=False):
    bw_out = bw if bw_out is None else bw_out
    f = np.ascontiguousarray(f, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    n = 2 * bw_out
    corr = np.zeros(n ** 3)
    vol = np.zeros(2 * n ** 3) if volume else None
    ref_lib().ref_spherical_correlation(bw, bw_out, f.shape[0], f.reshape(-1), g.reshape(-1),
                                        _ptr(corr), _ptr(vol))
    if volume:
        return corr, vol.view(np.complex128)
    return corr


def ref_spatial_correlation(f, g, N, laplace=True):
    f = np.ascontiguousarray(f, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    Cn = f.shape[0] if f.ndim == 2 else 1
    out = np.zeros(N ** 3)
    ref_lib().ref_spatial_correlation(N, Cn, f.reshape(-1), g.reshape(-1), 1 if laplace else 0, out)
    return out


def ref_register_pair(tgt, tgt_refl, src, src_refl, bw, N, lo, hi, max_sq=1e6, threads=None, sph_mode=0):
    tgt = np.ascontiguousarray(tgt, np.float32)
    src = np.ascontiguousarray(src, np.float32)
    tr = None if tgt_refl is None else np.ascontiguousarray(tgt_refl, np.float32)
    sr = None if src_refl is None else np.ascontiguousarray(src_refl, np.float32)
    threads = threads or os.cpu_count() or 1
    rb = C.c_uint32()
    vx = C.c_uint32()
    pose6 = np.zeros(6)
    ref_lib().ref_register_pair_mode(tgt.reshape(-1), tgt.shape[0], _ptr(tr), src.reshape(-1),
                                     src.shape[0], _ptr(sr), bw, N, lo, hi, max_sq, threads, int(sph_mode),
                                     C.byref(rb), C.byref(vx), pose6)
    return rb.value, vx.value, pose6


def voxel_grid(xyzi, leaf=(0.25, 0.25, 0.25), min_points=0, refl=None, amb=None):
    """pcl::VoxelGrid<PointXYZI> restated in float (orc_voxel_grid): leaf
    centroids (xyzi, refl, amb) in increasing leaf order; None where the
    grid leaves PCL's defined int range."""
    x = np.ascontiguousarray(xyzi, np.float32).reshape(-1, 4)
    n = x.shape[0]
    r = None if refl is None else np.ascontiguousarray(refl, np.float32)
    a = None if amb is None else np.ascontiguousarray(amb, np.float32)
    out = np.zeros((max(n, 1), 4), np.float32)
    orf = np.zeros(max(n, 1), np.float32) if r is not None else None
    oam = np.zeros(max(n, 1), np.float32) if a is not None else None
    lf = np.broadcast_to(np.asarray(leaf, np.float32), (3,))
    k = lib().orc_voxel_grid(x, _ptr(r), _ptr(a), n, float(lf[0]), float(lf[1]), float(lf[2]), int(min_points),
                             out, _ptr(orf), _ptr(oam))
    if k < 0:
        return None
    return out[:k], None if orf is None else orf[:k], None if oam is None else oam[:k]


def new_padded_state(N):
    """Fresh F_ / G_ buffers of a padded SpatialCorrelation (zero at construction)."""
    return np.zeros(2 * N ** 3), np.zeros(2 * N ** 3)


def spatial_correlation_padded(f, g, N, pad, mode=1, levels=5, lower=0, upper=None, state=None):
    """Literal restatement of the zero-padded spatial correlation
    (orc_spatial_correlation_padded).  f, g: [C][N^3]; mode 0 plain, 1
    Laplace, 2 low-pass.  state: (F_, G_) carried between calls (modified in
    place; fresh when None).  Returns (volume of (N + 2 pad)^3, the
    reference's correlation length)."""
    f = np.ascontiguousarray(f, np.float64).reshape(-1, N ** 3)
    g = np.ascontiguousarray(g, np.float64).reshape(-1, N ** 3)
    if state is None:
        state = new_padded_state(N)
    M = N + 2 * pad
    out = np.zeros(M ** 3)
    up = N if upper is None else int(upper)
    size = lib().orc_spatial_correlation_padded(N, pad, f.shape[0], f.ravel(), g.ravel(), mode, levels, int(lower),
                                                up, state[0], state[1], out)
    return out, int(size)
