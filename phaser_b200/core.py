"""Python mirror of phaser_core's correlation, aligner and registration classes
on top of the C ABI (phaser_b200.native).  Names, arguments and return values
follow the reference:

  SphericalSampler            phaser_common/include/phaser/common/spherical-sampler.h:13-18
  SphericalCorrelation        phaser_core/include/phaser/backend/correlation/spherical-correlation.h:19-33
  SphericalCorrelationLaplace .../spherical-correlation-laplace.h
  SpatialCorrelation          .../spatial-correlation.h:15-23
  SpatialCorrelationLaplace   .../spatial-correlation-laplace.h
  SphericalCorrelationLowPass .../spherical-correlation-low-pass.h
  SpatialCorrelationLowPass   .../spatial-correlation-low-pass.h
  PhaseAligner                phaser_core/include/phaser/backend/alignment/phase-aligner.h:17-26
  SphOptRegistration          phaser_core/include/phaser/backend/registration/sph-opt-registration.h
  PlyHelper / PlyPointCloud   phaser_common/include/phaser/common/data/ply-helper.h, model/ply-point-cloud.h
  VoxelGridCmd                phaser_pre/include/phaser_pre/commands/voxel-grid-cmd.h

Everything runs on the GPU through libphaser_gpu.so; there is no CPU fallback.
"""
from __future__ import annotations

import numpy as np

from . import native
from .native import Context, default_params


class SphericalSampler:
    """SphericalSampler(bw).sampleUniformly(cloud) -> [4, 4 bw^2] channels
    {range, intensity, reflectivity, ambient} in [theta][phi] order."""

    def __init__(self, bandwidth: int, **params):
        self._bw = int(bandwidth)
        self._ctx = Context(spherical_bandwidth=self._bw, spatial_n_voxels=params.pop("spatial_n_voxels", 4),
                            **params)

    def sampleUniformly(self, xyzi, reflectivity=None, ambient=None):
        self._ctx.sample_s2(xyzi, reflectivity, ambient, side=0)
        vals, _ = self._ctx.samples(0)
        return vals

    def getInitializedBandwith(self) -> int:
        return self._bw


class SphericalCorrelation:
    """SphericalCorrelation(bw, zero_padding); correlateSampledSignals uses the
    first channel (spherical-correlation.cc:69-80)."""

    _fusion = native.PHGPU_FUSION_NONE

    def __init__(self, bw: int = 100, zero_padding: int = 0):
        self._bw = int(bw)
        self._bw_out = int(bw) + int(zero_padding)
        self._ctx = Context(spherical_bandwidth=self._bw, spherical_zero_padding=int(zero_padding),
                            spatial_n_voxels=4, spherical_fusion=self._fusion,
                            flags=native.PHGPU_FLAG_KEEP_VOLUMES)
        self._have = False

    def correlateSampledSignals(self, f, g):
        if len(f) != len(g) or len(f) == 0:
            raise ValueError("channel counts differ or are zero")
        n = len(f) if self._fusion == native.PHGPU_FUSION_LAPLACE else 1
        self._ctx.sph_correlate(list(f)[:n], list(g)[:n])
        self._have = True

    def getCorrelation(self) -> np.ndarray:
        if not self._have:
            return np.zeros(8 * self._bw_out ** 3)
        return self._ctx.sph_result(volume=True)[2]

    def getPeak(self):
        return self._ctx.sph_result()

    def getBandwidth(self) -> int:
        return self._bw_out

    def shutdown(self):
        self._ctx.close()


class SphericalCorrelationLaplace(SphericalCorrelation):
    _fusion = native.PHGPU_FUSION_LAPLACE

    def correlateSampledSignals(self, f, g):
        if len(f) < 2:
            raise ValueError("SphericalCorrelationLaplace needs at least 2 channels")
        super().correlateSampledSignals(f, g)


class SphericalCorrelationLowPass(SphericalCorrelation):
    """SphericalCorrelationLowPass(bw, zero_padding): channel 0, coefficients
    outside the FFT-shifted band [lower, upper) removed
    (spherical-correlation-low-pass.cc:14-59)."""
    _fusion = native.PHGPU_FUSION_LOW_PASS

    def __init__(self, bw: int = 100, zero_padding: int = 0, lower: int = 0, upper: int = 100000):
        self._bw = int(bw)
        self._bw_out = int(bw) + int(zero_padding)
        self._ctx = Context(spherical_bandwidth=self._bw, spherical_zero_padding=int(zero_padding),
                            spatial_n_voxels=4, spherical_fusion=self._fusion, spherical_low_pass_lower=int(lower),
                            spherical_low_pass_upper=int(upper), flags=native.PHGPU_FLAG_KEEP_VOLUMES)
        self._have = False


class SpatialCorrelation:
    """SpatialCorrelation(n_voxels, zero_padding).correlateSignals(f, g) ->
    correlation of getCorrelationSize() values (spatial-correlation.cc:163-206):
    N^3, or on (N + 2 zero_padding)^3 voxels with padding.  Like the
    reference object, a padded Laplace correlation depends on the previous
    call (see phgpu_spatial_result)."""

    _fusion = native.PHGPU_FUSION_NONE

    def __init__(self, n_voxels: int, zero_padding: int = 0):
        self._n = int(n_voxels)
        self._pad = int(zero_padding)
        self._ctx = Context(spherical_bandwidth=2, spatial_n_voxels=self._n, spatial_fusion=self._fusion,
                            spatial_zero_padding=self._pad, flags=native.PHGPU_FLAG_KEEP_VOLUMES)

    def correlateSignals(self, f, g) -> np.ndarray:
        self._ctx.spatial_correlate(list(f), list(g))
        return self._ctx.spatial_result(volume=True)[2]

    def getZeroPadding(self) -> int:
        return self._pad

    def getCorrelationSize(self) -> int:
        return int(self._ctx.lib.phgpu_spatial_correlation_size(self._ctx.h))


class SpatialCorrelationLaplace(SpatialCorrelation):
    _fusion = native.PHGPU_FUSION_LAPLACE


class SpatialCorrelationLowPass(SpatialCorrelation):
    """SpatialCorrelationLowPass(n_voxels, zero_padding[, lower, upper]):
    channel 1 of the signals, products kept inside the FFT-shifted cube
    [lower, upper]^3 (spatial-correlation-low-pass.cc:11-98)."""
    _fusion = native.PHGPU_FUSION_LOW_PASS

    def __init__(self, n_voxels: int, zero_padding: int = 0, lower: int = 0, upper: int = 100000):
        self._n = int(n_voxels)
        self._pad = int(zero_padding)
        self._lower, self._upper = int(lower), min(int(upper), self._n)
        self._ctx = Context(spherical_bandwidth=2, spatial_n_voxels=self._n, spatial_fusion=self._fusion,
                            spatial_low_pass_lower=float(self._lower), spatial_low_pass_upper=float(self._upper),
                            spatial_zero_padding=self._pad, flags=native.PHGPU_FLAG_KEEP_VOLUMES)

    def getLowerBound(self) -> int:
        return self._lower

    def getUpperBound(self) -> int:
        return self._upper

    def getNumberOfIndices(self) -> int:
        return max(0, self._upper - self._lower + 1) ** 3


class PhaseAligner:
    """PhaseAligner: voxelise both clouds and correlate (phase-aligner.cc:47-69)."""

    def __init__(self, n_voxels=100, lower=-50, upper=50, zero_padding=0):
        self._n, self._lo, self._hi = int(n_voxels), int(lower), int(upper)
        self._pad = int(zero_padding)
        self._ctx = Context(spherical_bandwidth=2, spatial_n_voxels=self._n, spatial_discretize_lower=self._lo,
                            spatial_discretize_upper=self._hi, spatial_zero_padding=self._pad,
                            flags=native.PHGPU_FLAG_KEEP_VOLUMES)

    def alignRegistered(self, cloud_prev, cloud_reg):
        """cloud_* = (xyzi, reflectivity) or (xyzi, reflectivity, ambient)."""
        self._ctx.voxelize(*cloud_prev, side=0)
        self._ctx.voxelize(*cloud_reg, side=1)
        self._ctx.spatial_correlate_voxelized()

    def getCorrelation(self) -> np.ndarray:
        return self._ctx.spatial_result(volume=True)[2]

    def getNumberOfVoxels(self) -> int:
        return self._n + 2 * self._pad

    def getLowerBound(self) -> int:
        return self._lo

    def getUpperBound(self) -> int:
        return self._hi


class SphOptRegistration:
    """registerPointCloud(prev = target, cur = source) -> pose dict
    (sph-opt-registration.cc:34-95)."""

    def __init__(self, bandwidth=75, n_voxels=100, lower=-50, upper=50, **params):
        self._ctx = Context(spherical_bandwidth=int(bandwidth), spatial_n_voxels=int(n_voxels),
                            spatial_discretize_lower=int(lower), spatial_discretize_upper=int(upper), **params)

    def registerPointCloud(self, cloud_prev, cloud_cur) -> dict:
        return self._ctx.register_pair(cloud_prev, cloud_cur).as_dict()


class PlyPointCloud:
    """The fields PlyHelper reads (phaser_common/src/common/data/
    ply-helper.cc:26-64), as float32 arrays (the reference keeps doubles and
    narrows x, y, z, intensity to float when building the cloud)."""

    def __init__(self, xyzi, reflectivity=None, ambient=None, range_=None):
        self.xyzi, self.reflectivity, self.ambient, self.range = xyzi, reflectivity, ambient, range_

    def getXYZPoints(self):
        return self.xyzi[:, :3]

    def getIntentsities(self):
        return self.xyzi[:, 3]

    def getReflectivities(self):
        return self.reflectivity

    def getAmbientPoints(self):
        return self.ambient

    def getRange(self):
        return self.range

    def cloud(self):
        """(xyzi, reflectivity, ambient): the tuple the registration takes."""
        return self.xyzi, self.reflectivity, self.ambient


class PlyHelper:
    """PlyHelper::readPlyFromFile; field names default to the reference's
    --phaser_ply_{intensity,reflectivity,ambient,range}_str flags."""

    def __init__(self, intensity="intensity", reflectivity="reflectivity", ambient="noise", range_="range"):
        self._names = [intensity, reflectivity, ambient, range_]

    def readPlyFromFile(self, filename, pinned=False) -> PlyPointCloud:
        d = native.ply_read(filename, self._names, pinned=pinned)
        return PlyPointCloud(d["xyzi"], d["reflectivity"], d["ambient"], d["range"])


class VoxelGridCmd:
    """VoxelGridCmd::execute (phaser_pre/src/commands/voxel-grid-cmd.cc:11-22):
    pcl::VoxelGrid with leaf --phaser_voxel_grid_leaf_size (0.25) on the GPU.
    execute(cloud) returns the filtered (xyzi, reflectivity, ambient) tuple
    (the reference filters its cloud in place)."""

    def __init__(self, leaf_size=0.25, max_points=1 << 20, device=0, min_points_per_voxel=0):
        self._leaf = float(leaf_size)
        self._min = int(min_points_per_voxel)
        self._vg = None
        self._cap = int(max_points)
        self._device = int(device)

    def execute(self, cloud):
        xyzi = cloud[0]
        refl = cloud[1] if len(cloud) > 1 else None
        amb = cloud[2] if len(cloud) > 2 else None
        n = int(xyzi.shape[0])
        if self._vg is None or n > self._vg.max_points:
            if self._vg is not None:
                self._vg.close()
            self._vg = native.VoxelGrid(max(self._cap, n), self._device)
        return self._vg.filter(xyzi, (self._leaf,) * 3, self._min, refl, amb)
