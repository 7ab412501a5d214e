"""B200 (sm_100a) implementation of PHASER's correspondence-free registration
hot path.

The CUDA kernels live behind the C ABI of include/phaser_gpu.h
(phaser_b200/_lib/libphaser_gpu.so, built by ``python -m phaser_b200.build``).
``phaser_b200.native`` binds it with ctypes; ``phaser_b200.core`` mirrors the
reference's classes (SphericalCorrelation[Laplace], SpatialCorrelation[Laplace],
PhaseAligner, SphericalSampler, SphOptRegistration) on top of it.
"""
__all__ = ["native", "scene"]
