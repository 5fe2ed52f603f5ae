"""sph_swe_b200 — B200-native (sm_100a) spectral shallow-water hot path.

A from-scratch CUDA implementation of the spherical-harmonic transforms,
spectral operators, RK4 shallow-water tendency and REXI banded solves of
schreiberx/sph_swe behind a C ABI (``include/sph_gpu.h``, ``libsphgpu.so``).
This package holds the build recipe, the ctypes binding and a small
tensor-level host view used by the tests and the benchmark.
"""
from . import capi  # noqa: F401

__all__ = ["capi", "Sph"]


def __getattr__(name):
    if name == "Sph":
        from .sph import Sph

        return Sph
    raise AttributeError(name)
