"""ctypes binding of libsphgpu.so (the C ABI declared in include/sph_gpu.h).

The library is the product; this module only forwards plain pointers and
sizes.  It fails loudly when the library is missing: there is no CPU
fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsphgpu.so")

SPH_OK, SPH_ERR_ARG, SPH_ERR_CUDA, SPH_ERR_SINGULAR, SPH_ERR_NAN, SPH_ERR_TIMEOUT, SPH_ERR_NOMEM = range(7)
SPH_PREC_FP64, SPH_PREC_MIXED = 0, 1
SPH_TUNE_INT8, SPH_TUNE_TF32, SPH_TUNE_FP64 = 1, 2, 4
OPS = dict(diff_lon=0, d1mu2=1, mu=2, mu2=3, laplace=4, helmholtz=5, scale=6, axpy=7)

# every symbol declared in include/sph_gpu.h
EXPORTS = (
    "sph_create", "sph_destroy", "sph_info", "sph_grid",
    "sph_spat_to_SH", "sph_SH_to_spat", "sph_SH_to_spat_noalloc", "sph_cplx_spat_to_SH", "sph_cplx_SH_to_spat",
    "sph_vec_SH_to_spat", "sph_vec_spat_to_SH", "sph_legendre_synthesis", "sph_legendre_analysis", "sph_spec_op",
    "sph_spec_copy_modes",
    "sph_swe_tendency", "sph_swe_rk4", "sph_swe_rk4_batched", "sph_swe_rk4_launches",
    "sph_ensemble_create", "sph_ensemble_step", "sph_ensemble_launches", "sph_ensemble_destroy",
    "sph_autotune", "sph_autotune_ex", "sph_tune_load", "sph_tune_clear",
    "sph_spat_op", "sph_rexi_coefficients", "sph_rexi_create", "sph_rexi_destroy", "sph_rexi_step", "sph_sync", "sph_wait_selftest",
    "sph_last_error",
)


class SphError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[sph status {code}] {msg}")
        self.code = code


class SWEParams(ctypes.Structure):
    _fields_ = [("radius", ctypes.c_double), ("gravity", ctypes.c_double), ("omega", ctypes.c_double),
                ("h0", ctypes.c_double), ("viscosity", ctypes.c_double), ("dt", ctypes.c_double),
                ("nonlinear", ctypes.c_int), ("robert", ctypes.c_int)]


class RexiParams(ctypes.Structure):
    _fields_ = [("radius", ctypes.c_double), ("gravity", ctypes.c_double), ("omega", ctypes.c_double),
                ("h0", ctypes.c_double), ("viscosity", ctypes.c_double), ("tau", ctypes.c_double),
                ("robert", ctypes.c_int), ("coriolis", ctypes.c_int), ("fix_z5robert", ctypes.c_int),
                ("precision", ctypes.c_int), ("factor_each_step", ctypes.c_int)]


_lib = None


def lib():
    """Load libsphgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m sph_swe_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, ll, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.sph_create.argtypes = [i, i, i, i, i, ctypes.POINTER(vp)]
        L.sph_destroy.argtypes = [vp]
        L.sph_info.argtypes = [vp, ip, ip, ip, ip, ip]
        L.sph_grid.argtypes = [vp, dp, dp, dp, dp]
        for n in ("sph_spat_to_SH", "sph_SH_to_spat", "sph_cplx_spat_to_SH", "sph_cplx_SH_to_spat"):
            getattr(L, n).argtypes = [vp, vp, vp, i, ll, ll, vp]
        for n in ("sph_vec_SH_to_spat", "sph_vec_spat_to_SH"):
            getattr(L, n).argtypes = [vp, vp, vp, vp, vp, i, i, vp]
        L.sph_spec_op.argtypes = [vp, i, vp, vp, d, d, d, d, i, i, vp]
        L.sph_spec_copy_modes.argtypes = [vp, vp, vp, vp, i, vp]
        L.sph_SH_to_spat_noalloc.argtypes = [vp, vp, vp, i, vp]
        L.sph_legendre_synthesis.argtypes = [vp, vp, vp, i, vp]
        L.sph_legendre_analysis.argtypes = [vp, vp, vp, i, vp]
        L.sph_swe_tendency.argtypes = [vp, ctypes.POINTER(SWEParams), vp, vp, vp]
        L.sph_swe_rk4.argtypes = [vp, ctypes.POINTER(SWEParams), vp, i, vp]
        L.sph_swe_rk4_batched.argtypes = [vp, ctypes.POINTER(SWEParams), dp, vp, i, i, vp]
        L.sph_ensemble_create.argtypes = [i, ctypes.POINTER(vp), ctypes.POINTER(SWEParams), ctypes.POINTER(vp), ip,
                                          ctypes.POINTER(dp), ctypes.POINTER(vp)]
        L.sph_swe_rk4_launches.argtypes = [vp]
        L.sph_autotune.argtypes = [vp, i, ctypes.c_char_p, i, vp]
        L.sph_autotune_ex.argtypes = [vp, i, i, ctypes.c_char_p, i, vp]
        L.sph_tune_load.argtypes = [vp, ctypes.c_char_p]
        L.sph_tune_clear.argtypes = [vp]
        L.sph_ensemble_step.argtypes = [vp, i, vp]
        L.sph_ensemble_launches.argtypes = [vp]
        L.sph_ensemble_destroy.argtypes = [vp]
        L.sph_rexi_create.argtypes = [vp, dp, dp, i, ctypes.POINTER(RexiParams), ctypes.POINTER(vp)]
        L.sph_rexi_destroy.argtypes = [vp]
        L.sph_rexi_coefficients.argtypes = [d, i, i, i, dp, dp, dp, ip]
        L.sph_rexi_step.argtypes = [vp, vp, i, vp]
        L.sph_sync.argtypes = [vp, vp]
        L.sph_wait_selftest.argtypes = [vp, d, vp]
        L.sph_spat_op.argtypes = [vp, i, vp, vp, vp, d, d, ll, vp]
        L.sph_last_error.argtypes = [ctypes.c_char_p, i]
        for n in EXPORTS:
            getattr(L, n).restype = ctypes.c_int
        _lib = L
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().sph_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != SPH_OK:
        raise SphError(rc, last_error())
