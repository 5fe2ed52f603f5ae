"""CPU-side checks of the C ABI library: it builds for sm_100a, loads, and
exports every entry point declared in include/sph_gpu.h (no compute calls)."""
import os
import re

import numpy as np

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "sph_gpu.h")).read()
    return sorted(set(re.findall(r"^int\s+(sph_\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    from sph_swe_b200 import build, capi

    build.build()
    return capi.lib()


def test_header_and_binding_agree():
    from sph_swe_b200 import capi

    assert _declared() == sorted(capi.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in _declared():
        assert hasattr(lib, name), name


def test_build_targets_sm100a_only():
    from sph_swe_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_error_reporting_without_gpu(lib):
    import ctypes

    from sph_swe_b200 import capi

    h = ctypes.c_void_p()
    rc = lib.sph_create(8, 9, 0, 0, 0, ctypes.byref(h))
    assert rc == capi.SPH_ERR_ARG
    assert "lmax == mmax" in capi.last_error()
    assert lib.sph_info(None, None, None, None, None, None) == capi.SPH_ERR_ARG
    e = ctypes.c_void_p()
    assert lib.sph_ensemble_create(0, None, None, None, None, None, ctypes.byref(e)) == capi.SPH_ERR_ARG
    assert "sph_ensemble_create" in capi.last_error()
    assert lib.sph_ensemble_step(None, 1, None) == capi.SPH_ERR_ARG
    assert lib.sph_ensemble_launches(None) == 0
    assert lib.sph_ensemble_destroy(None) == capi.SPH_OK
    # argument checks of the other entry points come before any device call
    assert lib.sph_spec_copy_modes(None, None, None, None, 1, None) == capi.SPH_ERR_ARG
    assert "sph_spec_copy_modes" in capi.last_error()
    assert lib.sph_SH_to_spat_noalloc(None, None, None, 1, None) == capi.SPH_ERR_ARG
    assert "sph_SH_to_spat_noalloc" in capi.last_error()
    r = ctypes.c_void_p()
    assert lib.sph_rexi_create(None, None, None, 0, None, ctypes.byref(r)) == capi.SPH_ERR_ARG
    assert lib.sph_rexi_step(None, None, 1, None) == capi.SPH_ERR_ARG
    assert lib.sph_autotune(None, 8, None, 0, None) == capi.SPH_ERR_ARG
    assert lib.sph_tune_load(None, b"{}") == capi.SPH_ERR_ARG
    assert lib.sph_tune_clear(None) == capi.SPH_ERR_ARG


@pytest.mark.parametrize("M,half", [(64, False), (256, False), (256, True), (32, True)])
def test_rexi_coefficients_match_oracle(oracle_mod, M, half):
    """Host-side coefficient generation of the library against the oracle's
    REXI::setup restatement, and the approximation of e^{ix} it is built for."""
    from sph_swe_b200.sph import rexi_coefficients

    a, br, bi = rexi_coefficients(0.2, M, half)
    ra, rbr, rbi = oracle_mod.rexi_coeffs(0.2, M, half=half)
    assert len(a) == len(ra) == (M + 12 if half else 2 * (M + 11) + 1)
    for x, y in ((a, ra), (br, rbr), (bi, rbi)):
        assert np.max(np.abs(x - y)) <= 1e-14 * np.max(np.abs(y))
    # the full pole set approximates e^{ix} on |x| <= M h / 2 (both parts)
    xs = np.linspace(-0.5 * M * 0.2, 0.5 * M * 0.2, 101)
    if not half:
        approx = np.array([np.sum((br / (1j * x + a)).real) + 1j * np.sum((bi / (1j * x + a)).real) for x in xs])
        assert np.max(np.abs(approx - np.exp(1j * xs))) < 1e-7


def test_rexi_coefficients_reject_bad_arguments():
    import ctypes

    from sph_swe_b200 import capi

    n = ctypes.c_int()
    assert capi.lib().sph_rexi_coefficients(0.0, 10, 0, 0, None, None, None, ctypes.byref(n)) == capi.SPH_ERR_ARG
    buf = (ctypes.c_double * 4)()
    assert capi.lib().sph_rexi_coefficients(0.2, 10, 0, 2, buf, buf, buf, ctypes.byref(n)) == capi.SPH_ERR_ARG
    assert "capacity" in capi.last_error()
