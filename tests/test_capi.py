"""CPU-side checks of the C ABI library: it builds for sm_100a, loads, and
exports every entry point declared in include/sph_gpu.h (no compute calls)."""
import os
import re

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
