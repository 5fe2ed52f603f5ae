"""Failure paths of the CUDA path, made without a GPU fault.

* A zero pivot in a banded REXI solve must come back as SPH_ERR_SINGULAR, the
  error the reference's zgbsv call reports as INFO > 0
  (BandedMatrixSolver.hpp:429-434).  For |m| = L the velocity system of a pole
  is 1 x 1: alpha^2 + T^2 B(L, L) with T = 2 Omega and B the mu^2 identity
  coefficient (SPHIdentities.hpp), all formed on the host in IEEE double.  With
  tau = 1 s, a rotation rate and a purely imaginary pole alpha = i y chosen on
  the host so that fl(y^2) equals fl(T^2 B(L, L)) exactly, that pivot is
  exactly zero; the pole is injected among ordinary ones.
* A bounded device-side wait that runs out must come back as
  SPH_ERR_TIMEOUT through sph_sync, once, with the context still usable: the
  self-test waits, with the tensor-core kernels' own bounded wait, for a
  barrier that nothing completes.
"""
import ctypes
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _idR(k, m):
    n = k + 1.0
    if n < 0 or n < abs(m) or n * n - m * m < 0:
        return 0.0
    return math.sqrt((n * n - m * m) / (4.0 * n * n - 1.0))


def _idS(k, m):
    n = k - 1.0
    if n < 0 or n < abs(m) or n * n - m * m < 0:
        return 0.0
    return math.sqrt(((n + 1.0) * (n + 1.0) - m * m) / ((2.0 * n + 1.0) * (2.0 * n + 3.0)))


def singular_pole(L):
    """(omega, y): with tau = 1 the pole alpha = i y zeroes the velocity pivot
    of the |m| = L block exactly (the host arithmetic of the band builder)."""
    B = _idR(L - 1.0, L) * _idS(L, L) + _idS(L + 1.0, L) * _idR(L, L)
    for k in range(1000):
        omega = 7.292e-5 * (1.0 + k * 1e-6)
        T = 2.0 * omega
        d = (T * T) * B
        y0 = math.sqrt(d)
        for y in (math.nextafter(y0, 0.0), y0, math.nextafter(y0, 1.0)):
            if y * y == d:
                return omega, y
    raise AssertionError("no exact zero pivot found")


@pytest.mark.parametrize("precision,factor_each_step", [(0, 0), (0, 1), (1, 0)])
def test_rexi_zero_pivot_reports_singular(gpu, precision, factor_each_step):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Rexi, Sph, rexi_coefficients

    L = 31
    s = Sph(L)
    alpha, beta_re, _ = rexi_coefficients(0.2, 8, False)
    omega, y = singular_pole(L)
    alpha = alpha.copy()
    alpha[3] = 1j * y
    params = capi.RexiParams(6.371e6, 9.80616, omega, 1e4, 0.0, 1.0, 1, 1, 0, precision, factor_each_step)
    rx = Rexi(s, alpha, beta_re, params)
    state = torch.zeros(3, s.nlm, dtype=torch.complex128, device="cuda")
    state[0, 0] = 1.0
    with pytest.raises(capi.SphError) as e:
        rx.step(state, 1)
    assert e.value.code == capi.SPH_ERR_SINGULAR, str(e.value)
    # the same plan without the zero pole solves normally
    alpha_ok = rexi_coefficients(0.2, 8, False)[0]
    rx_ok = Rexi(s, alpha_ok, beta_re, params)
    state = torch.zeros(3, s.nlm, dtype=torch.complex128, device="cuda")
    state[0, 0] = 1.0
    rx_ok.step(state, 1)
    assert torch.isfinite(torch.view_as_real(state)).all()


def test_bounded_wait_times_out_and_reports_once(gpu):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph
    from tests.helpers import random_spec, rel_l2

    lib = capi.lib()
    s = Sph(31, precision=capi.SPH_PREC_MIXED)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.sph_sync(s.h, stream) == capi.SPH_OK
    assert lib.sph_wait_selftest(s.h, 0.05, stream) == capi.SPH_OK
    assert lib.sph_sync(s.h, stream) == capi.SPH_ERR_TIMEOUT
    assert "bounded wait" in capi.last_error()
    # reported once; the handle and the context still work
    assert lib.sph_sync(s.h, stream) == capi.SPH_OK
    spec = torch.from_numpy(random_spec(31, 2, seed=5)).cuda()
    grid = s.SH_to_spat(spec)
    back = s.spat_to_SH(grid)
    assert lib.sph_sync(s.h, stream) == capi.SPH_OK
    assert rel_l2(back.cpu().numpy(), spec.cpu().numpy()) < 1e-6
    # an FP64 handle has no tensor-core waits, and limits are checked
    s64 = Sph(31)
    assert lib.sph_wait_selftest(s64.h, 0.05, stream) == capi.SPH_ERR_ARG
    assert lib.sph_wait_selftest(s.h, 0.0, stream) == capi.SPH_ERR_ARG
    assert lib.sph_wait_selftest(s.h, 60.0, stream) == capi.SPH_ERR_ARG
