"""Nonlinear equations in Robert variables (sph_swe_params.nonlinear = 2; no
reference counterpart) against the oracle's restatement written with the
reference's Robert operators (SPHOperators.hpp:129-210), and the T1023
configuration: balanced sech^2 jet plus a 120 m bump, dt = 15 s."""
import numpy as np
import pytest
import torch

from sph_swe_b200 import scenarios as S
from tests.helpers import random_spec, rel_l2

pytestmark = pytest.mark.gpu

A, G, OM = 6.371e6, 9.80616, 7.292e-5


def _jet_state(grid, bump_amp=120.0):
    h, u, v = S.sech2_jet(grid, radius=A, bump_amp=bump_amp)
    c = np.cos(np.asarray(grid.lat))[None, :]
    return h, u * c, v * c


def _spec(g, grids):
    return np.stack([g.spat_to_SH(x) for x in grids])


@pytest.mark.parametrize("L,visc", [(31, 0.0), (63, 1e5)])
def test_robert_nonlinear_tendency_matches_oracle(gpu, oracle_mod, L, visc):
    from sph_swe_b200.sph import Sph

    s, g = Sph(L), oracle_mod.Grid(L)
    st0 = _spec(g, _jet_state(g))
    st0[1:] += random_spec(L, 2, seed=L, decay=3.0) * 2.0
    p = Sph.swe_params(radius=A, dt=15.0, viscosity=visc, nonlinear=2, robert=1)
    tend = s.swe_tendency(p, torch.from_numpy(st0).cuda()).cpu().numpy()
    ref = g.swe_tendency((A, G, OM, 1e4, visc, 15.0), *st0, nonlinear=2, robert=1)
    for q in range(3):
        assert rel_l2(tend[q], ref[q]) < 1e-10, q


def test_robert_nonlinear_rk4_matches_oracle(gpu, oracle_mod):
    from sph_swe_b200.sph import Sph

    L, n = 63, 40
    s, g = Sph(L), oracle_mod.Grid(L)
    st0 = _spec(g, _jet_state(g))
    p = Sph.swe_params(radius=A, dt=120.0, nonlinear=2, robert=1)
    st = torch.from_numpy(st0.copy()).cuda()
    s.swe_rk4(p, st, n)
    out = st.cpu().numpy()
    rh, ru, rv, rc = g.swe_run((A, G, OM, 1e4, 0.0, 120.0), *st0, n, nonlinear=2, robert=1)
    assert rc == 0
    for q, ref in enumerate((rh, ru, rv)):
        assert rel_l2(out[q], ref) < 1e-10, q


@pytest.mark.parametrize("prec", [0, 1])
def test_t1023_round_trip(gpu, prec):
    """T1023 on 1536 x 3072: analysis(synthesis(x)) = x (size-independent property)."""
    from sph_swe_b200.sph import Sph

    s = Sph(1023, precision=prec)
    assert (s.nlat, s.nphi) == (1536, 3072)
    x = torch.from_numpy(random_spec(1023, 3, seed=9)).cuda()
    back = s.spat_to_SH(s.SH_to_spat(x)).cpu().numpy()
    tol = 1e-11 if prec == 0 else 1e-6
    for b in range(3):
        assert rel_l2(back[b], x[b].cpu().numpy()) < tol


def test_t1023_jet_mass_and_mixed_form(gpu):
    """The T1023 configuration for 10 steps: finite, mass (the Y_00 coefficient
    of h) drifts by < 1e-12 relative, and the mixed form stays within 1e-6 of
    the FP64 form in h."""
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    out = {}
    for prec in (capi.SPH_PREC_FP64, capi.SPH_PREC_MIXED):
        s = Sph(1023, precision=prec)
        if prec == capi.SPH_PREC_FP64:
            grids = [torch.from_numpy(x).cuda() for x in _jet_state(s)]
            st0 = torch.stack([s.spat_to_SH(x) for x in grids])
        p = Sph.swe_params(radius=A, dt=15.0, nonlinear=2, robert=1)
        st = st0.clone()
        s.swe_rk4(p, st, 10)
        capi.check(capi.lib().sph_sync(s.h, None))
        out[prec] = st.cpu().numpy()
        s.close()
    h0 = st0[0, 0].item()
    f64 = out[capi.SPH_PREC_FP64]
    assert np.all(np.isfinite(f64))
    assert abs(f64[0, 0] - h0) / abs(h0) < 1e-12
    assert rel_l2(out[capi.SPH_PREC_MIXED][0], f64[0]) < 1e-6
