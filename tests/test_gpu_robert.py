"""The full nonlinear equations in vorticity-divergence form with Robert
velocities on the grid (sph_swe_params.nonlinear = 2; no reference
counterpart) against the oracle's numpy restatement (oracle/vortdiv.py), the
exact vector transforms against the same restatement, and the T1023
configuration: balanced sech^2 jet plus a 120 m bump, dt = 15 s."""
import numpy as np
import pytest
import torch

from sph_swe_b200 import scenarios as S
from tests.helpers import random_spec, rel_l2

pytestmark = pytest.mark.gpu

A, G, OM = 6.371e6, 9.80616, 7.292e-5


def _vd(grid):
    from oracle.vortdiv import VortDiv

    return VortDiv(grid)


def _jet_state(grid, vd, bump_amp=120.0):
    """[h, zeta, delta] spectra (physical) of the balanced jet plus a bump."""
    h, u, v = S.sech2_jet(grid, radius=A, bump_amp=bump_amp)
    c = np.cos(np.asarray(grid.lat))[None, :]
    z, d = vd.vec_analysis(u * c, v * c)
    return np.stack([grid.spat_to_SH(h), z / A, d / A])


@pytest.mark.parametrize("L", [31, 63])
def test_vector_transforms_match_oracle(gpu, oracle_mod, L):
    from sph_swe_b200.sph import Sph

    s, g = Sph(L), oracle_mod.Grid(L)
    vd = _vd(g)
    z, d = random_spec(L, 2, seed=L + 1)
    U, V = vd.vec_synthesis(z, d)
    u, v = s.vec_SH_to_spat(torch.from_numpy(z[None]).cuda(), torch.from_numpy(d[None]).cuda(), robert=True)
    assert rel_l2(u.cpu().numpy()[0], U) < 1e-12
    assert rel_l2(v.cpu().numpy()[0], V) < 1e-12
    zz, dd = vd.vec_analysis(U, V)
    z2, d2 = s.vec_spat_to_SH(torch.from_numpy(U[None].copy()).cuda(), torch.from_numpy(V[None].copy()).cuda(),
                              robert=True)
    assert rel_l2(z2.cpu().numpy()[0], zz) < 1e-12
    assert rel_l2(d2.cpu().numpy()[0], dd) < 1e-12


@pytest.mark.parametrize("L,visc", [(31, 0.0), (63, 1e5)])
def test_vort_div_tendency_matches_oracle(gpu, oracle_mod, L, visc):
    from sph_swe_b200.sph import Sph

    s, g = Sph(L), oracle_mod.Grid(L)
    vd = _vd(g)
    st0 = _jet_state(g, vd)
    st0[1:] += random_spec(L, 2, seed=L, decay=3.0) * 1e-5
    st0[1:, 0] = 0.0
    p = Sph.swe_params(radius=A, dt=15.0, viscosity=visc, nonlinear=2)
    tend = s.swe_tendency(p, torch.from_numpy(st0).cuda()).cpu().numpy()
    ref = vd.tendency((A, G, OM, 1e4, visc, 15.0), *st0)
    # the jet is balanced: delta_t is a small difference of the curl and
    # Laplacian terms, so its relative error is larger (measured 2.6e-11 at T63)
    for q in range(3):
        assert rel_l2(tend[q], ref[q]) < (1e-11 if q < 2 else 1e-10), q


def test_vort_div_rk4_matches_oracle(gpu, oracle_mod):
    from sph_swe_b200.sph import Sph

    L, n = 63, 40
    s, g = Sph(L), oracle_mod.Grid(L)
    vd = _vd(g)
    st0 = _jet_state(g, vd, bump_amp=300.0)
    p = Sph.swe_params(radius=A, dt=120.0, nonlinear=2)
    st = torch.from_numpy(st0.copy()).cuda()
    s.swe_rk4(p, st, n)
    out = st.cpu().numpy()
    ref = vd.rk4((A, G, OM, 1e4, 0.0, 120.0), *st0, n)
    for q in range(3):
        assert rel_l2(out[q], ref[q]) < 1e-10, q
    # mass and total circulation change by rounding only
    assert abs(out[0, 0] - st0[0, 0]) < 1e-14 * abs(st0[0, 0])
    assert abs(out[1, 0]) < 1e-18


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
    of h) changes by rounding only, and the mixed form stays within 1e-6 of the
    FP64 form in h and within 1e-4 in vorticity."""
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    out = {}
    st0 = None
    for prec in (capi.SPH_PREC_FP64, capi.SPH_PREC_MIXED):
        s = Sph(1023, precision=prec)
        if st0 is None:
            h, u, v = S.sech2_jet(s, radius=A, bump_amp=120.0)
            c = torch.from_numpy(np.cos(s.lat)).cuda()[None, :]
            z, d = s.vec_spat_to_SH(torch.from_numpy(u[None]).cuda() * c, torch.from_numpy(v[None]).cuda() * c,
                                    robert=True)
            st0 = torch.stack([s.spat_to_SH(torch.from_numpy(h).cuda()), z[0] / A, d[0] / A])
        p = Sph.swe_params(radius=A, dt=15.0, nonlinear=2)
        st = st0.clone()
        s.swe_rk4(p, st, 10)
        capi.check(capi.lib().sph_sync(s.h, None))
        out[prec] = st.cpu().numpy()
        s.close()
    h0 = st0[0, 0].item()
    f64, mx = out[capi.SPH_PREC_FP64], out[capi.SPH_PREC_MIXED]
    assert np.all(np.isfinite(f64))
    assert abs(f64[0, 0] - h0) < 1e-13 * abs(h0)
    assert rel_l2(mx[0], f64[0]) < 1e-6
    assert rel_l2(mx[1], f64[1]) < 1e-4
