"""Host-side initial states (sph_swe_b200.scenarios) and the nonlinear Robert
form of the oracle: the balanced jet is a steady state of that form up to the
truncation error, and the height integrator satisfies the gradient-wind
relation it integrates."""
import numpy as np
import pytest

from sph_swe_b200 import scenarios as S

A, G, OM = 6.371e6, 9.80616, 7.292e-5


def test_balanced_height_satisfies_gradient_wind():
    lat = np.linspace(np.pi / 2 - 1e-3, -np.pi / 2 + 1e-3, 2001)

    def u(phi):
        return 80.0 / np.cosh((phi - np.pi / 4) / 0.1) ** 2

    h = S.balanced_height(lat, u, A, G, OM, h_avg=1e4)
    # central differences on the (uniform) rings against -(a/g) u (f + u tan / a)
    dh = (h[:-2] - h[2:]) / (lat[:-2] - lat[2:])
    phi = lat[1:-1]
    rhs = -(A / G) * u(phi) * (2 * OM * np.sin(phi) + np.tan(phi) / A * u(phi))
    assert np.max(np.abs(dh - rhs)) < 1e-3 * np.max(np.abs(rhs))


def test_balanced_height_area_mean(oracle_mod):
    g = oracle_mod.Grid(63)
    h, _, _ = S.sech2_jet(g, radius=A, bump_amp=0.0)
    # area mean by Gauss quadrature: the reference's ring-interval rule (each
    # interval weighted with the value at its end) is first-order accurate; at
    # T63 the two means differ by 6.6 m
    mean = float(np.sum(h[0] * np.asarray(g.w))) / 2.0
    assert abs(mean - 1e4) < 10.0


@pytest.mark.parametrize("L", [63, 127])
def test_jet_is_steady_in_robert_nonlinear_form(oracle_mod, L):
    g = oracle_mod.Grid(L)
    h, u, v = S.sech2_jet(g, radius=A, bump_amp=0.0)
    c = np.cos(np.asarray(g.lat))[None, :]
    hs, us, vs = g.spat_to_SH(h), g.spat_to_SH(u * c), g.spat_to_SH(v * c)
    ht, ut, vt = g.swe_tendency((A, G, OM, 1e4, 0.0, 15.0), hs, us, vs, nonlinear=2, robert=1)
    # the gravity term alone, for scale
    _, _, vg = g.swe_tendency((A, G, 0.0, 1e4, 0.0, 15.0), hs, 0 * us, 0 * vs, nonlinear=2, robert=1)
    scale = np.linalg.norm(vg)
    assert np.linalg.norm(ht) < 1e-12 * scale
    assert np.linalg.norm(ut) < 1e-12 * scale
    assert np.linalg.norm(vt) < (1e-2 if L == 63 else 1e-5) * scale


def test_galewsky_state_shapes(oracle_mod):
    g = oracle_mod.Grid(31)
    h, u, v = S.galewsky(g)
    assert h.shape == u.shape == v.shape == (g.nphi, g.nlat)
    assert np.all(np.isfinite(h)) and np.max(u) <= 80.0 + 1e-9 and np.all(v == 0)
    assert 9000 < h.min() < h.max() < 11000
