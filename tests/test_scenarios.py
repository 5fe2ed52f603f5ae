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
def test_jet_is_steady_in_vorticity_divergence_form(oracle_mod, L):
    from oracle.vortdiv import VortDiv

    g = oracle_mod.Grid(L)
    vd = VortDiv(g)
    h, u, v = S.sech2_jet(g, radius=A, bump_amp=0.0)
    c = np.cos(np.asarray(g.lat))[None, :]
    z, d = vd.vec_analysis(u * c, v * c)
    st = (g.spat_to_SH(h), z / A, d / A)
    ht, zt, dt = vd.tendency((A, G, OM, 1e4, 0.0, 15.0), *st)
    # advective scales u_max / a and u_max / (a width) of each field; the
    # gravity term of the divergence equation
    s_h = np.linalg.norm(st[0]) * 80.0 / A
    s_z = np.linalg.norm(st[1]) * 80.0 / (A * 0.1)
    s_d = np.linalg.norm(G * st[0]) / A ** 2 * L * L
    assert np.linalg.norm(ht) < 1e-12 * s_h
    assert np.linalg.norm(zt) < 1e-12 * s_z
    assert np.linalg.norm(dt) < (1e-6 if L == 63 else 1e-10) * s_d


def test_oracle_vector_transforms(oracle_mod):
    """Exact vector pair of the oracle: round trip, and solid-body rotation
    U = cos^2(phi) has vorticity 2 mu and no divergence."""
    from oracle.vortdiv import VortDiv
    from tests.helpers import random_spec

    g = oracle_mod.Grid(31)
    vd = VortDiv(g)
    z, d = random_spec(31, 2, seed=4)
    z[0] = d[0] = 0
    z2, d2 = vd.vec_analysis(*vd.vec_synthesis(z, d))
    assert np.linalg.norm(z2 - z) < 1e-13 * np.linalg.norm(z)
    assert np.linalg.norm(d2 - d) < 1e-13 * np.linalg.norm(d)
    mu = np.asarray(g.mu)
    U = np.broadcast_to((1 - mu ** 2)[None, :], (g.nphi, g.nlat)).copy()
    zz, dd = vd.vec_analysis(U, 0 * U)
    ref = g.spat_to_SH(g.grid_from(lambda lon, m: 2 * m + 0 * lon))
    assert np.abs(zz - ref).max() < 1e-12 and np.abs(dd).max() < 1e-14


def test_vorticity_divergence_form_conserves_mass(oracle_mod):
    from oracle.vortdiv import VortDiv

    g = oracle_mod.Grid(31)
    vd = VortDiv(g)
    h, u, v = S.sech2_jet(g, radius=A, bump_amp=300.0)
    c = np.cos(np.asarray(g.lat))[None, :]
    z, d = vd.vec_analysis(u * c, v * c)
    h0 = g.spat_to_SH(h)
    out = vd.rk4((A, G, OM, 1e4, 0.0, 300.0), h0, z / A, d / A, 20)
    assert abs(out[0][0] - h0[0]) < 1e-14 * abs(h0[0])
    assert abs(out[1][0]) < 1e-20


def test_galewsky_state_shapes(oracle_mod):
    g = oracle_mod.Grid(31)
    h, u, v = S.galewsky(g)
    assert h.shape == u.shape == v.shape == (g.nphi, g.nlat)
    assert np.all(np.isfinite(h)) and np.max(u) <= 80.0 + 1e-9 and np.all(v == 0)
    assert 9000 < h.min() < h.max() < 11000


@pytest.mark.parametrize("L", [63, 127])
def test_galewsky_state_matches_oracle_restatement(oracle_mod, L):
    """scenarios.galewsky (fixed 24-point Gauss rule per ring interval) against
    the oracle's restatement of BenchmarkGalewsky::setup_initial_h with the
    bump (oracle/galewsky.py, adaptive quadrature to the reference's 1e-13)."""
    from oracle import galewsky as G

    g = oracle_mod.Grid(L)
    h, u, v = S.galewsky(g)
    ho, uo, vo = G.initial_state(g.lat, g.nphi, 6.37122e6, 9.80616, 7.292e-5)
    assert np.abs(h - ho).max() < 1e-9  # metres on a 1e4 m mean
    assert np.abs(u - uo).max() < 1e-12
    assert np.array_equal(v, vo)
