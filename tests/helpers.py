"""Shared test inputs: seeded spectra and the analytic fields of the
reference's test programs (SphereTestSolutions_Gaussian.hpp,
SphereTestSolutions_SPH.hpp), restated in numpy."""
from __future__ import annotations

import numpy as np

# Gaussian bump exp(-10 d^2) centred at (lat pi/4, lon pi/5)
# (SphereTestSolutions_Gaussian.hpp:18-47)
GA_E, GA_CLON, GA_CLAT = 10.0, np.pi / 5, np.pi / 4


def _ga_parts(lon, mu):
    p1 = np.arcsin(mu)
    da = np.sin(p1) * np.sin(GA_CLAT) + np.cos(p1) * np.cos(GA_CLAT) * np.cos(lon - GA_CLON)
    return p1, da, np.arccos(np.clip(da, -1.0, 1.0))


def ga_f(lon, mu):
    _, _, d = _ga_parts(lon, mu)
    return np.exp(-d * d * GA_E)


def ga_dlambda(lon, mu):
    p1, da, d = _ga_parts(lon, mu)
    return -(GA_E * 2.0 * np.cos(p1) * np.cos(GA_CLAT) * np.sin(lon - GA_CLON)) * d * np.exp(-d * d * GA_E) / np.sqrt(
        1 - da ** 2)


def ga_dphi(lon, mu):
    p1, da, d = _ga_parts(lon, mu)
    return GA_E * 2.0 * d * (np.cos(p1) * np.sin(GA_CLAT) - np.sin(p1) * np.cos(GA_CLAT) * np.cos(lon - GA_CLON)) * \
        np.exp(-d * d * GA_E) / np.sqrt(1.0 - da ** 2)


def ga_div_mu(lon, mu):
    p1, da, d = _ga_parts(lon, mu)
    o = np.exp(-GA_E * d * d) * (2.0 * GA_E * np.cos(p1) * d * (
        np.cos(p1) * np.sin(GA_CLAT) - np.sin(p1) * np.cos(GA_CLAT) * np.cos(lon - GA_CLON)) / np.sqrt(1.0 - da * da)
        - np.sin(p1))
    return o / np.cos(p1)


def random_spec(L, nfields, seed, decay=1.5, cplx=False):
    """complex N(0,1) coefficients scaled by (l+1)^-decay; Im = 0 at m = 0 for real fields."""
    rng = np.random.default_rng(seed)
    if cplx:
        n = (L + 1) ** 2
        ls = np.concatenate([np.full(2 * l + 1, l) for l in range(L + 1)])
        x = (rng.standard_normal((nfields, n)) + 1j * rng.standard_normal((nfields, n))) * (ls + 1.0) ** -decay
        return x
    nlm = (L + 1) * (L + 2) // 2
    ls = np.concatenate([np.arange(m, L + 1) for m in range(L + 1)])
    x = (rng.standard_normal((nfields, nlm)) + 1j * rng.standard_normal((nfields, nlm))) * (ls + 1.0) ** -decay
    x[:, : L + 1] = x[:, : L + 1].real
    return x


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def bump_state(grid, amp=500.0, lat0_deg=30.0, lon0_deg=60.0, sigma_frac=0.1, h0=1e4):
    """h = h0 + amp exp(-(d/sigma)^2), d great-circle distance, sigma = sigma_frac * a (angles in radians)."""
    lat0, lon0 = np.deg2rad(lat0_deg), np.deg2rad(lon0_deg)

    def f(lon, mu):
        p = np.arcsin(mu)
        c = np.sin(p) * np.sin(lat0) + np.cos(p) * np.cos(lat0) * np.cos(lon - lon0)
        d = np.arccos(np.clip(c, -1, 1))
        return h0 + amp * np.exp(-(d / sigma_frac) ** 2)

    return grid.grid_from(f)


def random_bumps(grid, n, rng, h0=1e4):
    """n grids h0 + A exp(-(d/sigma)^2): A ~ U(100, 800) m, centre uniform on
    the sphere (sin(lat) ~ U(-1, 1), lon ~ U(0, 2 pi)), sigma ~ U(0.05, 0.2)
    radians; returns an array (n, nphi, nlat)."""
    out = []
    for _ in range(n):
        amp, z, lon0, sig = rng.uniform(100, 800), rng.uniform(-1, 1), rng.uniform(0, 2 * np.pi), rng.uniform(0.05, 0.2)
        lat0 = np.arcsin(z)

        def f(lon, mu, lat0=lat0, lon0=lon0, amp=amp, sig=sig):
            p = np.arcsin(mu)
            c = np.sin(p) * np.sin(lat0) + np.cos(p) * np.cos(lat0) * np.cos(lon - lon0)
            return h0 + amp * np.exp(-(np.arccos(np.clip(c, -1, 1)) / sig) ** 2)

        out.append(grid.grid_from(f))
    return np.stack(out)
