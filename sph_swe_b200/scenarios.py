"""Initial states on the Gauss grid of a handle (host side, FP64 numpy).

Grids are arrays shaped (nphi, nlat) with latitude index j = 0 at the
northernmost ring, as the handle's ``lat`` / ``mu`` tables.

* ``balanced_height``: depth in gradient-wind balance with a zonal flow u(phi),
  g dh/dphi = -a u (2 Omega sin(phi) + u tan(phi) / a), integrated from the
  south pole ring by ring and shifted to a prescribed area mean, following
  BenchmarkGalewsky::setup_initial_h (BenchmarkGalewsky.hpp:101-218).  Each
  interval between neighbouring rings is integrated with a fixed Gauss-Legendre
  rule (the reference uses an adaptive 5-point rule to 1e-13,
  GaussQuadrature.hpp:66-96); the mean uses the same ring-interval area terms.
* ``galewsky``: the barotropically unstable jet and height bump of Galewsky,
  Scott and Polvani (2004) with the constants of BenchmarkGalewsky.hpp:18-36.
* ``sech2_jet``: u = u_max sech^2((phi - phi_c) / width), balanced h, plus the
  Gaussian bump of ``bump``.
"""
from __future__ import annotations

import numpy as np

_GL_ORDER = 24


def _interval_integrals(f, a, b):
    x, w = np.polynomial.legendre.leggauss(_GL_ORDER)
    mid, half = 0.5 * (a + b), 0.5 * (b - a)
    phi = mid[:, None] + half[:, None] * x[None, :]
    return half * (f(phi) @ w)


def balanced_height(lat, u_of_phi, radius, gravity, omega, h_avg=1e4):
    """h on the rings lat[j] (radians, j = 0 north) balancing the zonal flow u_of_phi."""
    lat = np.asarray(lat, np.float64)
    south_to_north = lat[::-1]
    edges = np.concatenate([[-0.5 * np.pi], south_to_north, [0.5 * np.pi]])

    def integrand(phi):
        u = u_of_phi(phi)
        return radius * u * (2.0 * omega * np.sin(phi) + np.tan(phi) / radius * u)

    seg = _interval_integrals(integrand, edges[:-1], edges[1:])
    hg = -np.cumsum(seg)  # geopotential at the end of each interval (last = north pole)
    mterm = (np.sin(edges[1:]) - np.sin(edges[:-1])) * 2.0 * np.pi
    h_comp_avg = float(np.sum(hg * mterm)) / gravity / float(np.sum(mterm))
    h_rings = hg[:-1] / gravity + (h_avg - h_comp_avg)
    return h_rings[::-1].copy()


def bump(lon, mu, amp=500.0, lat0=np.pi / 6, lon0=np.pi / 3, sigma=0.1):
    """amp exp(-(d / sigma)^2), d the great-circle angle to (lat0, lon0)."""
    p = np.arcsin(mu)
    c = np.sin(p) * np.sin(lat0) + np.cos(p) * np.cos(lat0) * np.cos(lon - lon0)
    return amp * np.exp(-(np.arccos(np.clip(c, -1.0, 1.0)) / sigma) ** 2)


def _grids(s):
    return np.meshgrid(np.asarray(s.lon), np.asarray(s.mu), indexing="ij")


def sech2_jet(s, radius=6.371e6, gravity=9.80616, omega=7.292e-5, u_max=80.0, phi_c=np.pi / 4, width=0.1,
              h_avg=1e4, bump_amp=120.0):
    """(h, u, v) grids: zonal jet u_max sech^2((phi - phi_c)/width), v = 0, h in
    gradient-wind balance with area mean h_avg, plus a bump of bump_amp metres
    at (30N, 60E) with sigma = 0.1 rad."""
    def u_of_phi(phi):
        return u_max / np.cosh((phi - phi_c) / width) ** 2

    LON, MU = _grids(s)
    hr = balanced_height(s.lat, u_of_phi, radius, gravity, omega, h_avg)
    h = np.broadcast_to(hr[None, :], LON.shape) + bump(LON, MU, amp=bump_amp)
    u = np.broadcast_to(u_of_phi(np.asarray(s.lat))[None, :], LON.shape)
    return np.ascontiguousarray(h), np.ascontiguousarray(u), np.zeros_like(LON)


def galewsky(s, radius=6.37122e6, gravity=9.80616, omega=7.292e-5, h_avg=1e4, with_bump=True):
    """(h, u, v) grids of the Galewsky test (BenchmarkGalewsky.hpp:18-36,
    59-71, 101-243): jet between phi0 = pi/7 and phi1 = pi/2 - phi0 with
    u_max = 80, balanced h with mean h_avg, bump
    h_hat cos(phi) exp(-((lambda - pi)/alpha)^2) exp(-((phi2 - phi)/beta)^2)."""
    phi0, u_max = np.pi / 7.0, 80.0
    phi1 = 0.5 * np.pi - phi0
    en = np.exp(-4.0 / (phi1 - phi0) ** 2)

    def u_of_phi(phi):
        phi = np.asarray(phi, np.float64)
        inside = (phi > phi0) & (phi < phi1)
        out = np.zeros_like(phi)
        q = phi[inside]
        out[inside] = u_max / en * np.exp(1.0 / ((q - phi0) * (q - phi1)))
        return out

    LON, MU = _grids(s)
    hr = balanced_height(s.lat, u_of_phi, radius, gravity, omega, h_avg)
    h = np.broadcast_to(hr[None, :], LON.shape).copy()
    if with_bump:
        phi2, alpha, beta, h_hat = np.pi / 4.0, 1.0 / 3.0, 1.0 / 15.0, 120.0
        phi = np.arcsin(MU)
        h += h_hat * np.cos(phi) * np.exp(-((LON - np.pi) / alpha) ** 2) * np.exp(-((phi2 - phi) / beta) ** 2)
    u = np.broadcast_to(u_of_phi(np.asarray(s.lat))[None, :], LON.shape)
    return np.ascontiguousarray(h), np.ascontiguousarray(u), np.zeros_like(LON)
