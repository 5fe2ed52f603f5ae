"""TEST INFRASTRUCTURE ONLY (the oracle): restatement of the Galewsky initial
state of the reference, BenchmarkGalewsky (src/include/benchmarks/
BenchmarkGalewsky.hpp), for checking the library's scenario Q1.

* Jet (BenchmarkGalewsky.hpp:18-36 constants, 59-71 profile):
  u(phi) = u_max / e_n exp(1 / ((phi - phi0)(phi - phi1))) on phi0 < phi < phi1,
  phi0 = pi/7, phi1 = pi/2 - phi0, u_max = 80, e_n = exp(-4 / (phi1 - phi0)^2).
* Height (setup_initial_h, :101-218): the geopotential of gradient-wind balance
  g dh/dphi = -a u (2 Omega sin(phi) + tan(phi) u / a) is accumulated from the
  south pole ring by ring, hg_j = hg_{j+1} - int_{lat_{j+1}}^{lat_j} f; every
  interval (and the last one, from the northernmost ring to the pole) is
  weighted by its area term (sin(end) - sin(start)) 2 pi to form the mean, and
  h_j = hg_j / g + (h_avg - mean / g).  The reference integrates each interval
  with an adaptive 5-point Gauss rule to 1e-13 (GaussQuadrature.hpp:66-96, a
  published algorithm, restated here by scipy's adaptive quadrature at the
  same relative tolerance).
* Bump (setup_initial_h_add_bump, :221-229):
  h += h_hat cos(phi) exp(-((lambda - pi)/alpha)^2) exp(-((phi2 - phi)/beta)^2),
  phi2 = pi/4, alpha = 1/3, beta = 1/15, h_hat = 120.
* AppSWE stores the jet itself in prog_u, in the Robert form as well
  (AppSWE.hpp:199-206), and v = 0.
"""
from __future__ import annotations

import numpy as np
from scipy import integrate

PHI0 = np.pi / 7.0
PHI1 = 0.5 * np.pi - PHI0
U_MAX = 80.0
EN = np.exp(-4.0 / (PHI1 - PHI0) ** 2)


def u_jet(phi: float) -> float:
    if phi <= PHI0 or phi >= PHI1:
        return 0.0
    return U_MAX / EN * np.exp(1.0 / ((phi - PHI0) * (phi - PHI1)))


def _interval(f, a: float, b: float) -> float:
    v, _ = integrate.quad(f, a, b, epsabs=0.0, epsrel=1e-13, limit=400)
    return v


def initial_h(lat, radius: float, gravity: float, omega: float, h_avg: float = 1e4) -> np.ndarray:
    """h on the rings lat[j] (radians, j = 0 the northernmost), without the bump."""
    lat = np.asarray(lat, np.float64)
    nlat = lat.size

    def f(phi):
        u = u_jet(phi)
        return radius * u * (2.0 * omega * np.sin(phi) + (np.tan(phi) / radius) * u)

    hg = np.zeros(nlat)
    hg_sum = 0.0
    h_area = 0.0
    j = nlat - 1
    start = -0.5 * np.pi
    end = lat[j]
    hg[j] = -_interval(f, start, end)
    mterm = (np.sin(end) - np.sin(start)) * 2.0 * np.pi
    hg_sum += hg[j] * mterm
    h_area += mterm
    start = end
    for j in range(nlat - 2, -1, -1):
        end = lat[j]
        hg[j] = hg[j + 1] - _interval(f, start, end)
        mterm = (np.sin(end) - np.sin(start)) * 2.0 * np.pi
        hg_sum += hg[j] * mterm
        h_area += mterm
        start = end
    end = 0.5 * np.pi
    mterm = (np.sin(end) - np.sin(start)) * 2.0 * np.pi
    hg_sum += (hg[0] - _interval(f, start, end)) * mterm
    h_area += mterm
    h_comp_avg = hg_sum / gravity / h_area
    return hg / gravity + (h_avg - h_comp_avg)


def initial_state(lat, nphi: int, radius: float, gravity: float, omega: float, h_avg: float = 1e4):
    """(h, u, v) grids [nphi][nlat] of scenario Q1 as AppSWE sets it up:
    balanced height plus bump, the jet in prog_u, v = 0."""
    lat = np.asarray(lat, np.float64)
    lam = 2.0 * np.pi * np.arange(nphi) / nphi
    LAM, PHI = np.meshgrid(lam, lat, indexing="ij")
    h = np.broadcast_to(initial_h(lat, radius, gravity, omega, h_avg)[None, :], LAM.shape).copy()
    phi2, alpha, beta, h_hat = np.pi / 4.0, 1.0 / 3.0, 1.0 / 15.0, 120.0
    h += h_hat * np.cos(PHI) * np.exp(-(((LAM - np.pi) / alpha) ** 2)) * np.exp(-(((phi2 - PHI) / beta) ** 2))
    u = np.array([[u_jet(p) for p in lat]] * nphi)
    return h, u, np.zeros_like(h)
