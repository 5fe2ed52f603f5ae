"""TEST INFRASTRUCTURE ONLY (the oracle): numpy restatement of the nonlinear
shallow-water equations in vorticity-divergence form with Robert velocity
variables U = u cos(phi), V = v cos(phi) on the grid, the formulation of the
NCAR spectral shallow-water model (Hack and Jakob 1992, NCAR/TN-343+STR,
eqs. 2.4-2.6 with the grid fields A..E of their section 3).  The reference
has no such form: its nonlinear branch integrates u, v advectively
(AppSWE.hpp:622-650); this restatement is the checker of the library's
`nonlinear = 2` form and of its exact vector transforms.

Prognostic spectra (packed real layout of degree L): h, vorticity zeta,
divergence delta (physical units, radius a).  With eta = zeta + 2 Omega mu:
    zeta_t  = -(1/a) div(eta v)
    delta_t =  (1/a) curl(eta v) - (1/a^2) lap(g h + (u^2 + v^2)/2)
    h_t     = -(1/a) div(h v)
(+ nu lap of each field), div / curl on the unit sphere from the Robert grid
components divided by cos^2(phi), by the degree-(L+1) Gauss analysis and the
identity (1 - mu^2) dP_l/dmu = (l+1) e_l P_{l-1} - l e_{l+1} P_{l+1},
e_l = sqrt((l^2 - m^2) / (4 l^2 - 1)) (integration by parts in mu).
"""
from __future__ import annotations

import numpy as np


def _pidx(T, n, m):
    return (m * (2 * T - m + 1)) // 2 + n


def _e(l, m):
    l = np.asarray(l, np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        v = np.sqrt(np.maximum(l * l - m * m, 0.0) / (4.0 * l * l - 1.0))
    return np.where((l >= abs(m)) & (l >= 1), v, 0.0)


class VortDiv:
    """Exact vector transforms and the vorticity-divergence SWE on an oracle Grid."""

    def __init__(self, grid):
        self.g = grid
        self.L = grid.L
        self.Lp = grid.L + 1
        self.mu = np.asarray(grid.mu, np.float64)
        self.c2 = (1.0 - self.mu) * (1.0 + self.mu)
        L, Lp = self.L, self.Lp
        self.nlm = (L + 1) * (L + 2) // 2
        self.nlmp = (Lp + 1) * (Lp + 2) // 2
        # (n, m) of every packed entry of degree L and of degree L+1
        self.nm = [(n, m) for m in range(L + 1) for n in range(m, L + 1)]
        self.nmp = [(n, m) for m in range(Lp + 1) for n in range(m, Lp + 1)]

    # ---------------------------------------------------------------- helpers
    def _gather(self, x, T, n, m):
        """x at (n, m) of a packed degree-T array, zero outside m <= n <= T (vectorised)."""
        ok = (n >= m) & (n <= T) & (n >= 0)
        k = np.where(ok, (m * (2 * T - m + 1)) // 2 + np.where(ok, n, m), 0)
        return np.where(ok, x[k], 0.0)

    def vec_synthesis(self, vort, div):
        """unit-sphere vort/div (degree L) -> Robert grids U, V (degree L+1 kept)."""
        L, Lp = self.L, self.Lp
        n0 = np.array([n for n, _ in self.nm], np.int64)
        inv = np.where(n0 > 0, -1.0 / np.maximum(n0 * (n0 + 1.0), 1.0), 0.0)
        psi = np.asarray(vort, complex) * inv
        chi = np.asarray(div, complex) * inv
        n = np.array([n for n, _ in self.nmp], np.int64)
        m = np.array([m for _, m in self.nmp], np.int64)
        # (1 - mu^2) d x / dmu at degree n: (n+2) e_{n+1} x_{n+1} - (n-1) e_n x_{n-1}
        cl = -(n - 1.0) * _e(n, m)
        ch = (n + 2.0) * _e(n + 1, m)
        dpsi = cl * self._gather(psi, L, n - 1, m) + ch * self._gather(psi, L, n + 1, m)
        dchi = cl * self._gather(chi, L, n - 1, m) + ch * self._gather(chi, L, n + 1, m)
        keep = m <= L
        Us = np.where(keep, 1j * m * self._gather(chi, L, n, m) - dpsi, 0.0)
        Vs = np.where(keep, 1j * m * self._gather(psi, L, n, m) + dchi, 0.0)
        return self.g.SH_to_spat_l(Us, Lp), self.g.SH_to_spat_l(Vs, Lp)

    def vec_analysis(self, Ug, Vg):
        """Robert grids U, V -> unit-sphere vort, div (degree L)."""
        Lp = self.Lp
        aU = self.g.spat_to_SH_l(Ug / self.c2[None, :], Lp)
        aV = self.g.spat_to_SH_l(Vg / self.c2[None, :], Lp)
        n = np.array([n for n, _ in self.nm], np.int64)
        m = np.array([m for _, m in self.nm], np.int64)
        el = (n + 1.0) * _e(n, m)
        eh = n * _e(n + 1, m)
        vort = 1j * m * self._gather(aV, Lp, n, m) + el * self._gather(aU, Lp, n - 1, m) - eh * self._gather(aU, Lp, n + 1, m)
        div = 1j * m * self._gather(aU, Lp, n, m) - el * self._gather(aV, Lp, n - 1, m) + eh * self._gather(aV, Lp, n + 1, m)
        return vort, div

    # ---------------------------------------------------------------- SWE
    def tendency(self, params, h, zeta, delta):
        """params = (a, g, omega, h0, visc, dt) as the other oracle entry points."""
        a, grav, om, _, visc, _ = params
        U, V = self.vec_synthesis(a * zeta, a * delta)
        Z = self.g.SH_to_spat(zeta)
        H = self.g.SH_to_spat(h)
        ic2 = 1.0 / self.c2[None, :]
        eta = Z + 2.0 * om * self.mu[None, :]
        vf, df = self.vec_analysis(eta * U, eta * V)
        _, dh = self.vec_analysis(H * U, H * V)
        E = self.g.spat_to_SH(grav * H + 0.5 * (U * U + V * V) * ic2)
        ll = np.array([n * (n + 1.0) for n, _ in self.nm])
        ht = -dh / a
        zt = -df / a
        dt_ = vf / a + ll / (a * a) * E
        if visc != 0.0:
            s = -visc / (a * a) * ll
            ht = ht + s * h
            zt = zt + s * zeta
            dt_ = dt_ + s * delta
        return ht, zt, dt_

    def rk4(self, params, h, zeta, delta, nsteps):
        dt = params[5]
        x = [np.array(h, complex), np.array(zeta, complex), np.array(delta, complex)]
        b = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
        for _ in range(nsteps):
            k1 = self.tendency(params, *x)
            k2 = self.tendency(params, *[x[q] + dt * (0.5 * k1[q]) for q in range(3)])
            k3 = self.tendency(params, *[x[q] + dt * (0.5 * k2[q]) for q in range(3)])
            k4 = self.tendency(params, *[x[q] + dt * (1.0 * k3[q]) for q in range(3)])
            x = [x[q] + dt * ((b[0] * k1[q]) + (b[1] * k2[q]) + (b[2] * k3[q]) + (b[3] * k4[q])) for q in range(3)]
        return x
