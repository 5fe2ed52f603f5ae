"""TEST INFRASTRUCTURE ONLY — ctypes view of the oracle library.

The oracle is a CPU restatement (C++/OpenMP/FP64) of the reference's spectral
shallow-water algorithm.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
bench's ``cpu_baseline`` / ``--impl reference`` legs may use this module, and
only as the checker or the timed CPU baseline, never as the product.

Arrays: real grids are float64 ``(nphi, nlat)`` (index ``i_lon*nlat + j``),
spectral fields are complex128 in the reference's packed layouts.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsph_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_grid_new.restype = ctypes.c_void_p
        L.orc_grid_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_grid_free.argtypes = [ctypes.c_void_p]
        L.orc_grid_info.argtypes = [ctypes.c_void_p, _ip]
        L.orc_grid_arrays.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_plm.restype = ctypes.c_double
        L.orc_plm.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        for name in ("orc_spat_to_SH", "orc_SH_to_spat", "orc_cplx_spat_to_SH", "orc_cplx_SH_to_spat"):
            getattr(L, name).argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        for name in ("orc_spat_to_SH_l", "orc_SH_to_spat_l"):
            getattr(L, name).argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        for name in ("orc_real_op", "orc_cplx_op"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _ip]
            getattr(L, name).restype = ctypes.c_int
        L.orc_zgbsv.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _ip, _dp]
        L.orc_solver.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_solver_rows.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_double,
                                      ctypes.c_int, _dp]
        L.orc_rexi_coeffs.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                      ctypes.c_int]
        L.orc_swe_tendency.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp,
                                       _dp]
        L.orc_swe_run.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]
        L.orc_rexi_run.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]
        L.orc_rexi_pole.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_dp] * 8
        L.orc_auto_grid.argtypes = [ctypes.c_int, _ip, _ip]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def auto_grid(L: int):
    a, b = ctypes.c_int(), ctypes.c_int()
    lib().orc_auto_grid(L, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# operator ids of orc_real_op / orc_cplx_op
OP = dict(diff_lon=0, d1mu2=1, mu=2, mu2=3, laplace=4, grad_lon=5, grad_lat=6, div_lat=7, diff_lat_mu=8,
          robert_div_lon=9, robert_div_lat=10, spec_truncate=11, mul123=12, add100=13, identity=14)
# solver component ids of orc_solver
COMP = dict(scalar_phi=0, mu_phi=1, one_minus_mu_mu_diff_mu_phi=2, z1=3, z2=4, z3=5, z4=6, z4robert=7, z5=8,
            z5robert=9, z6=10, z6robert=11, z7=12, z8=13)


class Grid:
    """Oracle grid (Gauss-Legendre x equispaced) with its transforms."""

    def __init__(self, L: int, nlat: int = 0, nphi: int = 0):
        self.h = lib().orc_grid_new(L, nlat, nphi)
        if not self.h:
            raise ValueError("oracle grid setup failed")
        info = np.zeros(5, np.int32)
        lib().orc_grid_info(self.h, info.ctypes.data_as(_ip))
        self.L, self.nlat, self.nphi, self.nlm, self.ncplx = (int(x) for x in info)
        self.mu = np.zeros(self.nlat)
        self.w = np.zeros(self.nlat)
        self.cosphi = np.zeros(self.nlat)
        self.lat = np.zeros(self.nlat)
        lib().orc_grid_arrays(self.h, _p(self.mu), _p(self.w), _p(self.cosphi), _p(self.lat))
        self.lon = np.arange(self.nphi) / self.nphi * 2.0 * np.pi

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_grid_free(self.h)
            self.h = None

    # layouts
    def idx(self, n, m):
        L = self.L
        return (m * (2 * L - m + 1)) // 2 + n

    def cidx(self, n, m):
        return n * n + n + m

    def plm(self, l, m, j):
        return lib().orc_plm(self.h, l, m, j)

    # grids as (nphi, nlat) from a function of (lon, mu)
    def grid_from(self, f):
        LON, MU = np.meshgrid(self.lon, self.mu, indexing="ij")
        out = np.asarray(f(LON, MU))
        return np.ascontiguousarray(out, dtype=np.complex128 if np.iscomplexobj(out) else np.float64)

    # transforms
    def spat_to_SH(self, spat):
        spat = np.ascontiguousarray(spat, np.float64)
        batch = spat.size // (self.nlat * self.nphi)
        out = np.zeros(spat.shape[:-2] + (self.nlm,), np.complex128)
        lib().orc_spat_to_SH(self.h, _p(spat), out.view(np.float64).ctypes.data_as(_dp), batch)
        return out

    def SH_to_spat(self, spec):
        spec = np.ascontiguousarray(spec, np.complex128)
        batch = spec.size // self.nlm
        out = np.zeros(spec.shape[:-1] + (self.nphi, self.nlat), np.float64)
        lib().orc_SH_to_spat(self.h, spec.view(np.float64).ctypes.data_as(_dp), _p(out), batch)
        return out

    def spat_to_SH_l(self, spat, lmax):
        spat = np.ascontiguousarray(spat, np.float64)
        out = np.zeros(((lmax + 1) * (lmax + 2)) // 2, np.complex128)
        lib().orc_spat_to_SH_l(self.h, _p(spat), out.view(np.float64).ctypes.data_as(_dp), lmax)
        return out

    def SH_to_spat_l(self, spec, lmax):
        spec = np.ascontiguousarray(spec, np.complex128)
        out = np.zeros((self.nphi, self.nlat), np.float64)
        lib().orc_SH_to_spat_l(self.h, spec.view(np.float64).ctypes.data_as(_dp), _p(out), lmax)
        return out

    def cplx_spat_to_SH(self, spat):
        spat = np.ascontiguousarray(spat, np.complex128)
        batch = spat.size // (self.nlat * self.nphi)
        out = np.zeros(spat.shape[:-2] + (self.ncplx,), np.complex128)
        lib().orc_cplx_spat_to_SH(self.h, spat.view(np.float64).ctypes.data_as(_dp),
                                  out.view(np.float64).ctypes.data_as(_dp), batch)
        return out

    def cplx_SH_to_spat(self, spec):
        spec = np.ascontiguousarray(spec, np.complex128)
        batch = spec.size // self.ncplx
        out = np.zeros(spec.shape[:-1] + (self.nphi, self.nlat), np.complex128)
        lib().orc_cplx_SH_to_spat(self.h, spec.view(np.float64).ctypes.data_as(_dp),
                                  out.view(np.float64).ctypes.data_as(_dp), batch)
        return out

    # operators through the lazy-field semantics; returns (kind, array), kind 'spat' or 'spec'
    def real_op(self, op, x, kind="spat"):
        op_id = OP[op] if isinstance(op, str) else op
        if kind == "spat":
            xin = np.ascontiguousarray(x, np.float64).reshape(-1)
            ik = 0
        else:
            xin = np.ascontiguousarray(x, np.complex128).view(np.float64).reshape(-1)
            ik = 1
        buf = np.zeros(max(self.nlat * self.nphi, 2 * self.nlm), np.float64)
        ok = ctypes.c_int()
        rc = lib().orc_real_op(self.h, op_id, ik, _p(xin), _p(buf), ctypes.byref(ok))
        if rc:
            raise RuntimeError(f"orc_real_op rc={rc}")
        if ok.value == 0:
            return "spat", buf[: self.nlat * self.nphi].reshape(self.nphi, self.nlat).copy()
        return "spec", buf[: 2 * self.nlm].view(np.complex128).copy()

    def cplx_op(self, op, x, kind="spat"):
        op_id = OP[op] if isinstance(op, str) else op
        xin = np.ascontiguousarray(x, np.complex128).view(np.float64).reshape(-1)
        ik = 0 if kind == "spat" else 1
        buf = np.zeros(2 * max(self.nlat * self.nphi, self.ncplx), np.float64)
        ok = ctypes.c_int()
        rc = lib().orc_cplx_op(self.h, op_id, ik, _p(xin), _p(buf), ctypes.byref(ok))
        if rc:
            raise RuntimeError(f"orc_cplx_op rc={rc}")
        if ok.value == 0:
            return "spat", buf[: 2 * self.nlat * self.nphi].view(np.complex128).reshape(self.nphi, self.nlat).copy()
        return "spec", buf[: 2 * self.ncplx].view(np.complex128).copy()

    def solver(self, halo, comps, rhs, r=1.0, mode="solve", fix_z5robert=False):
        """comps: list of (name, complex scalar)."""
        ids = np.array([COMP[c] for c, _ in comps], np.int32)
        sc = np.array([[complex(s).real, complex(s).imag] for _, s in comps], np.float64).reshape(-1)
        rhs = np.ascontiguousarray(rhs, np.complex128)
        out = np.zeros(self.ncplx, np.complex128)
        rc = lib().orc_solver(self.h, halo, len(comps), ids.ctypes.data_as(_ip), _p(sc), r, int(fix_z5robert),
                              0 if mode == "solve" else 1, rhs.view(np.float64).ctypes.data_as(_dp),
                              out.view(np.float64).ctypes.data_as(_dp))
        if rc:
            raise RuntimeError(f"orc_solver rc={rc}")
        return out

    def solver_rows(self, halo, comps, r=1.0, fix_z5robert=False):
        ids = np.array([COMP[c] for c, _ in comps], np.int32)
        sc = np.array([[complex(s).real, complex(s).imag] for _, s in comps], np.float64).reshape(-1)
        out = np.zeros((self.ncplx, 2 * halo + 1), np.complex128)
        lib().orc_solver_rows(self.h, halo, len(comps), ids.ctypes.data_as(_ip), _p(sc), r, int(fix_z5robert),
                              out.view(np.float64).ctypes.data_as(_dp))
        return out

    def swe_tendency(self, params, h, u, v, nonlinear=1, robert=0):
        p = np.array(params, np.float64)
        hs, us, vs = (np.ascontiguousarray(a, np.complex128) for a in (h, u, v))
        outs = [np.zeros(self.nlm, np.complex128) for _ in range(3)]
        rc = lib().orc_swe_tendency(self.h, _p(p), nonlinear, robert,
                                    *[a.view(np.float64).ctypes.data_as(_dp) for a in (hs, us, vs)],
                                    *[a.view(np.float64).ctypes.data_as(_dp) for a in outs])
        if rc:
            raise RuntimeError(f"orc_swe_tendency rc={rc}")
        return outs

    def swe_run(self, params, h, u, v, nsteps, nonlinear=1, robert=0):
        """params = (a, g, omega, h0, visc, dt); spectral state in, spectral state out."""
        p = np.array(params, np.float64)
        hs, us, vs = (np.array(a, np.complex128, copy=True) for a in (h, u, v))
        rc = lib().orc_swe_run(self.h, _p(p), nonlinear, robert,
                               *[a.view(np.float64).ctypes.data_as(_dp) for a in (hs, us, vs)], nsteps)
        if rc not in (0, 3):
            raise RuntimeError(f"orc_swe_run rc={rc}")
        return hs, us, vs, rc

    def rexi_pole(self, params, alpha, beta, phi0, u, v, robert=1, coriolis=1, fix_z5robert=False):
        """One pole of SWERexiSPH[Robert]::setup+solve; returns the real spectra of Re(I(beta x))."""
        p = np.array(params, np.float64)
        al = np.array([complex(alpha).real, complex(alpha).imag])
        be = np.array([complex(beta).real, complex(beta).imag])
        ins = [np.ascontiguousarray(a, np.complex128) for a in (phi0, u, v)]
        outs = [np.zeros(self.nlm, np.complex128) for _ in range(3)]
        rc = lib().orc_rexi_pole(self.h, _p(p), robert, coriolis, int(fix_z5robert), _p(al), _p(be),
                                 *[a.view(np.float64).ctypes.data_as(_dp) for a in ins],
                                 *[a.view(np.float64).ctypes.data_as(_dp) for a in outs])
        if rc:
            raise RuntimeError(f"orc_rexi_pole rc={rc}")
        return outs

    def rexi_run(self, params, h, u, v, nsteps, rexi_h=0.2, rexi_M=256, half=False, robert=1, coriolis=1,
                 fix_z5robert=False):
        p = np.array(params, np.float64)
        hs, us, vs = (np.array(a, np.complex128, copy=True) for a in (h, u, v))
        rc = lib().orc_rexi_run(self.h, _p(p), robert, coriolis, rexi_h, rexi_M, int(half), int(fix_z5robert),
                                *[a.view(np.float64).ctypes.data_as(_dp) for a in (hs, us, vs)], nsteps)
        if rc < 0:
            raise RuntimeError(f"orc_rexi_run rc={rc}")
        return hs, us, vs, rc


def zgbsv(n, kl, ku, ab, b):
    ab = np.array(ab, np.complex128, order="F", copy=True)
    ldab = ab.shape[0]
    abc = np.ascontiguousarray(ab.T)  # column j contiguous -> ab[i + j*ldab]
    bb = np.array(b, np.complex128, copy=True)
    ipiv = np.zeros(n, np.int32)
    info = lib().orc_zgbsv(n, kl, ku, abc.view(np.float64).ctypes.data_as(_dp), ldab, ipiv.ctypes.data_as(_ip),
                           bb.view(np.float64).ctypes.data_as(_dp))
    return bb, info


def rexi_coeffs(h, M, L=0, half=True):
    cap = 2 * (M + 11) + 1
    a = np.zeros(cap, np.complex128)
    br = np.zeros(cap, np.complex128)
    bi = np.zeros(cap, np.complex128)
    n = lib().orc_rexi_coeffs(h, M, L, int(half), a.view(np.float64).ctypes.data_as(_dp),
                              br.view(np.float64).ctypes.data_as(_dp), bi.view(np.float64).ctypes.data_as(_dp), cap)
    if n < 0:
        raise ValueError("rexi setup failed")
    return a[:n].copy(), br[:n].copy(), bi[:n].copy()
