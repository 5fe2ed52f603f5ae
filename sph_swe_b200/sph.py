"""Python host view of the C ABI, on torch CUDA tensors (device memory and
streams only; all arithmetic runs in libsphgpu.so).

Names mirror the reference's SPHConfig surface (SPHConfig.hpp): a ``Sph``
object owns one transform handle for a triangular truncation on a Gauss grid.
Grids are float64 tensors shaped ``(..., nphi, nlat)`` (index i_lon*nlat+j),
spectra complex128 ``(..., nlm)`` (real layout) or ``(..., (L+1)**2)``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import capi


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    if not t.is_cuda:
        raise ValueError("device tensor required")
    if not t.is_contiguous():
        raise ValueError("contiguous tensor required")
    return ctypes.c_void_p(t.data_ptr())


def rexi_coefficients(h: float = 0.2, M: int = 256, half: bool = False):
    """REXI poles alpha and weights beta_re, beta_im (complex128 arrays) of
    e^{ix} ~ sum_n beta_n / (ix + alpha_n); see sph_rexi_coefficients."""
    L = capi.lib()
    n = ctypes.c_int()
    capi.check(L.sph_rexi_coefficients(h, M, int(half), 0, None, None, None, ctypes.byref(n)))
    out = [np.zeros(n.value, np.complex128) for _ in range(3)]
    dp = ctypes.POINTER(ctypes.c_double)
    capi.check(L.sph_rexi_coefficients(h, M, int(half), n.value, *(o.view(np.float64).ctypes.data_as(dp) for o in out),
                                       ctypes.byref(n)))
    return tuple(out)


class Sph:
    """One transform handle (replaces SPHConfig + its shtns_cfg)."""

    def __init__(self, lmax: int, nlat: int = 0, nphi: int = 0, precision: int = capi.SPH_PREC_FP64):
        torch.cuda.init()
        h = ctypes.c_void_p()
        capi.check(capi.lib().sph_create(lmax, lmax, nlat, nphi, precision, ctypes.byref(h)))
        self.h = h
        vals = [ctypes.c_int() for _ in range(5)]
        capi.check(capi.lib().sph_info(self.h, *[ctypes.byref(v) for v in vals]))
        self.L, self.nlat, self.nphi, self.nlm, self.ncplx = (v.value for v in vals)
        self.mu = np.zeros(self.nlat)
        self.cosphi = np.zeros(self.nlat)
        self.w = np.zeros(self.nlat)
        self.lat = np.zeros(self.nlat)
        dp = ctypes.POINTER(ctypes.c_double)
        capi.check(capi.lib().sph_grid(self.h, *[a.ctypes.data_as(dp) for a in (self.mu, self.cosphi, self.w, self.lat)]))
        self.lon = np.arange(self.nphi) / self.nphi * 2.0 * np.pi
        self.precision = precision

    def close(self):
        if getattr(self, "h", None):
            capi.lib().sph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ transforms
    def spat_to_SH(self, spat: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        batch = spat.numel() // (self.nlat * self.nphi)
        if out is None:
            out = torch.empty(spat.shape[:-2] + (self.nlm,), dtype=torch.complex128, device=spat.device)
        capi.check(capi.lib().sph_spat_to_SH(self.h, _ptr(spat), _ptr(out), batch, 0, 0, _stream()))
        return out

    def SH_to_spat(self, spec: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        batch = spec.numel() // self.nlm
        if out is None:
            out = torch.empty(spec.shape[:-1] + (self.nphi, self.nlat), dtype=torch.float64, device=spec.device)
        capi.check(capi.lib().sph_SH_to_spat(self.h, _ptr(spec), _ptr(out), batch, 0, 0, _stream()))
        return out

    def cplx_spat_to_SH(self, spat: torch.Tensor) -> torch.Tensor:
        batch = spat.numel() // (self.nlat * self.nphi)
        out = torch.empty(spat.shape[:-2] + (self.ncplx,), dtype=torch.complex128, device=spat.device)
        capi.check(capi.lib().sph_cplx_spat_to_SH(self.h, _ptr(spat), _ptr(out), batch, 0, 0, _stream()))
        return out

    def cplx_SH_to_spat(self, spec: torch.Tensor) -> torch.Tensor:
        batch = spec.numel() // self.ncplx
        out = torch.empty(spec.shape[:-1] + (self.nphi, self.nlat), dtype=torch.complex128, device=spec.device)
        capi.check(capi.lib().sph_cplx_SH_to_spat(self.h, _ptr(spec), _ptr(out), batch, 0, 0, _stream()))
        return out

    def vec_SH_to_spat(self, vort: torch.Tensor, div: torch.Tensor, robert: bool = False, out=None):
        batch = vort.numel() // self.nlm
        if out is None:
            u = torch.empty(vort.shape[:-1] + (self.nphi, self.nlat), dtype=torch.float64, device=vort.device)
            v = torch.empty_like(u)
        else:
            u, v = out
        capi.check(capi.lib().sph_vec_SH_to_spat(self.h, _ptr(vort), _ptr(div), _ptr(u), _ptr(v), batch, int(robert),
                                                 _stream()))
        return u, v

    def vec_spat_to_SH(self, u: torch.Tensor, v: torch.Tensor, robert: bool = False, out=None):
        batch = u.numel() // (self.nlat * self.nphi)
        if out is None:
            vort = torch.empty(u.shape[:-2] + (self.nlm,), dtype=torch.complex128, device=u.device)
            div = torch.empty_like(vort)
        else:
            vort, div = out
        capi.check(capi.lib().sph_vec_spat_to_SH(self.h, _ptr(u), _ptr(v), _ptr(vort), _ptr(div), batch, int(robert),
                                                 _stream()))
        return vort, div

    def legendre_synthesis(self, spec: torch.Tensor, four: torch.Tensor) -> torch.Tensor:
        batch = spec.numel() // self.nlm
        capi.check(capi.lib().sph_legendre_synthesis(self.h, _ptr(spec), _ptr(four), batch, _stream()))
        return four

    def legendre_analysis(self, four: torch.Tensor, spec: torch.Tensor) -> torch.Tensor:
        batch = spec.numel() // self.nlm
        capi.check(capi.lib().sph_legendre_analysis(self.h, _ptr(four), _ptr(spec), batch, _stream()))
        return spec

    # ------------------------------------------------------------ operators
    def spec_op(self, op, x: torch.Tensor, a: complex = 0.0, b: complex = 0.0, cplx: bool = False,
                out: torch.Tensor | None = None) -> torch.Tensor:
        n = self.ncplx if cplx else self.nlm
        batch = x.numel() // n
        if out is None:
            out = torch.zeros_like(x) if op in ("axpy", capi.OPS["axpy"]) else torch.empty_like(x)
        op_id = capi.OPS[op] if isinstance(op, str) else int(op)
        a, b = complex(a), complex(b)
        capi.check(capi.lib().sph_spec_op(self.h, op_id, _ptr(x), _ptr(out), a.real, a.imag, b.real, b.imag, batch,
                                          int(cplx), _stream()))
        return out

    def spec_copy_modes(self, x: torch.Tensor, dst: "Sph") -> torch.Tensor:
        """Real spectra of this handle's truncation re-laid out for `dst`'s
        truncation: shared coefficients copied, the rest zero
        (SPHData::spec_copyToDifferentModes; see sph_spec_copy_modes)."""
        batch = x.numel() // self.nlm
        out = torch.empty(x.shape[:-1] + (dst.nlm,), dtype=torch.complex128, device=x.device)
        capi.check(capi.lib().sph_spec_copy_modes(self.h, _ptr(x), dst.h, _ptr(out), batch, _stream()))
        return out

    # ------------------------------------------------------------ autotuner
    def autotune(self, batch: int, families: int | None = None) -> dict:
        """Time the kernel variants for `batch` fields per launch, keep the
        fastest in the handle, return the table (see sph_autotune; families: a
        mask of capi.SPH_TUNE_*, default int8 and FP64)."""
        import json

        buf = ctypes.create_string_buffer(1 << 16)
        if families is None:
            capi.check(capi.lib().sph_autotune(self.h, batch, buf, len(buf), _stream()))
        else:
            capi.check(capi.lib().sph_autotune_ex(self.h, batch, families, buf, len(buf), _stream()))
        return json.loads(buf.value.decode())

    def tune_load(self, table) -> None:
        import json

        text = table if isinstance(table, str) else json.dumps(table)
        capi.check(capi.lib().sph_tune_load(self.h, text.encode()))

    def tune_clear(self) -> None:
        capi.check(capi.lib().sph_tune_clear(self.h))

    @staticmethod
    def rk4_batches(nmem: int, nonlinear: int = 1) -> list:
        """Fields per launch of the transform stages of one RK4 stage over nmem
        members: Legendre synthesis 6n and 2n, analysis 4n and n, ring
        synthesis 9n, ring analysis 4n (reference forms); 4n and 5n for the
        vorticity-divergence form (nonlinear = 2)."""
        if nonlinear == 2:
            return sorted({4 * nmem, 5 * nmem})
        return sorted({6 * nmem, 2 * nmem, 4 * nmem, nmem, 9 * nmem})

    # ------------------------------------------------------------ SWE
    @staticmethod
    def swe_params(radius=6.37122e6, gravity=9.80616, omega=7.292e-5, h0=1e4, viscosity=0.0, dt=120.0,
                   nonlinear=1, robert=0) -> capi.SWEParams:
        return capi.SWEParams(radius, gravity, omega, h0, viscosity, dt, nonlinear, robert)

    def swe_tendency(self, p: capi.SWEParams, state: torch.Tensor) -> torch.Tensor:
        tend = torch.empty_like(state)
        capi.check(capi.lib().sph_swe_tendency(self.h, ctypes.byref(p), _ptr(state), _ptr(tend), _stream()))
        return tend

    def swe_rk4(self, p: capi.SWEParams, state: torch.Tensor, nsteps: int) -> torch.Tensor:
        """In place on state (3, nlm) complex128 = [h, u, v]."""
        capi.check(capi.lib().sph_swe_rk4(self.h, ctypes.byref(p), _ptr(state), nsteps, _stream()))
        return state

    def swe_rk4_batched(self, p: capi.SWEParams, state: torch.Tensor, nsteps: int, dts=None) -> torch.Tensor:
        nmem = state.numel() // (3 * self.nlm)
        arr = None
        if dts is not None:
            arr = np.ascontiguousarray(dts, np.float64)
            arr_p = arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        else:
            arr_p = None
        capi.check(capi.lib().sph_swe_rk4_batched(self.h, ctypes.byref(p), arr_p, _ptr(state), nmem, nsteps,
                                                  _stream()))
        return state

    # ------------------------------------------------------------ REXI
    def rexi(self, alpha, beta, radius=6.37122e6, gravity=9.80616, omega=7.292e-5, h0=1e4, viscosity=0.0,
             tau=3600.0, robert=1, coriolis=1, fix_z5robert=0, precision=capi.SPH_PREC_FP64) -> "Rexi":
        return Rexi(self, alpha, beta, capi.RexiParams(radius, gravity, omega, h0, viscosity, tau, robert, coriolis,
                                                       fix_z5robert, precision))

    # ------------------------------------------------------------ helpers
    def grid_from(self, f) -> np.ndarray:
        LON, MU = np.meshgrid(self.lon, self.mu, indexing="ij")
        return np.ascontiguousarray(f(LON, MU))


class Rexi:
    """REXI integrator (replaces the per-pole SWERexiSPHRobert set of AppSWE::run)."""

    def __init__(self, sph: Sph, alpha, beta, params: capi.RexiParams):
        self.sph = sph
        a = np.ascontiguousarray(np.asarray(alpha, np.complex128)).view(np.float64)
        b = np.ascontiguousarray(np.asarray(beta, np.complex128)).view(np.float64)
        dp = ctypes.POINTER(ctypes.c_double)
        r = ctypes.c_void_p()
        capi.check(capi.lib().sph_rexi_create(sph.h, a.ctypes.data_as(dp), b.ctypes.data_as(dp), len(a) // 2,
                                              ctypes.byref(params), ctypes.byref(r)))
        self.r = r
        self.npoles = len(a) // 2

    def step(self, state: torch.Tensor, nsteps: int = 1) -> torch.Tensor:
        """In place on state (3, nlm) complex128 = [h, u, v] (Robert u cos(phi), v cos(phi))."""
        capi.check(capi.lib().sph_rexi_step(self.r, _ptr(state), nsteps, _stream()))
        return state

    def close(self):
        if getattr(self, "r", None):
            capi.lib().sph_rexi_destroy(self.r)
            self.r = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass



class ShardedRexi:
    """REXI with its poles split across the ranks of a torch.distributed
    process group, one GPU per rank (the reference loops over all poles one
    after another, AppSWE.hpp:452-523).  Rank r keeps poles r, r + W, r + 2W,
    ... of the W ranks and each step sums only those; one all-reduce (sum) of
    the state [h, u, v] per step then adds the ranks' parts.  The split is
    exact: everything after the per-pole solves (the beta-weighted sum, the
    real-part extraction, the implicit viscosity factor) is linear in the
    poles' contributions.  Every rank takes the same collectives in the same
    order, also when its own step fails; a failure on any rank (or a
    non-finite h after the sum) raises SphError on all of them.

    make_rexi(alpha_part, beta_part) builds the per-rank integrator (an
    object with step(state, nsteps)); ShardedRexi.on(...) uses Rexi."""

    def __init__(self, alpha, beta, make_rexi, group=None):
        import torch.distributed as dist

        self.group = group
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        a = np.asarray(alpha, np.complex128)[rank::world]
        b = np.asarray(beta, np.complex128)[rank::world]
        self.npoles = len(a)
        self.rx = make_rexi(a, b) if len(a) else None

    @classmethod
    def on(cls, sph: Sph, alpha, beta, params: capi.RexiParams, group=None) -> "ShardedRexi":
        return cls(alpha, beta, lambda a, b: Rexi(sph, a, b, params), group)

    def step(self, state: torch.Tensor, nsteps: int = 1) -> torch.Tensor:
        """In place on state (3, nlm) complex128 = [h, u, v], on every rank."""
        import torch.distributed as dist

        for _ in range(nsteps):
            err = None
            try:
                if self.rx is None:
                    state.zero_()
                else:
                    self.rx.step(state, 1)
            except capi.SphError as e:
                err = e
                state.zero_()
            dist.all_reduce(torch.view_as_real(state), group=self.group)
            code = torch.tensor([0.0 if err is None else float(err.code)], dtype=torch.float64, device=state.device)
            dist.all_reduce(code, op=dist.ReduceOp.MAX, group=self.group)
            if code.item() != 0.0:
                if err is not None:
                    raise err
                raise capi.SphError(int(code.item()), "REXI step failed on another rank")
            if not bool(torch.isfinite(torch.view_as_real(state[0])).all()):
                raise capi.SphError(capi.SPH_ERR_NAN, "REXI step: instability detected (non-finite value in h)")
        return state

    def close(self):
        if self.rx is not None and hasattr(self.rx, "close"):
            self.rx.close()
        self.rx = None

class Ensemble:
    """Members of several truncations advanced by one CUDA graph.

    groups: list of (sph, params, state, dts) with state a contiguous
    complex128 tensor of shape (nmem, 3, nlm) on the device (bound at creation,
    stepped in place) and dts a per-member array or None (params.dt)."""

    def __init__(self, groups):
        n = len(groups)
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        self._keep = []
        handles = (vp * n)(*[g[0].h for g in groups])
        params = (capi.SWEParams * n)(*[g[1] for g in groups])
        states = (vp * n)(*[g[2].data_ptr() for g in groups])
        nmem = (ctypes.c_int * n)(*[g[2].numel() // (3 * g[0].nlm) for g in groups])
        dts = (dp * n)()
        for k, g in enumerate(groups):
            if g[0].nlm * 3 * nmem[k] != g[2].numel() or not g[2].is_contiguous():
                raise ValueError(f"group {k}: state must be contiguous (nmem, 3, nlm)")
            if g[3] is not None:
                arr = np.ascontiguousarray(g[3], np.float64)
                self._keep.append(arr)
                dts[k] = arr.ctypes.data_as(dp)
        self.groups = groups
        e = ctypes.c_void_p()
        capi.check(capi.lib().sph_ensemble_create(n, handles, params, states, nmem, dts, ctypes.byref(e)))
        self.e = e

    @property
    def launches(self) -> int:
        return capi.lib().sph_ensemble_launches(self.e)

    def step(self, nsteps: int = 1):
        capi.check(capi.lib().sph_ensemble_step(self.e, nsteps, _stream()))

    def close(self):
        if getattr(self, "e", None):
            capi.lib().sph_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
