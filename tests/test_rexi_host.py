"""CPU unit test of the host-side REXI band-matrix assembly of the CUDA
library (sph_swe_b200/csrc/rexi_tables.h) against the oracle's
SPHSolverComplex restatement, component by component."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def shim():
    d = tempfile.mkdtemp()
    so = os.path.join(d, "librexi_shim.so")
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I/usr/local/cuda/include", "-o", so,
                    os.path.join(ROOT, "tests", "rexi_tables_shim.cpp")], check=True)
    lib = ctypes.CDLL(so)
    lib.shim_block_row.argtypes = [ctypes.c_int] * 3
    lib.shim_component.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    return lib


COMPS = {2: "z2", 3: "z3", 4: "z4robert", 5: "z5robert", 6: "z6robert", 7: "z7", 8: "z8",
         14: "z4", 15: "z5", 16: "z6"}


@pytest.mark.parametrize("fix", [0, 1])
def test_band_tables_match_oracle(shim, oracle_mod, fix):
    L = 15
    g = oracle_mod.Grid(L)
    nc = g.ncplx
    # block rows are the oracle's N-compact rows
    for m in range(-L, L + 1):
        for n in range(abs(m), L + 1):
            pass
    r, s = 6.37122e6, 0.3 - 0.7j
    for cid, name in COMPS.items():
        out = np.zeros(nc * 5, np.complex128)
        shim.shim_component(L, cid, s.real, s.imag, r, fix, out.view(np.float64).ctypes.data_as(
            ctypes.POINTER(ctypes.c_double)))
        mine = out.reshape(nc, 5)
        halo = 4
        ref = g.solver_rows(halo, [(name, s)], r=r, fix_z5robert=bool(fix))
        # keep only in-block entries of the reference rows (out-of-block ones are
        # stored by the reference but dropped by its band conversion)
        for m in range(-L, L + 1):
            for n in range(abs(m), L + 1):
                row = shim.shim_block_row(L, n, m)
                for k, off in enumerate((-4, -2, 0, 2, 4)):
                    n2 = n + off
                    want = ref[row, off + 4] if abs(m) <= n2 <= L else 0.0
                    assert abs(mine[row, k] - want) <= 1e-15 * max(1.0, abs(want)), (name, n, m, off)
        assert np.all(ref[:, [1, 3, 5, 7]] == 0)


def _cplx_block(g, x_real, brow):
    """complex representation of a real field, in block rows"""
    L = g.L
    out = np.zeros(g.ncplx, complex)
    for n in range(L + 1):
        for m in range(0, n + 1):
            q = x_real[g.idx(n, m)]
            out[brow(n, m)] = q
            if m:
                out[brow(n, -m)] = (-1) ** m * np.conj(q)
    return out


def test_rexi_lane_matches_oracle_pole(shim, oracle_mod):
    """The per-pole arithmetic of the CUDA REXI kernel (rexi_lane.h), run on
    the host over all m-blocks for one pole, against SWERexiSPHRobert::solve."""
    from tests.helpers import bump_state, random_spec, rel_l2

    L = 15
    g = oracle_mod.Grid(L)
    nc = g.ncplx
    shim.shim_rexi_pole.restype = ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    shim.shim_rexi_pole.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 5 + [dp] * 5
    brow = lambda n, m: shim.shim_block_row(L, n, m)
    a_, g_, om, h0, tau = 6.371e6, 9.80616, 7.292e-5, 1e4, 3600.0
    T, P, r = 2 * om, g_ * h0, a_
    ir = 1.0 / r

    def comp(cid, s):
        out = np.zeros(nc * 5, np.complex128)
        shim.shim_component(L, cid, complex(s).real, complex(s).imag, r, 0, out.view(np.float64).ctypes.data_as(dp))
        return out.reshape(nc, 5)

    C2 = comp(7, -P) + comp(2, 2 * T * T)
    C1 = comp(4, -P * T)
    Cm1 = comp(5, P * T ** 3)
    C0 = comp(3, T ** 4) + comp(6, 2 * P * T * T) + comp(8, -P * T * T)
    cphi = np.ascontiguousarray(np.stack([C2, C1, Cm1, C0]))
    cvel = np.ascontiguousarray(comp(2, T * T)[:, 1:4])

    def R(k, m):
        n = k + 1
        return 0.0 if (n < 0 or n < abs(m) or n * n - m * m < 0) else np.sqrt((n * n - m * m) / (4 * n * n - 1))

    def S(k, m):
        n = k - 1
        return 0.0 if (n < 0 or n < abs(m) or n * n - m * m < 0) else np.sqrt(((n + 1) ** 2 - m * m) / ((2 * n + 1) * (2 * n + 3)))

    coef = np.zeros((nc, 4))
    for m in range(-L, L + 1):
        for n in range(abs(m), L + 1):
            coef[brow(n, m)] = [R(n - 1, m), S(n + 1, m), (1 - n) * R(n - 1, m), (n + 2) * S(n + 1, m)]
    h = g.spat_to_SH(bump_state(g))
    u, v = random_spec(L, 2, seed=3, decay=3.0) * 5.0
    phi0 = h * g_
    # pole-independent vectors (as the GPU prep kernels compute them)
    X = g.real_op("diff_lon", u, kind="spec")[1] + g.real_op("d1mu2", v, kind="spec")[1]
    divr = g.spat_to_SH(g.SH_to_spat(X) / g.cosphi[None, :] ** 2)

    def to_cidx(b):
        c = np.zeros(nc, complex)
        for n in range(L + 1):
            for m in range(-n, n + 1):
                c[g.cidx(n, m)] = b[brow(n, m)]
        return c

    def to_block(c):
        b = np.zeros(nc, complex)
        for n in range(L + 1):
            for m in range(-n, n + 1):
                b[brow(n, m)] = c[g.cidx(n, m)]
        return b

    op = lambda name, b: to_block(g.cplx_op(name, to_cidx(b), kind="spec")[1])
    U0, V0, P0 = (_cplx_block(g, x, brow) for x in (u, v, phi0))
    div0 = ir * _cplx_block(g, divr, brow)
    eta0 = ir * (op("diff_lon", V0) - op("d1mu2", U0))
    Me = op("mu", eta0)
    M2p = op("mu2", P0)
    M2u = op("mu2", U0)
    Mv = op("mu", V0)
    V = [div0, Me, P0, M2p, op("mu2", div0), op("mu2", Me), op("mu2", M2p), U0 - M2u, M2u - op("mu2", M2u),
         Mv - op("mu2", Mv), U0, V0, Mv, op("mu", U0)] + [np.zeros(nc, complex)] * 4
    Vst = np.ascontiguousarray(np.stack(V))
    alpha, br, _ = oracle_mod.rexi_coeffs(0.2, 8, half=False)
    for k in (0, 7, 20):
        a, b = alpha[k] / tau, br[k] / tau
        out = np.zeros((3, nc), np.complex128)
        rc = shim.shim_rexi_pole(L, 1, r, T, P, a.real, a.imag, *[x.view(np.float64).ctypes.data_as(dp) if
                                 x.dtype == np.complex128 else x.ctypes.data_as(dp) for x in (cphi, cvel, coef, Vst)],
                                 out.view(np.float64).ctypes.data_as(dp))
        assert rc == 0
        # factors stored once, substitutions from the stored planes: the same numbers
        outs = np.zeros((3, nc), np.complex128)
        shim.shim_rexi_pole_stored.restype = ctypes.c_int
        shim.shim_rexi_pole_stored.argtypes = shim.shim_rexi_pole.argtypes
        rc = shim.shim_rexi_pole_stored(L, 1, r, T, P, a.real, a.imag, *[
            x.view(np.float64).ctypes.data_as(dp) if x.dtype == np.complex128 else x.ctypes.data_as(dp)
            for x in (cphi, cvel, coef, Vst)], outs.view(np.float64).ctypes.data_as(dp))
        assert rc == 0
        assert np.abs(outs - out).max() <= 1e-14 * np.abs(out).max(), k
        ref = g.rexi_pole((a_, g_, om, h0, 0.0, tau), alpha[k], br[k], phi0, u, v)
        for q in range(3):
            c = to_cidx(b * out[q])
            got = np.array([0.5 * (c[g.cidx(n, m)] + (-1) ** m * np.conj(c[g.cidx(n, -m)]))
                            for m in range(L + 1) for n in range(m, L + 1)])
            assert rel_l2(got, ref[q]) < 1e-12, (k, q, rel_l2(got, ref[q]))
