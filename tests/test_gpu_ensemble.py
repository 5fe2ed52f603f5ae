"""Ensembles of uneven truncations advanced by one CUDA graph
(sph_ensemble_*): every member against the FP64 oracle's RK4 run
(AppSWE::run, AppSWE.hpp:293-336, one run per member), and against the
single-member sph_swe_rk4 path of the same library."""
import numpy as np
import pytest
import torch

from tests.helpers import random_bumps, rel_l2

pytestmark = pytest.mark.gpu

RADIUS = 6.371e6


def _members(s, g, n, seed):
    rng = np.random.default_rng(seed)
    h = g.spat_to_SH(random_bumps(g, n, rng))
    st = np.zeros((n, 3, g.nlm), np.complex128)
    st[:, 0] = h
    return st


def _groups(prec, spec):
    from sph_swe_b200.sph import Sph

    out = []
    for L, n, dts in spec:
        s = Sph(L, precision=prec)
        p = s.swe_params(radius=RADIUS, dt=120.0 * 63 / L, nonlinear=1)
        out.append((s, p, n, dts))
    return out


@pytest.mark.parametrize("nsteps", [1, 12])
def test_uneven_ensemble_fp64_vs_oracle(gpu, oracle_mod, nsteps):
    from sph_swe_b200.sph import Ensemble

    spec = [(31, 3, None), (63, 2, [100.0, 80.0]), (127, 1, None)]
    groups, states, init = [], [], []
    for k, (s, p, n, dts) in enumerate(_groups(0, spec)):
        g = oracle_mod.Grid(s.L)
        st0 = _members(s, g, n, seed=20 + k)
        st = torch.from_numpy(st0.copy()).cuda()
        groups.append((s, p, st, dts))
        init.append((g, st0))
    e = Ensemble(groups)
    assert e.launches > 0
    e.step(nsteps)
    for (s, p, st, dts), (g, st0) in zip(groups, init):
        out = st.cpu().numpy()
        for k in range(out.shape[0]):
            dt = p.dt if dts is None else dts[k]
            ref = g.swe_run((p.radius, p.gravity, p.omega, p.h0, p.viscosity, dt), *st0[k], nsteps)
            assert ref[3] == 0
            for q in range(3):
                if q > 0 and np.linalg.norm(ref[q]) == 0:
                    continue
                # the reference's re-projection of h through F(I(h)) moves one
                # tendency evaluation by ~1e-11 at T63 and more at T127
                # (measured 1.1e-10 .. 1.5e-10 in v after 1 .. 12 steps)
                assert rel_l2(out[k, q], ref[q]) < 5e-10, (s.L, k, q)
    e.close()


def test_ensemble_matches_single_member_runs(gpu, oracle_mod):
    """The ensemble graph computes, member by member, what sph_swe_rk4 does."""
    from sph_swe_b200.sph import Ensemble

    spec = [(63, 4, None), (31, 5, None)]
    groups, singles = [], []
    for k, (s, p, n, dts) in enumerate(_groups(0, spec)):
        g = oracle_mod.Grid(s.L)
        st0 = _members(s, g, n, seed=40 + k)
        groups.append((s, p, torch.from_numpy(st0.copy()).cuda(), None))
        for m in range(n):
            one = torch.from_numpy(st0[m].copy()).cuda()
            s.swe_rk4(p, one, 6)
            singles.append((k, m, one.cpu().numpy()))
    e = Ensemble(groups)
    e.step(6)
    for k, m, one in singles:
        out = groups[k][2][m].cpu().numpy()
        for q in range(3):
            assert rel_l2(out[q], one[q]) < 1e-13, (k, m, q)


def test_mixed_ensemble_vs_oracle(gpu, oracle_mod):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Ensemble

    spec = [(31, 2, None), (63, 3, None)]
    groups, init = [], []
    for k, (s, p, n, dts) in enumerate(_groups(capi.SPH_PREC_MIXED, spec)):
        g = oracle_mod.Grid(s.L)
        st0 = _members(s, g, n, seed=60 + k)
        groups.append((s, p, torch.from_numpy(st0.copy()).cuda(), None))
        init.append((g, st0))
    e = Ensemble(groups)
    e.step(10)
    for (s, p, st, _), (g, st0) in zip(groups, init):
        out = st.cpu().numpy()
        for k in range(out.shape[0]):
            ref = g.swe_run((p.radius, p.gravity, p.omega, p.h0, p.viscosity, p.dt), *st0[k], 10)
            assert rel_l2(out[k, 0], ref[0]) < 1e-6
            assert rel_l2(out[k, 1], ref[1]) < 1e-4
            assert rel_l2(out[k, 2], ref[2]) < 1e-4


def test_ensemble_reports_unstable_group(gpu, oracle_mod):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Ensemble

    spec = [(31, 2, None), (63, 2, None)]
    groups = []
    for k, (s, p, n, dts) in enumerate(_groups(0, spec)):
        g = oracle_mod.Grid(s.L)
        st0 = _members(s, g, n, seed=80 + k)
        if k == 1:
            st0[1, 0, 3] = np.nan
        groups.append((s, p, torch.from_numpy(st0).cuda(), None))
    e = Ensemble(groups)
    with pytest.raises(capi.SphError) as ex:
        e.step(2)
    assert ex.value.code == capi.SPH_ERR_NAN
    assert "group(s) 1" in str(ex.value)
