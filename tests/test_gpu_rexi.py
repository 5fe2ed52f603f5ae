"""Parity of the GPU REXI integrator with the oracle, which follows
SWERexiSPHRobert::setup/solve (Robert form, S1), SWERexiSPH::setup/solve
(non-Robert form, S0) and SPHSolverComplex with LAPACK zgbsv semantics
(full-grid Coriolis product, see the oracle header)."""
import numpy as np
import pytest
import torch

from tests.helpers import bump_state, random_spec, rel_l2

pytestmark = pytest.mark.gpu

P6 = (6.371e6, 9.80616, 7.292e-5, 1e4, 0.0, 3600.0)


def _run(gpu_sph, g, oracle_mod, L, M, half, steps, coriolis=1, fix=0, visc=0.0, seed=None, precision=0, robert=1):
    a, br, bi = oracle_mod.rexi_coeffs(0.2, M, half=half)
    h = g.spat_to_SH(bump_state(g))
    if seed is None:
        u = np.zeros(g.nlm, complex)
        v = np.zeros(g.nlm, complex)
    else:
        u, v = random_spec(L, 2, seed=seed, decay=3.0) * 5.0
    p = list(P6)
    p[4] = visc
    rx = gpu_sph.rexi(a, br, radius=p[0], gravity=p[1], omega=p[2], h0=p[3], viscosity=visc, tau=p[5],
                      coriolis=coriolis, fix_z5robert=fix, precision=precision, robert=robert)
    st = torch.from_numpy(np.stack([h, u, v])).cuda()
    rx.step(st, steps)
    out = st.cpu().numpy()
    rh, ru, rv, npol = g.rexi_run(tuple(p), h, u, v, steps, rexi_h=0.2, rexi_M=M, half=half, robert=robert,
                                  coriolis=coriolis, fix_z5robert=fix)
    assert npol == len(a)
    return out, (rh, ru, rv)


@pytest.mark.parametrize("L,M,half,coriolis,fix,visc,seed", [
    (31, 64, False, 1, 0, 0.0, None),
    (31, 64, True, 1, 0, 0.0, 3),
    (31, 32, False, 1, 1, 1e5, 4),
    (31, 32, False, 0, 0, 0.0, 5),
    (63, 64, False, 1, 0, 0.0, 6),
])
def test_rexi_matches_oracle(gpu, oracle_mod, L, M, half, coriolis, fix, visc, seed):
    from sph_swe_b200.sph import Sph

    s, g = Sph(L), oracle_mod.Grid(L)
    out, ref = _run(s, g, oracle_mod, L, M, half, 2, coriolis, fix, visc, seed)
    for q in range(3):
        assert rel_l2(out[q], ref[q]) < 1e-10, q


@pytest.mark.parametrize("L,M,half,coriolis,visc,seed,precision", [
    (31, 64, False, 1, 0.0, None, 0),
    (31, 64, True, 1, 1e5, 7, 0),
    (31, 32, False, 0, 0.0, 8, 0),
    (63, 64, False, 1, 0.0, 9, 0),
    (63, 32, False, 0, 1e5, 10, 0),
    (31, 64, False, 1, 0.0, 11, 1),
])
def test_non_robert_rexi_matches_oracle(gpu, oracle_mod, L, M, half, coriolis, visc, seed, precision):
    """The non-Robert form (SWERexiSPH, S0): Phi systems from the non-Robert z4,
    z5, z6 components (SPHSolverComplex.hpp:221-367), div0 / eta0 and the
    velocity recovery through the grid divisions by cos(phi) of
    SPHOperatorsComplex.  FP64 within 1e-10 of the oracle; the mixed form
    (complex FP32 solves, FP64 refinement) within 1e-9."""
    from sph_swe_b200.sph import Sph

    s, g = Sph(L), oracle_mod.Grid(L)
    out, ref = _run(s, g, oracle_mod, L, M, half, 2, coriolis, 0, visc, seed, precision=precision, robert=0)
    for q in range(3):
        assert rel_l2(out[q], ref[q]) < (1e-10 if precision == 0 else 1e-9), q


def test_non_robert_rexi_config2_size(gpu, oracle_mod):
    """Configuration 2 in the non-Robert form: T127, M = 256 (535 poles),
    tau = 3600 s from the bump, FP64 against the oracle: within 1e-10 after one
    step (measured u 9e-13, v 6e-12).  The map of this configuration grows the
    state geometrically (the reference's own formulation does, oracle and GPU
    alike), and it amplifies the rounding difference of the first step about
    60x in the second (measured u 1.3e-10, v 3.3e-10), so the second step is
    held to 1e-9."""
    from sph_swe_b200.sph import Sph

    L = 127
    s, g = Sph(L), oracle_mod.Grid(L)
    for steps, tol in ((1, 1e-10), (2, 1e-9)):
        out, ref = _run(s, g, oracle_mod, L, 256, False, steps, robert=0)
        for q in range(3):
            assert rel_l2(out[q], ref[q]) < tol, (steps, q, rel_l2(out[q], ref[q]))


def test_rexi_stored_factors_match_on_the_fly(gpu, oracle_mod, monkeypatch):
    """FP64 plans factor every banded system once at creation and only
    substitute per step; SPH_REXI_STORE=0 factors on the fly every step.  Same
    operations in the same order: the two agree to rounding over 4 steps."""
    from sph_swe_b200.sph import Sph

    L = 63
    s, g = Sph(L), oracle_mod.Grid(L)
    a, br, _ = oracle_mod.rexi_coeffs(0.2, 64, half=False)
    h = g.spat_to_SH(bump_state(g))
    u, v = random_spec(L, 2, seed=8, decay=3.0) * 5.0
    outs = []
    for store in ("1", "0"):
        monkeypatch.setenv("SPH_REXI_STORE", store)
        rx = s.rexi(a, br, radius=P6[0], gravity=P6[1], omega=P6[2], h0=P6[3], tau=P6[5])
        st = torch.from_numpy(np.stack([h, u, v])).cuda()
        rx.step(st, 4)
        outs.append(st.cpu().numpy())
        rx.close()
    for q in range(3):
        assert rel_l2(outs[0][q], outs[1][q]) < 1e-14, q


def test_rexi_config2_t127_full_poles(gpu, oracle_mod):
    """REXI config: T127 192x384, Robert, h=0.2, M=256, full pole set (535 poles), tau = 3600 s."""
    from sph_swe_b200.sph import Sph

    s, g = Sph(127), oracle_mod.Grid(127)
    assert (s.nlat, s.nphi) == (192, 384)
    out, ref = _run(s, g, oracle_mod, 127, 256, False, 1)
    for q in range(3):
        assert rel_l2(out[q], ref[q]) < 1e-10, q


@pytest.mark.parametrize("L,M,half,coriolis,seed", [(31, 64, False, 1, 3), (31, 32, True, 0, 4), (63, 64, False, 1, 6)])
def test_mixed_rexi_matches_oracle(gpu, oracle_mod, L, M, half, coriolis, seed):
    """Complex FP32 factorisation and solves with two FP64 refinement steps:
    the refined solution reaches the FP64 result to ~1e-12 (tolerance 1e-9)."""
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    s, g = Sph(L), oracle_mod.Grid(L)
    out, ref = _run(s, g, oracle_mod, L, M, half, 2, coriolis, 0, 0.0, seed, precision=capi.SPH_PREC_MIXED)
    for q in range(3):
        assert rel_l2(out[q], ref[q]) < 1e-9, q


def test_mixed_rexi_config2_vs_fp64(gpu, oracle_mod):
    """REXI configuration (T127, M = 256, 535 poles, tau = 3600 s), 2 steps:
    mixed form against the FP64 direct form.  (Over many steps the Robert
    REXI integration of the reference is not stable at this size: the oracle
    itself grows without bound, so the forms are compared while the solution
    is physical.)"""
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph, rexi_coefficients

    s, g = Sph(127), oracle_mod.Grid(127)
    a, br, _ = rexi_coefficients(0.2, 256, False)
    h = g.spat_to_SH(bump_state(g))
    st0 = torch.from_numpy(np.stack([h, 0 * h, 0 * h])).cuda()
    outs = []
    for prec in (capi.SPH_PREC_FP64, capi.SPH_PREC_MIXED):
        rx = s.rexi(a, br, radius=6.371e6, tau=3600.0, precision=prec)
        st = st0.clone()
        rx.step(st, 2)
        outs.append(st.cpu().numpy())
        rx.close()
    for q in range(3):
        assert rel_l2(outs[1][q], outs[0][q]) < 1e-9, q


def test_rexi_rejects_unsupported(gpu):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    s = Sph(15)
    with pytest.raises(capi.SphError):
        s.rexi([1 + 1j], [1 + 0j], tau=0.0)
    with pytest.raises(capi.SphError):
        s.rexi([1 + 1j], [1 + 0j], precision=7)
