"""The autotuner (sph_autotune / sph_tune_load / sph_tune_clear): every
candidate variant runs, the chosen table re-applies, and the transforms give
the same results with any variant: within the int8 family the column tiles
and the m orders are exact alternatives (bitwise equal); the split-TF32
variants and the FP64 kernel that a mixed handle may take instead agree with
it to the mixed-form tolerance."""
import numpy as np
import pytest
import torch

from tests.helpers import random_spec, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,prec", [(63, 1), (127, 0), (255, 1)])
def test_autotune_table_and_results(gpu, oracle_mod, L, prec):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    s = Sph(L, precision=prec)
    nb = 24
    spec = torch.from_numpy(random_spec(L, nb, seed=L)).cuda()
    grid0 = s.SH_to_spat(spec)
    back0 = s.spat_to_SH(grid0)
    table = s.autotune(nb)
    assert table["lmax"] == L and table["batch"] == nb
    names = {k["name"] for k in table["kernels"]}
    assert {"ring_analysis", "ring_synthesis"} <= names
    if prec == capi.SPH_PREC_MIXED:
        assert {"legendre_synthesis_tc", "legendre_analysis_tc"} <= names
        tc = [k for k in table["kernels"] if k["name"].endswith("_tc")]
        # the default families: int8 (4 kernels x 3 tiles) and the FP64 kernel
        assert all(len(k["candidates"]) == 13 for k in tc)
        full = s.autotune(nb, families=capi.SPH_TUNE_INT8 | capi.SPH_TUNE_TF32 | capi.SPH_TUNE_FP64)
        tcf = [k for k in full["kernels"] if k["name"].endswith("_tc")]
        assert all(len(k["candidates"]) == 22 for k in tcf)
        s.tune_load(table)
    for k in table["kernels"]:
        assert k["us"] > 0 and k["us"] == min(c["us"] for c in k["candidates"])
    grid1 = s.SH_to_spat(spec)
    back1 = s.spat_to_SH(grid1)
    capi.check(capi.lib().sph_sync(s.h, None))
    tol = 1e-15
    # a mixed handle's tuner may pick a split-TF32 variant or the FP64 kernel:
    # within the mixed form's 1e-6
    tuned_tol = tol if prec == 0 else 1e-6
    assert rel_l2(grid1.cpu().numpy(), grid0.cpu().numpy()) < tuned_tol
    assert rel_l2(back1.cpu().numpy(), back0.cpu().numpy()) < tuned_tol
    # every variant forced through a loaded table gives the same transforms
    variants = [0, 1, 2] if prec == 0 else [1, 2, 3, 65, 66, 67, 129, 130, 131, 193, 194, 195, 33, 34, 35, 5, 6, 7,
                                         9, 10, 11, 16]
    for v in variants:
        forced = {"lmax": L, "nphi": s.nphi, "kernels": [
            {"kind": kind, "batch": nb, "variant": (v if kind < 2 else v % 3)} for kind in range(4)]}
        s.tune_load(forced)
        g = s.SH_to_spat(spec)
        b = s.spat_to_SH(g)
        # int8 variants (no bit among 4, 8, 16, 32) are bitwise alternatives of the
        # default; the split-TF32 variants and the FP64 kernel (16) differ from it
        # by the mixed form's error
        same_family = prec == 0 or not (v & (4 | 8 | 16 | 32))
        vt = 1e-15 if same_family else tuned_tol
        assert rel_l2(g.cpu().numpy(), grid0.cpu().numpy()) < vt, v
        assert rel_l2(b.cpu().numpy(), back0.cpu().numpy()) < (vt if same_family else 2 * tuned_tol), v
    s.tune_clear()
    with pytest.raises(capi.SphError):
        s.tune_load({"lmax": L + 1, "nphi": s.nphi, "kernels": [{"kind": 0, "batch": 1, "variant": 1}]})


def test_autotuned_rk4_matches_untuned(gpu, oracle_mod):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph
    from tests.helpers import bump_state

    L = 63
    g = oracle_mod.Grid(L)
    h = g.spat_to_SH(bump_state(g))
    st0 = torch.from_numpy(np.stack([h, 0 * h, 0 * h])).cuda()
    p = Sph.swe_params(radius=6.371e6, dt=120.0)
    out = []
    for tune in (False, True):
        s = Sph(L, precision=capi.SPH_PREC_MIXED)
        st = st0.clone()
        s.swe_rk4(p, st, 5)  # captures the step graph with the built-in rules
        if tune:
            for b in Sph.rk4_batches(1):
                s.autotune(b)
            st = st0.clone()
            s.swe_rk4(p, st, 5)  # re-captured with the tuned variants
            assert capi.lib().sph_swe_rk4_launches(s.h) > 0
        else:
            st = st0.clone()
            s.swe_rk4(p, st, 5)
        out.append(st.cpu().numpy())
    # the tuned handle may run some stages on the FP64 kernel: the two runs then
    # differ by the mixed form's error (h 2.6e-8 after 200 steps at T63)
    for q in range(3):
        assert rel_l2(out[1][q], out[0][q]) < (1e-6 if q else 1e-8)
