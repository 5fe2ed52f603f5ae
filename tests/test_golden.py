"""The committed golden vectors (tests/golden/golden.npz, written by
tests/golden/make_golden.py from the oracle) against the oracle as it is now:
the inputs regenerate bit for bit from their seeds, and the oracle's answers
have not moved (CPU only)."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import C0, C1, C2, OUT
from tests.helpers import bump_state, random_spec, rel_l2


@pytest.fixture(scope="module")
def gold():
    assert os.path.exists(OUT), "tests/golden/golden.npz is missing"
    return dict(np.load(OUT))


def test_golden_inputs_regenerate(gold, oracle_mod):
    assert np.array_equal(random_spec(C1["L"], 2, seed=C1["seeds"][0]), gold["c1_spec"])
    g = oracle_mod.Grid(C0["L"])
    assert rel_l2(g.spat_to_SH(bump_state(g)), gold["c0_h0"]) < 1e-15


def test_oracle_reproduces_config0(gold, oracle_mod):
    g = oracle_mod.Grid(C0["L"])
    z = np.zeros(g.nlm, complex)
    rh, ru, rv, rc = g.swe_run(C0["params"], gold["c0_h0"], z, z, C0["nsteps"])
    assert rc == 0
    for q, r in zip("huv", (rh, ru, rv)):
        assert rel_l2(r, gold["c0_" + q]) < 1e-12, q


def test_oracle_reproduces_config1_transforms(gold, oracle_mod):
    from oracle.vortdiv import VortDiv

    g = oracle_mod.Grid(C1["L"])
    assert rel_l2(g.SH_to_spat(gold["c1_spec"]), gold["c1_grid"]) < 1e-14
    assert rel_l2(g.spat_to_SH(gold["c1_grid"]), gold["c1_back"]) < 1e-14
    assert rel_l2(gold["c1_back"], gold["c1_spec"]) < 1e-13
    U, V = VortDiv(g).vec_synthesis(gold["c1_vort"], gold["c1_div"])
    assert rel_l2(U, gold["c1_U"]) < 1e-14
    assert rel_l2(V, gold["c1_V"]) < 1e-14


def test_oracle_reproduces_config2_rexi(gold, oracle_mod):
    g = oracle_mod.Grid(C2["L"])
    z = np.zeros(g.nlm, complex)
    rh, ru, rv, npol = g.rexi_run(C2["params"], gold["c2_h0"], z, z, C2["nsteps"], rexi_h=C2["rexi_h"],
                                  rexi_M=C2["rexi_M"], half=False, robert=1)
    assert npol == 151
    for q, r in zip("huv", (rh, ru, rv)):
        assert rel_l2(r, gold["c2_" + q]) < 1e-12, q
