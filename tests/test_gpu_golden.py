"""The CUDA path against the committed golden vectors (oracle outputs for
reduced configurations 0-2, tests/golden/make_golden.py), with the
tolerances of the oracle parity tests: transforms 1e-12, RK4 and REXI 1e-10."""
import numpy as np
import pytest
import torch

from tests.golden.make_golden import C0, C1, C2, OUT
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(OUT))


def test_config0_rk4_matches_golden(gpu, gold):
    from sph_swe_b200.sph import Sph

    a, g, om, h0, nu, dt = C0["params"]
    s = Sph(C0["L"])
    p = Sph.swe_params(radius=a, gravity=g, omega=om, h0=h0, viscosity=nu, dt=dt, nonlinear=1, robert=0)
    z = np.zeros_like(gold["c0_h0"])
    st = torch.from_numpy(np.stack([gold["c0_h0"], z, z])).cuda()
    s.swe_rk4(p, st, C0["nsteps"])
    out = st.cpu().numpy()
    for k, q in enumerate("huv"):
        assert rel_l2(out[k], gold["c0_" + q]) < 1e-10, q


def test_config1_transforms_match_golden(gpu, gold):
    from sph_swe_b200.sph import Sph

    s = Sph(C1["L"])
    grid = s.SH_to_spat(torch.from_numpy(gold["c1_spec"]).cuda()).cpu().numpy()
    assert rel_l2(grid, gold["c1_grid"]) < 1e-12
    back = s.spat_to_SH(torch.from_numpy(gold["c1_grid"]).cuda()).cpu().numpy()
    assert rel_l2(back, gold["c1_back"]) < 1e-12
    U, V = s.vec_SH_to_spat(torch.from_numpy(gold["c1_vort"][None]).cuda(),
                            torch.from_numpy(gold["c1_div"][None]).cuda(), robert=True)
    assert rel_l2(U.cpu().numpy()[0], gold["c1_U"]) < 1e-12
    assert rel_l2(V.cpu().numpy()[0], gold["c1_V"]) < 1e-12


def test_config2_rexi_matches_golden(gpu, gold, oracle_mod):
    from sph_swe_b200.sph import Sph

    a, br, _ = oracle_mod.rexi_coeffs(C2["rexi_h"], C2["rexi_M"], half=False)
    r, g, om, h0, nu, tau = C2["params"]
    s = Sph(C2["L"])
    rx = s.rexi(a, br, radius=r, gravity=g, omega=om, h0=h0, viscosity=nu, tau=tau)
    z = np.zeros_like(gold["c2_h0"])
    st = torch.from_numpy(np.stack([gold["c2_h0"], z, z])).cuda()
    rx.step(st, C2["nsteps"])
    out = st.cpu().numpy()
    for k, q in enumerate("huv"):
        assert rel_l2(out[k], gold["c2_" + q]) < 1e-10, q
