"""The pole split of ShardedRexi with the GPU integrator: on a one-rank
process group over NCCL it must give exactly the all-pole step of Rexi, so
that the split tested with gloo ranks on the CPU (tests/test_rexi_sharded.py,
oracle integrator) carries over to the GPU step: its pole subset, its beta
weights and its linear implicit viscosity."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture()
def one_rank_group(gpu):
    import torch.distributed as dist

    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1)
    try:
        yield None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("viscosity", [0.0, 1e5])
def test_sharded_rexi_on_gpu_matches_all_pole_step(one_rank_group, oracle_mod, viscosity):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Rexi, ShardedRexi, Sph, rexi_coefficients
    from tests.helpers import bump_state, rel_l2

    L = 63
    s = Sph(L)
    g = oracle_mod.Grid(L)
    h0 = g.spat_to_SH(bump_state(g))
    z = np.zeros(g.nlm, complex)
    alpha, beta_re, _ = rexi_coefficients(0.2, 32, False)
    params = capi.RexiParams(6.371e6, 9.80616, 7.292e-5, 1e4, viscosity, 3600.0, 1, 1, 0, 0, 0)
    start = torch.from_numpy(np.stack([h0, z, z])).cuda()
    full = Rexi(s, alpha, beta_re, params)
    ref = full.step(start.clone(), 2).cpu().numpy()
    sh = ShardedRexi.on(s, alpha, beta_re, params)
    assert sh.npoles == len(alpha)
    got = sh.step(start.clone(), 2).cpu().numpy()
    for q in range(3):
        assert rel_l2(got[q], ref[q]) < 1e-13, q
    sh.close()
    full.close()
