"""REXI poles split across ranks (sph_swe_b200.sph.ShardedRexi) on CPU:
gloo, world size 2, each rank's integrator being the oracle's per-pole solve
(SWERexiSPHRobert::solve restated) summed over that rank's poles.  The
all-reduced state must equal the oracle's full REXI step, a rank with no poles
must still take part, and a failure on one rank must raise on both without
leaving the other waiting in a collective."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

P = (6.371e6, 9.80616, 7.292e-5, 1e4, 0.0, 3600.0)
L, M = 15, 16


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _OraclePoles:
    """step(state): state <- sum over this rank's poles of the oracle's pole solve"""

    def __init__(self, g, alpha, beta, fail=False):
        self.g, self.alpha, self.beta, self.fail = g, alpha, beta, fail

    def step(self, state, nsteps=1):
        from sph_swe_b200 import capi

        if self.fail:
            raise capi.SphError(capi.SPH_ERR_SINGULAR, "planted failure")
        h, u, v = (state[q].numpy().copy() for q in range(3))
        acc = [np.zeros_like(h) for _ in range(3)]
        for a, b in zip(self.alpha, self.beta):
            out = self.g.rexi_pole(P, a, b, h * P[1], u, v)
            for q in range(3):
                acc[q] += out[q]
        acc[0] /= P[1]
        state.copy_(torch.from_numpy(np.stack(acc)))
        return state


def _rank(rank, world, port, out, mode):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle
        from sph_swe_b200 import capi
        from sph_swe_b200.sph import ShardedRexi
        from tests.helpers import bump_state, random_spec

        g = oracle.Grid(L)
        alpha, br, _ = oracle.rexi_coeffs(0.2, M, half=False)
        if mode == "one_pole":
            alpha, br = alpha[:1], br[:1]
        h = g.spat_to_SH(bump_state(g))
        u, v = random_spec(L, 2, seed=3, decay=3.0) * 5.0
        st = torch.from_numpy(np.stack([h, u, v]))
        fail = mode == "fail" and rank == 1
        rx = ShardedRexi(alpha, br, lambda a, b: _OraclePoles(g, a, b, fail))
        try:
            rx.step(st, 2)
            out[rank] = ("ok", rx.npoles, st.numpy())
        except capi.SphError as e:
            out[rank] = ("error", rx.npoles, str(e))
    finally:
        dist.destroy_process_group()


def _run(mode):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out, mode), nprocs=world, join=True)
    return dict(out)


def test_sharded_rexi_matches_the_full_step(oracle_mod):
    from tests.helpers import bump_state, random_spec, rel_l2

    res = _run("all")
    g = oracle_mod.Grid(L)
    alpha, _, _ = oracle_mod.rexi_coeffs(0.2, M, half=False)
    assert res[0][1] + res[1][1] == len(alpha)
    h = g.spat_to_SH(bump_state(g))
    u, v = random_spec(L, 2, seed=3, decay=3.0) * 5.0
    rh, ru, rv, _ = g.rexi_run(P, h, u, v, 2, rexi_h=0.2, rexi_M=M, half=False, robert=1)
    for r in (0, 1):
        assert res[r][0] == "ok"
        for q, ref in enumerate((rh, ru, rv)):
            assert rel_l2(res[r][2][q], ref) < 1e-13, (r, q)


def test_sharded_rexi_rank_without_poles():
    res = _run("one_pole")
    assert res[0][1] == 1 and res[1][1] == 0
    assert res[0][0] == res[1][0] == "ok"
    assert np.array_equal(res[0][2], res[1][2])


def test_sharded_rexi_failure_reaches_every_rank():
    res = _run("fail")
    assert res[0][0] == res[1][0] == "error"
    assert "planted failure" in res[1][2]
    assert "another rank" in res[0][2]
