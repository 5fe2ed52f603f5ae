"""Generate tests/golden/golden.npz: oracle outputs for reduced versions of
the benchmark configurations, with the seeds and parameters that made them.

    python -m tests.golden.make_golden

The reference itself cannot run here (it needs SHTNS, FFTW and LAPACK), and
its own tests hold no golden vectors, so these fixtures are outputs of the
oracle (oracle/), whose transforms, operators, band matrices and banded LU are
pinned separately (tests/test_oracle.py).  They freeze the oracle's answers
so that a change to it shows up as a failing CPU test, and they give the GPU
tests a fixed answer that does not depend on running the oracle.

Contents (all spectra in the real packed layout, complex128):
  c0_*  configuration 0 reduced to 20 steps: T63, nonlinear RK4, a = 6.371e6,
        g = 9.80616, Omega = 7.292e-5, h0 = 1e4, nu = 0, dt = 120 s, the 500 m
        bump at (30N, 60E) with sigma = 0.1 a, rest state.
  c1_*  configuration 1 reduced to T31: 2 scalar fields (seed 20261203) and
        one vorticity/divergence pair (seeds 20261204, 20261205), coefficients
        N(0,1) (l+1)^-1.5 with Im = 0 at m = 0; grids of the syntheses
        (nphi x nlat, theta contiguous) and the spectra of their analyses;
        Robert velocities U, V = (u, v) cos(phi) of the pair.
  c2_*  configuration 2 reduced to T31: REXI (Robert), h = 0.2, M = 64, full
        pole set (151 poles), tau = 3600 s, nu = 0, the config-0 bump on
        h0 = 1e4, rest state, 2 steps.
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "golden.npz")

C0 = dict(L=63, params=(6.371e6, 9.80616, 7.292e-5, 1e4, 0.0, 120.0), nsteps=20)
C1 = dict(L=31, seeds=(20261203, 20261204, 20261205))
C2 = dict(L=31, params=(6.371e6, 9.80616, 7.292e-5, 1e4, 0.0, 3600.0), rexi_h=0.2, rexi_M=64, nsteps=2)


def make():
    from oracle import oracle
    from oracle.vortdiv import VortDiv
    from tests.helpers import bump_state, random_spec

    oracle.build()
    out = {}
    g = oracle.Grid(C0["L"])
    h = g.spat_to_SH(bump_state(g))
    z = np.zeros(g.nlm, complex)
    rh, ru, rv, rc = g.swe_run(C0["params"], h, z, z, C0["nsteps"])
    assert rc == 0
    out.update(c0_h0=h, c0_h=rh, c0_u=ru, c0_v=rv)

    g = oracle.Grid(C1["L"])
    spec = random_spec(C1["L"], 2, seed=C1["seeds"][0])
    grid = g.SH_to_spat(spec)
    vort = random_spec(C1["L"], 1, seed=C1["seeds"][1])[0]
    div = random_spec(C1["L"], 1, seed=C1["seeds"][2])[0]
    vort[0] = div[0] = 0.0
    U, V = VortDiv(g).vec_synthesis(vort, div)
    out.update(c1_spec=spec, c1_grid=grid, c1_back=g.spat_to_SH(grid), c1_vort=vort, c1_div=div, c1_U=U, c1_V=V)

    g = oracle.Grid(C2["L"])
    a, br, _ = oracle.rexi_coeffs(C2["rexi_h"], C2["rexi_M"], half=False)
    h = g.spat_to_SH(bump_state(g))
    z = np.zeros(g.nlm, complex)
    rh, ru, rv, npol = g.rexi_run(C2["params"], h, z, z, C2["nsteps"], rexi_h=C2["rexi_h"], rexi_M=C2["rexi_M"],
                                  half=False, robert=1)
    assert npol == len(a) == 151
    out.update(c2_h0=h, c2_h=rh, c2_u=ru, c2_v=rv)
    return out


if __name__ == "__main__":
    np.savez_compressed(OUT, **make())
    print(OUT, os.path.getsize(OUT), "bytes")
