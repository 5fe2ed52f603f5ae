"""Mixed-precision form (SPH_PREC_MIXED): Legendre stage on tcgen05, by
default the int8 integer-split kernels (exact int32 digit-product sums, one
FP64 combination per tile), everything else FP64.

Tolerances (relative L2 against the FP64 oracle / FP64 GPU path):
  scalar synthesis and analysis           <= 1e-6  (measured ~1e-8)
  vector synthesis u, v                   <= 1e-6  (the m = 0 column of the
      Robert velocities is synthesised in FP64: it vanishes like cos^2 at the
      poles while its terms do not, and u = U / cos would amplify the error)
  vector round trip vort -> u,v -> vort   <= 1e-6
  nonlinear RK4, T63, 200 steps: h <= 1e-6; u, v <= 1e-4 (the 200-step map
      amplifies each transform's error in the velocity, which starts from rest)
The split-TF32 kernels (autotuner variants) reach ~3e-7 per transform.
"""
import numpy as np
import pytest
import torch

from tests.helpers import ga_f, random_spec, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _mixed(L):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    return Sph(L, precision=capi.SPH_PREC_MIXED)


def _sync_ok(s):
    from sph_swe_b200 import capi

    assert capi.lib().sph_sync(s.h, None) == capi.SPH_OK, capi.last_error()


# batch sizes exercise the 8-, 16- and 32-field column tiles and a ragged last tile
@pytest.mark.parametrize("L,nb", [(31, 1), (31, 13), (63, 8), (63, 37), (127, 16), (127, 20), (255, 3), (255, 64)])
def test_scalar_transforms_vs_oracle(gpu, oracle_mod, L, nb):
    s = _mixed(L)
    g = oracle_mod.Grid(L)
    spec = random_spec(L, nb, seed=100 + L + nb)
    ref = g.SH_to_spat(spec)
    out = s.SH_to_spat(torch.from_numpy(spec).cuda()).cpu().numpy()
    _sync_ok(s)
    for b in range(nb):
        assert rel_l2(out[b], ref[b]) < TOL
    back = s.spat_to_SH(torch.from_numpy(ref).cuda()).cpu().numpy()
    _sync_ok(s)
    ana = g.spat_to_SH(ref)
    for b in range(nb):
        assert rel_l2(back[b], ana[b]) < TOL


def test_analysis_of_non_bandlimited_field(gpu, oracle_mod):
    s = _mixed(63)
    g = oracle_mod.Grid(63)
    f = g.grid_from(ga_f)
    out = s.spat_to_SH(torch.from_numpy(f).cuda()).cpu().numpy()
    _sync_ok(s)
    assert rel_l2(out, g.spat_to_SH(f)) < TOL


@pytest.mark.parametrize("L", [63, 255])
def test_vector_pair_vs_fp64(gpu, L):
    from sph_swe_b200.sph import Sph

    s, s64 = _mixed(L), Sph(L)
    vort = torch.from_numpy(random_spec(L, 2, seed=5)).cuda()
    div = torch.from_numpy(random_spec(L, 2, seed=6)).cuda()
    vort[:, 0] = 0
    div[:, 0] = 0
    for robert in (False, True):
        u, v = s.vec_SH_to_spat(vort, div, robert=robert)
        u64, v64 = s64.vec_SH_to_spat(vort, div, robert=robert)
        eu = rel_l2(u.cpu().numpy(), u64.cpu().numpy())
        ev = rel_l2(v.cpu().numpy(), v64.cpu().numpy())
        assert eu < TOL and ev < TOL, (robert, eu, ev)
        z, d = s.vec_spat_to_SH(u, v, robert=robert)
        ez = rel_l2(z.cpu().numpy(), vort.cpu().numpy())
        ed = rel_l2(d.cpu().numpy(), div.cpu().numpy())
        assert ez < TOL and ed < TOL, (robert, ez, ed)
    _sync_ok(s)


def test_config0_rk4_vs_oracle(gpu, oracle_mod):
    """Plain-method configuration (T63 96x192, nonlinear RK4, bump 500 m at
    (30N, 60E), dt = 120 s, 200 steps) run in the mixed form: h, u, v within
    the tolerances of the module docstring of the FP64 oracle."""
    from tests.helpers import bump_state

    L = 63
    s = _mixed(L)
    g = oracle_mod.Grid(L)
    p = s.swe_params(radius=6.371e6, dt=120.0, nonlinear=1)
    h = g.spat_to_SH(bump_state(g))
    u = np.zeros(g.nlm, complex)
    v = np.zeros(g.nlm, complex)
    st = torch.from_numpy(np.stack([h, u, v])).cuda()
    s.swe_rk4(p, st, 200)
    _sync_ok(s)
    out = st.cpu().numpy()
    rh, ru, rv, rc = g.swe_run((p.radius, p.gravity, p.omega, p.h0, p.viscosity, p.dt), h, u, v, 200)
    assert rc == 0
    for q, (ref, tol) in enumerate(((rh, TOL), (ru, 1e-4), (rv, 1e-4))):
        assert rel_l2(out[q], ref) < tol, q


def test_reuse_and_sync_stay_clean(gpu):
    s = _mixed(127)
    x = torch.from_numpy(random_spec(127, 20, seed=7)).cuda()
    first = s.SH_to_spat(x)
    for _ in range(5):
        again = s.SH_to_spat(x)
    _sync_ok(s)
    assert torch.equal(first, again)


_GEN_SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from oracle import oracle as O
from sph_swe_b200 import capi
from sph_swe_b200.sph import Sph
from tests.helpers import random_spec, rel_l2
L, nb = 127, 20
s, g = Sph(L, precision=capi.SPH_PREC_MIXED), O.Grid(L)
spec = random_spec(L, nb, seed=3)
ref = g.SH_to_spat(spec)
out = s.SH_to_spat(torch.from_numpy(spec).cuda()).cpu().numpy()
back = s.spat_to_SH(torch.from_numpy(ref).cuda()).cpu().numpy()
assert capi.lib().sph_sync(s.h, None) == 0
ana = g.spat_to_SH(ref)
print(max(rel_l2(out[b], ref[b]) for b in range(nb)), max(rel_l2(back[b], ana[b]) for b in range(nb)))
"""


def test_checkpoint_generator_path_vs_oracle(gpu):
    """The P operand regenerated on the CUDA cores from recurrence checkpoints
    (SPH_TC_STREAM=0) instead of streamed from the split tables."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, SPH_TC_STREAM="0", PYTHONPATH=root)
    r = subprocess.run([sys.executable, "-c", _GEN_SCRIPT, root], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    syn, ana = (float(x) for x in r.stdout.split()[-2:])
    assert syn < TOL and ana < TOL


def _plm_at(mu_north, T):
    import scipy.special as sp

    th = np.arccos(np.asarray(mu_north))
    cache = {}

    def P(m):
        if m not in cache:
            cache[m] = np.nan_to_num(np.array([sp.sph_harm_y(l, m, th, 0.0).real for l in range(m, T + 1)]))
        return cache[m]

    return P


@pytest.mark.parametrize("L,nb", [(31, 3), (63, 5), (127, 17), (255, 40)])
@pytest.mark.parametrize("variant", [0, 128])
def test_int8_legendre_matches_integer_split_model(gpu, oracle_mod, L, nb, variant):
    """The Legendre stages of the mixed form (int8 kernels: B prepared by a
    separate kernel and loaded by the TMA unit, the default, or staged by
    producer warps, variant 128) carry out the arithmetic of the integer-split
    model (oracle/intsplit.py) given P at the handle's own Gauss nodes: the same
    row and column exponents, digits and exact integer group sums, so the
    results agree far below the form's own error (the model's P comes from
    scipy, the kernel's from its FP64 recurrence, so a digit may differ in the
    last place), and both are within 2e-8 of the FP64 oracle."""
    from oracle import intsplit

    s = _mixed(L)
    if variant:
        s.tune_load({"lmax": L, "nphi": s.nphi,
                     "kernels": [{"kind": k, "batch": nb, "variant": variant} for k in (0, 1)]})
    g = oracle_mod.Grid(L)
    nh = s.nlat // 2
    P = _plm_at(s.mu[:nh], L + 1)  # the handle's tables reach degree L + 1
    spec = random_spec(L, nb, seed=40 + L)
    four = torch.empty(nb, L + 1, s.nlat, dtype=torch.complex128, device="cuda")
    s.legendre_synthesis(torch.from_numpy(spec).cuda(), four)
    _sync_ok(s)
    Fm, gmax = intsplit.synthesis(P, nh, s.nlat, L, spec, 4)
    assert gmax < 2 ** 31
    got = four.cpu().numpy()
    assert rel_l2(got, Fm) < 1e-11
    grid = g.SH_to_spat(spec)
    F = (2 * np.pi / s.nphi) * np.fft.fft(grid, axis=1)[:, : L + 1, :]
    out = torch.empty(nb, s.nlm, dtype=torch.complex128, device="cuda")
    s.legendre_analysis(torch.from_numpy(np.ascontiguousarray(F)).cuda(), out)
    _sync_ok(s)
    sm, gmax = intsplit.analysis(P, nh, s.nlat, L, F, np.asarray(s.w), 4)
    assert gmax < 2 ** 31
    assert rel_l2(out.cpu().numpy(), sm) < 1e-11
    assert rel_l2(out.cpu().numpy(), g.spat_to_SH(grid)) < 2e-8


@pytest.mark.parametrize("L,nb", [(63, 8), (255, 20)])
def test_split_tf32_variant_vs_oracle(gpu, oracle_mod, L, nb):
    """The split-TF32 kernels stay selectable (autotuner variants 33-35: P by
    TMA, B staged by producer warps) and within relL2 1e-6 of the oracle for
    scalar transforms."""
    s = _mixed(L)
    g = oracle_mod.Grid(L)
    s.tune_load({"lmax": L, "nphi": s.nphi, "kernels": [{"kind": k, "batch": nb, "variant": 33} for k in (0, 1)]})
    spec = random_spec(L, nb, seed=300 + L)
    ref = g.SH_to_spat(spec)
    out = s.SH_to_spat(torch.from_numpy(spec).cuda()).cpu().numpy()
    back = s.spat_to_SH(torch.from_numpy(ref).cuda()).cpu().numpy()
    _sync_ok(s)
    ana = g.spat_to_SH(ref)
    for b in range(nb):
        assert rel_l2(out[b], ref[b]) < TOL
        assert rel_l2(back[b], ana[b]) < TOL

