"""Parity of the CUDA transforms and spectral operators (through the C ABI)
with the oracle.  Tolerance: relative L2 <= 1e-12 for FP64 transforms."""
import numpy as np
import pytest
import torch

from tests.helpers import ga_f, random_spec, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module", params=[31, 63, 127, 255])
def pair(request, gpu, oracle_mod):
    from sph_swe_b200.sph import Sph

    L = request.param
    return Sph(L), oracle_mod.Grid(L)


def test_grid_matches_oracle(pair):
    s, g = pair
    assert (s.nlat, s.nphi, s.nlm) == (g.nlat, g.nphi, g.nlm)
    # nodes converged to within rounding on both sides: at most 2 ulp apart
    assert np.abs(s.mu - g.mu).max() <= 4.5e-16
    assert np.abs(s.w - g.w).max() < 1e-15
    assert np.abs(s.cosphi - g.cosphi).max() <= 4.5e-16


def test_real_synthesis_and_analysis(pair):
    s, g = pair
    spec = random_spec(g.L, 5, seed=11)
    ref = g.SH_to_spat(spec)
    out = s.SH_to_spat(torch.from_numpy(spec).cuda()).cpu().numpy()
    assert rel_l2(out, ref) < TOL
    back = s.spat_to_SH(torch.from_numpy(ref).cuda()).cpu().numpy()
    assert rel_l2(back, g.spat_to_SH(ref)) < TOL
    assert rel_l2(back, spec) < TOL


def test_analysis_of_non_bandlimited_field(pair):
    s, g = pair
    f = g.grid_from(ga_f)
    out = s.spat_to_SH(torch.from_numpy(f).cuda()).cpu().numpy()
    assert rel_l2(out, g.spat_to_SH(f)) < TOL


def test_complex_transforms(pair):
    s, g = pair
    cs = random_spec(g.L, 3, seed=12, cplx=True)
    ref = g.cplx_SH_to_spat(cs)
    out = s.cplx_SH_to_spat(torch.from_numpy(cs).cuda()).cpu().numpy()
    assert rel_l2(out, ref) < TOL
    back = s.cplx_spat_to_SH(torch.from_numpy(ref).cuda()).cpu().numpy()
    assert rel_l2(back, g.cplx_spat_to_SH(ref)) < TOL


@pytest.mark.parametrize("op", ["diff_lon", "d1mu2", "mu", "mu2", "laplace"])
def test_spec_ops_real(pair, op):
    s, g = pair
    x = random_spec(g.L, 2, seed=13)
    out = s.spec_op(op, torch.from_numpy(x).cuda()).cpu().numpy()
    for b in range(2):
        kind, ref = g.real_op(op, x[b], kind="spec")
        assert kind == "spec"
        assert rel_l2(out[b], ref) < 1e-14


@pytest.mark.parametrize("op", ["diff_lon", "d1mu2", "mu", "mu2", "laplace"])
def test_spec_ops_complex(pair, op):
    s, g = pair
    x = random_spec(g.L, 1, seed=14, cplx=True)
    out = s.spec_op(op, torch.from_numpy(x).cuda(), cplx=True).cpu().numpy()
    kind, ref = g.cplx_op(op, x[0], kind="spec")
    assert rel_l2(out[0], ref) < 1e-14


def test_helmholtz_scale_axpy(pair):
    s, g = pair
    x = random_spec(g.L, 1, seed=15)
    xt = torch.from_numpy(x).cuda()
    a, b = 1.0 + 0.5j, 2.5e-3 - 1e-3j
    out = s.spec_op("helmholtz", xt, a=a, b=b).cpu().numpy()[0]
    n = np.concatenate([np.arange(m, g.L + 1) for m in range(g.L + 1)])
    assert rel_l2(out, x[0] / (a - b * n * (n + 1))) < 1e-14
    y = torch.zeros_like(xt)
    s.spec_op("axpy", xt, a=2.0 - 1j, out=y)
    assert rel_l2(y.cpu().numpy(), (2.0 - 1j) * x) < 1e-15


def test_batched_strides_and_large_batch(gpu, oracle_mod):
    from sph_swe_b200.sph import Sph

    s = Sph(63)
    g = oracle_mod.Grid(63)
    spec = random_spec(63, 40, seed=16)
    out = s.SH_to_spat(torch.from_numpy(spec).cuda()).cpu().numpy()
    assert rel_l2(out, g.SH_to_spat(spec)) < TOL


@pytest.mark.parametrize("L,nb", [(31, 17), (127, 37), (255, 64)])
def test_wide_batches_match_oracle(gpu, oracle_mod, L, nb):
    """Batches above 16 fields take several 16-field column blocks of the FP64
    tensor-core Legendre kernels: ragged and full column blocks, real, complex
    and vector."""
    from sph_swe_b200.sph import Sph

    s, g = Sph(L), oracle_mod.Grid(L)
    spec = random_spec(L, nb, seed=L + nb)
    ref = g.SH_to_spat(spec)
    out = s.SH_to_spat(torch.from_numpy(spec).cuda()).cpu().numpy()
    assert rel_l2(out, ref) < TOL
    back = s.spat_to_SH(torch.from_numpy(ref).cuda()).cpu().numpy()
    assert rel_l2(back, g.spat_to_SH(ref)) < TOL
    cs = random_spec(L, nb, seed=L + nb + 1, cplx=True)
    cref = g.cplx_SH_to_spat(cs)
    cout = s.cplx_SH_to_spat(torch.from_numpy(cs).cuda()).cpu().numpy()
    assert rel_l2(cout, cref) < TOL
    cback = s.cplx_spat_to_SH(torch.from_numpy(cref).cuda()).cpu().numpy()
    assert rel_l2(cback, g.cplx_spat_to_SH(cref)) < TOL
    vort = torch.from_numpy(spec).cuda()
    div = torch.from_numpy(random_spec(L, nb, seed=L + nb + 2)).cuda()
    vort[:, 0] = 0
    div[:, 0] = 0
    u, v = s.vec_SH_to_spat(vort, div)
    z, d = s.vec_spat_to_SH(u, v)
    # the vector round trip weights high degrees by n(n+1): 1.5e-12 .. 2e-12 at T255 (any kernel)
    assert rel_l2(z.cpu().numpy(), vort.cpu().numpy()) < 5e-12
    assert rel_l2(d.cpu().numpy(), div.cpu().numpy()) < 5e-12


def test_vector_roundtrip_and_divergence_free(gpu, oracle_mod):
    from sph_swe_b200.sph import Sph

    s = Sph(63)
    vort = torch.from_numpy(random_spec(63, 2, seed=17)).cuda()
    div = torch.from_numpy(random_spec(63, 2, seed=18)).cuda()
    vort[:, 0] = 0
    div[:, 0] = 0
    for robert in (False, True):
        u, v = s.vec_SH_to_spat(vort, div, robert=robert)
        z, d = s.vec_spat_to_SH(u, v, robert=robert)
        assert rel_l2(z.cpu().numpy(), vort.cpu().numpy()) < 1e-12
        assert rel_l2(d.cpu().numpy(), div.cpu().numpy()) < 1e-12
    # solid-body rotation u = cos(phi): vorticity 2 mu, no divergence
    g = oracle_mod.Grid(63)
    u = torch.from_numpy(np.broadcast_to(g.cosphi[None, :], (g.nphi, g.nlat)).copy()).cuda()
    v = torch.zeros_like(u)
    z, d = s.vec_spat_to_SH(u, v)
    ref = g.spat_to_SH(g.grid_from(lambda lon, mu: 2 * mu + 0 * lon))
    assert np.abs(z.cpu().numpy() - ref).max() < 1e-12
    assert np.abs(d.cpu().numpy()).max() < 1e-12


def test_bad_arguments_fail_loudly(gpu):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph
    import ctypes

    h = ctypes.c_void_p()
    assert capi.lib().sph_create(10, 11, 0, 0, 0, ctypes.byref(h)) == capi.SPH_ERR_ARG
    assert "lmax == mmax" in capi.last_error()
    assert capi.lib().sph_create(10, 10, 15, 32, 0, ctypes.byref(h)) == capi.SPH_ERR_ARG
    s = Sph(15)
    assert capi.lib().sph_spat_to_SH(s.h, None, None, 1, 0, 0, None) == capi.SPH_ERR_ARG
    x = torch.zeros(s.nlm, dtype=torch.complex128, device="cuda")
    with pytest.raises(capi.SphError):
        s.spec_op("mu", x, out=x)


def test_spec_copy_modes_between_truncations(gpu, oracle_mod):
    """sph_spec_copy_modes (SPHData::spec_copyToDifferentModes): T31 -> T33
    zero-pads, T33 -> T31 truncates, both exact."""
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    s31, s33 = Sph(31), Sph(33)
    g31, g33 = oracle_mod.Grid(31), oracle_mod.Grid(33)
    x = random_spec(31, 3, seed=41)
    up = s31.spec_copy_modes(torch.from_numpy(x).cuda(), s33).cpu().numpy()
    want = np.zeros((3, g33.nlm), complex)
    for m in range(32):
        for n in range(m, 32):
            want[:, g33.idx(n, m)] = x[:, g31.idx(n, m)]
    assert np.array_equal(up, want)
    y = random_spec(33, 2, seed=42)
    down = s33.spec_copy_modes(torch.from_numpy(y).cuda(), s31).cpu().numpy()
    want = np.array([[y[b, g33.idx(n, m)] for m in range(32) for n in range(m, 32)] for b in range(2)])
    order = [g31.idx(n, m) for m in range(32) for n in range(m, 32)]
    assert np.array_equal(down[:, order], want)
    t = torch.from_numpy(x).cuda()
    with pytest.raises(capi.SphError):
        capi.check(capi.lib().sph_spec_copy_modes(s31.h, t.data_ptr(), s31.h, t.data_ptr(), 3, None))
