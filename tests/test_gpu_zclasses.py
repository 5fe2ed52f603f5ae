"""The later additions to the C++ class surface (include/sph_swe/sph_swe.hpp)
against the oracle: SPHOperatorsComplex, the per-pole REXI class
SWERexiSPHRobert, and the real-field SPHOperators additions (d/dmu and the
Robert-variable operators).  Kept in a file of their own, collected after the
other GPU tests."""
import os
import subprocess

import numpy as np
import pytest

from tests.helpers import bump_state, random_spec, rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sph_swe_b200")


def _compile(src, out):
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I",
                    "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", src), "-o", out, "-L", PKG,
                    "-lsphgpu", "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + PKG,
                    "-Wl,-rpath,/usr/local/cuda/lib64"], check=True)
    return out


def test_real_class_operator_additions_match_oracle(gpu, oracle_mod, tmp_path):
    """Blocks 16-20 of tests/cpp/classes_check.cpp: diff_lat_mu, robert_div_lon,
    robert_div_lat (grids), robert_grad_lat, robert_grad_lon (spectra)."""
    L = 31
    exe = _compile("classes_check.cpp", str(tmp_path / "classes_check"))
    g = oracle_mod.Grid(L)
    x, y = random_spec(L, 2, seed=40 + L)
    inp = tmp_path / "in.bin"
    np.concatenate([x, y]).astype(np.complex128).tofile(inp)
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, str(L), str(inp), str(outp)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nphi, nlat, nlm, _ = map(int, r.stdout.split()[:4])
    raw = np.fromfile(outp, np.uint8)
    blocks, off = [], 0
    for k in "sssssgggsssgsss" + "s" + "gggss":
        n = nlm * 16 if k == "s" else nphi * nlat * 8
        blocks.append(raw[off:off + n].view(np.complex128 if k == "s" else np.float64))
        off += n
    assert off == raw.size
    for i, op in zip((16, 17, 18), ("diff_lat_mu", "robert_div_lon", "robert_div_lat")):
        kind, ref = g.real_op(op, x, kind="spec")
        assert kind == "spat"
        assert rel_l2(blocks[i].reshape(nphi, nlat), ref) < 1e-12, op
    assert rel_l2(blocks[19], g.real_op("d1mu2", x, kind="spec")[1]) < 1e-12
    assert rel_l2(blocks[20], g.real_op("diff_lon", x, kind="spec")[1]) < 1e-12


@pytest.fixture(scope="module")
def classes_cplx_bin(gpu, tmp_path_factory):
    return _compile("classes_check_cplx.cpp", str(tmp_path_factory.mktemp("cppc") / "classes_check_cplx"))


def test_complex_class_operators_match_oracle(classes_cplx_bin, oracle_mod, tmp_path):
    """SPHDataComplex / SPHOperatorsComplex (SPHOperatorsComplex.hpp) against the
    oracle's complex operators; the compositions the oracle lacks (Helmholtz,
    robert_vort, robert_div, diff_lat_mu) against the same compositions of
    oracle pieces; the real <-> complex grid conversions (spat_RealToSPHData,
    spat_ImagToSPHData, spat_fromSPHData, assignment from SPHData) against the
    oracle's transforms of the parts."""
    L = 31
    g = oracle_mod.Grid(L)
    x, y = random_spec(L, 2, seed=77, cplx=True)
    inp = tmp_path / "in.bin"
    np.concatenate([x, y]).astype(np.complex128).tofile(inp)
    outp = tmp_path / "out.bin"
    r = subprocess.run([classes_cplx_bin, str(L), str(inp), str(outp)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nphi, nlat, ncplx = map(int, r.stdout.split()[:3])
    assert (nphi, nlat, ncplx) == (g.nphi, g.nlat, g.ncplx)
    kinds = "cccccgggccggrrcgg"
    raw = np.fromfile(outp, np.uint8)
    blocks, off = [], 0
    for k in kinds:
        n = ncplx if k == "c" else nphi * nlat
        dt = np.float64 if k == "r" else np.complex128
        v = raw[off:off + n * np.dtype(dt).itemsize].view(dt)
        blocks.append(v if k == "c" else v.reshape(nphi, nlat))
        off += n * np.dtype(dt).itemsize
    assert off == raw.size
    op = lambda name, v: g.cplx_op(name, v, kind="spec")[1]
    for i, name in enumerate(["diff_lon", "d1mu2", "mu", "mu2", "laplace", "grad_lon", "grad_lat", "div_lat"]):
        assert rel_l2(blocks[i], op(name, x)) < 1e-12, name
    n = np.concatenate([np.full(2 * l + 1, l) for l in range(L + 1)]).astype(float)
    a, b = 1.5 + 0.5j, (2.0e-3 + 1.0e-3j) / 9.0
    assert rel_l2(blocks[8], x / (a - b * n * (n + 1))) < 1e-14
    assert rel_l2(blocks[9], op("diff_lon", y) - op("d1mu2", x)) < 1e-13
    c2 = g.cosphi[None, :] ** 2
    assert rel_l2(blocks[10], g.cplx_SH_to_spat(op("diff_lon", x) + op("d1mu2", y)) / c2) < 1e-12
    assert rel_l2(blocks[11], g.cplx_SH_to_spat(op("d1mu2", x)) / c2) < 1e-12
    # real <-> complex through the grid: spat_RealToSPHData / spat_ImagToSPHData
    # copy the parts of the synthesised grid exactly, operator= and
    # spat_fromSPHData build (part, 0), and a spectral-only real field is
    # synthesised first
    gx = g.cplx_SH_to_spat(x)
    assert rel_l2(blocks[12], gx.real) < 1e-12
    assert rel_l2(blocks[13], gx.imag) < 1e-12
    assert rel_l2(blocks[14], g.cplx_spat_to_SH(gx.real.astype(complex))) < 1e-12
    assert np.array_equal(blocks[15].imag, np.zeros_like(blocks[13]))
    assert np.array_equal(blocks[15].real, blocks[13])
    assert np.array_equal(blocks[16].imag, np.zeros_like(blocks[12]))
    assert rel_l2(blocks[16].real, g.SH_to_spat(g.spat_to_SH(gx.real))) < 1e-12


@pytest.mark.parametrize("robert", [1, 0])
def test_per_pole_rexi_class_matches_oracle(gpu, oracle_mod, tmp_path, robert):
    """SWERexiSPHRobert (robert = 1) and SWERexiSPH (robert = 0) used as
    AppSWE::run uses them (one object per pole, solve, sum over the poles,
    divide by g) equal one SWERexi step over all poles and the oracle's REXI
    step of the same form (T31, M = 16, full pole set)."""
    exe = _compile("rexi_pole_check.cpp", str(tmp_path / "rexi_pole_check"))
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, "31", str(outp), str(robert)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nlm, npoles = map(int, r.stdout.split()[:2])
    assert npoles == 55
    loop, full = np.fromfile(outp, np.complex128).reshape(2, 3, nlm)
    g = oracle_mod.Grid(31)
    h = g.spat_to_SH(bump_state(g))
    z = np.zeros(g.nlm, complex)
    ref = g.rexi_run((6.371e6, 9.80616, 7.292e-5, 1e4, 0.0, 3600.0), h, z, z, 1, rexi_h=0.2, rexi_M=16, half=False,
                     robert=robert)[:3]
    for q in range(3):
        assert rel_l2(loop[q], full[q]) < 1e-12, q
        assert rel_l2(loop[q], ref[q]) < 1e-10, q
