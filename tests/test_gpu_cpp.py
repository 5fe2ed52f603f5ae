"""The C++ class surface (include/sph_swe/sph_swe.hpp) and the sh_example
driver against the oracle: operators of SPHData / SPHOperators through a
compiled C++ program, and shallow-water runs of sh_example (RK4 and REXI)
compared with the oracle's runs of the same configuration."""
import os
import subprocess

import numpy as np
import pytest

from tests.helpers import bump_state, random_spec, rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sph_swe_b200")


@pytest.fixture(scope="module")
def classes_bin(gpu, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "classes_check")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "classes_check.cpp"), "-o", out, "-L", PKG, "-lsphgpu",
           "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + PKG, "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True)
    return out


@pytest.mark.parametrize("L", [31, 63])
def test_class_operators_match_oracle(classes_bin, oracle_mod, tmp_path, L):
    g = oracle_mod.Grid(L)
    x, y = random_spec(L, 2, seed=40 + L)
    inp = tmp_path / "in.bin"
    np.concatenate([x, y]).astype(np.complex128).tofile(inp)
    outp = tmp_path / "out.bin"
    r = subprocess.run([classes_bin, str(L), str(inp), str(outp)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nphi, nlat, nlm, ncplx = map(int, r.stdout.split()[:4])
    assert (nphi, nlat, nlm) == (g.nphi, g.nlat, g.nlm)
    raw = np.fromfile(outp, np.uint8)
    kinds = "sssssgggsssgsss" + "s" + "gggss"
    blocks, off = [], 0
    for k in kinds:
        n = nlm * 16 if k == "s" else nphi * nlat * 8
        blocks.append(raw[off:off + n].view(np.complex128 if k == "s" else np.float64))
        off += n
    assert off == raw.size
    ref = {}
    for i, op in enumerate(["diff_lon", "d1mu2", "mu", "mu2", "laplace", "grad_lon", "grad_lat", "div_lat", "mul123",
                            "add100"]):
        ref[i] = g.real_op(op, x, kind="spec")[1]
    for i in range(10):
        b = blocks[i] if kinds[i] == "s" else blocks[i].reshape(nphi, nlat)
        assert rel_l2(b, ref[i]) < 1e-12, i
    assert rel_l2(blocks[10], x - y) < 1e-14
    assert rel_l2(blocks[11].reshape(nphi, nlat), g.SH_to_spat(x) * g.SH_to_spat(y)) < 1e-12
    n = np.concatenate([np.arange(m, L + 1) for m in range(L + 1)])
    assert rel_l2(blocks[12], x / (1.5 - 2.0e-3 / 9.0 * n * (n + 1))) < 1e-14
    # vort = F(grad_lon(y)) - F(grad_lat(x)), div = F(grad_lon(x)) + F(div_lat(y))
    vort = g.spat_to_SH(g.real_op("grad_lon", y, kind="spec")[1]) - g.spat_to_SH(g.real_op("grad_lat", x, kind="spec")[1])
    div = g.spat_to_SH(g.real_op("grad_lon", x, kind="spec")[1]) + g.spat_to_SH(g.real_op("div_lat", y, kind="spec")[1])
    assert rel_l2(blocks[13], vort) < 1e-12
    assert rel_l2(blocks[14], div) < 1e-12
    assert rel_l2(blocks[15], g.spat_to_SH(g.grid_from(lambda lon, mu: mu * np.cos(lon) + 2.0))) < 1e-13
    assert "nan 0" in r.stdout


def _run_cli(args, tmp_path):
    dump = tmp_path / "state.bin"
    r = subprocess.run([os.path.join(PKG, "sh_example"), *args, f"D{dump}"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.fromfile(dump, np.complex128), r.stdout


def _read_csv(path):
    """the reference's CSV layout: three '#T' lines, a longitude row led by 0, rows of latitude + values"""
    lines = open(path).read().splitlines()
    assert lines[0].startswith("#TI") and lines[1] == "#TX Longitude" and lines[2] == "#TY Latitude"
    rows = [np.array(l.split("\t"), float) for l in lines[3:]]
    lon = rows[0][1:]
    assert rows[0][0] == 0
    lat = np.array([r[0] for r in rows[1:]])
    vals = np.array([r[1:] for r in rows[1:]])
    return lon, lat, vals


def test_sh_example_rk4_matches_oracle(gpu, oracle_mod, tmp_path):
    """sh_example T31 P0 N1 R120 E2400 Q10 (reference defaults otherwise: a = 6.37122e6,
    viscosity 1e5), 20 RK4 steps; a trailing T<k> is ignored as in the reference."""
    st, out = _run_cli(["T31", "P0", "N1", "R120", "E2400", "O1e9", "Q10", "T99"], tmp_path)
    assert "Using T=31 on 48 x 96" in out
    g = oracle_mod.Grid(31)
    h = g.spat_to_SH(bump_state(g))
    z = np.zeros(g.nlm, complex)
    rh, ru, rv, rc = g.swe_run((6.37122e6, 9.80616, 7.292e-5, 1e4, 1e5, 120.0), h, z, z, 20)
    assert rc == 0
    for q, ref in enumerate((rh, ru, rv)):
        assert rel_l2(st[q * g.nlm:(q + 1) * g.nlm], ref) < 1e-10, q


@pytest.mark.parametrize("robert", [1, 0])
def test_sh_example_rexi_matches_oracle(gpu, oracle_mod, tmp_path, robert):
    """sh_example T31 P0 N0 S<robert> M64 H0.2 I0 R3600 E7200 Q10: REXI in the
    Robert (S1, SWERexiSPHRobert) or non-Robert (S0, SWERexiSPH) form, full pole set."""
    st, out = _run_cli(["T31", "P0", "N0", f"S{robert}", "M64", "H0.2", "I0", "R3600", "E7200", "O1e9", "Q10"],
                       tmp_path)
    assert "REXI poles: 151" in out
    g = oracle_mod.Grid(31)
    h = g.spat_to_SH(bump_state(g))
    z = np.zeros(g.nlm, complex)
    rh, ru, rv, npol = g.rexi_run((6.37122e6, 9.80616, 7.292e-5, 1e4, 1e5, 3600.0), h, z, z, 2, rexi_h=0.2, rexi_M=64,
                                  half=False, robert=robert)
    for q, ref in enumerate((rh, ru, rv)):
        assert rel_l2(st[q * g.nlm:(q + 1) * g.nlm], ref) < 1e-10, q


def test_sh_example_rexi_extended_modes_matches_oracle(gpu, oracle_mod, tmp_path):
    """sh_example ... X2: every REXI step runs at T33 on its own grid, the state
    copied up (zero-padded) before and truncated to T31 after it
    (rexi_use_extended_modes, AppSWE.hpp:338-350, 434-445, 524-535)."""
    st, out = _run_cli(["T31", "P0", "N0", "S1", "M64", "H0.2", "I0", "X2", "R3600", "E7200", "O1e9", "Q10"], tmp_path)
    assert "REXI additional modes: 2 (T33" in out
    g, ge = oracle_mod.Grid(31), oracle_mod.Grid(33)
    pairs = [(g.idx(n, m), ge.idx(n, m)) for m in range(32) for n in range(m, 32)]
    small, big = (np.array(x) for x in zip(*pairs))
    state = [g.spat_to_SH(bump_state(g)), np.zeros(g.nlm, complex), np.zeros(g.nlm, complex)]
    for _ in range(2):
        ext = []
        for q in range(3):
            e = np.zeros(ge.nlm, complex)
            e[big] = state[q][small]
            ext.append(e)
        rh, ru, rv, _ = ge.rexi_run((6.37122e6, 9.80616, 7.292e-5, 1e4, 1e5, 3600.0), *ext, 1, rexi_h=0.2, rexi_M=64,
                                    half=False, robert=1)
        for q, r in enumerate((rh, ru, rv)):
            state[q] = np.zeros(g.nlm, complex)
            state[q][small] = r[big]
    for q in range(3):
        assert rel_l2(st[q * g.nlm:(q + 1) * g.nlm], state[q]) < 1e-10, q


def test_sh_example_writes_reference_csv(gpu, oracle_mod, tmp_path):
    """Output as AppSWE::write_output: files at t = 0, every O seconds and at the
    end, in the reference's CSV layout; the final h grid equals the synthesis of
    the dumped spectral state."""
    st, out = _run_cli(["T31", "P0", "N1", "R120", "E1200", "O600", "Q10"], tmp_path)
    names = sorted(p.name for p in tmp_path.glob("prog_*.csv"))
    hours = sorted({n.split("_t")[1][:-4] for n in names})
    np.testing.assert_allclose([float(x) for x in hours], [0.0, 600 / 3600, 1200 / 3600], atol=1e-8)
    assert len(names) == 4 * len(hours)
    g = oracle_mod.Grid(31)
    lon, lat, vals = _read_csv(tmp_path / f"prog_h_t{1200 / 3600:020.8f}.csv")
    assert vals.shape == (g.nlat, g.nphi)
    np.testing.assert_allclose(lon, np.arange(g.nphi) * 360.0 / g.nphi, rtol=1e-7)
    np.testing.assert_allclose(lat, np.degrees(np.asarray(g.lat))[::-1], rtol=1e-7)
    grid = g.SH_to_spat(st[:g.nlm])  # (nphi, nlat), ring j = 0 north
    np.testing.assert_allclose(vals, grid[:, ::-1].T, rtol=1e-7)


def test_sh_example_galewsky(gpu, tmp_path):
    """Q1 (BenchmarkGalewsky.hpp): balanced jet with its bump, Robert RK4 and the
    vorticity-divergence form, a few steps, finite and mass-conserving in N2."""
    for args in (["T63", "P0", "N1", "S1", "R60", "E600", "O1e9", "V0", "Q1"],
                 ["T63", "P0", "N2", "R60", "E600", "O1e9", "V0", "Q1"]):
        st, out = _run_cli(args, tmp_path)
        assert np.all(np.isfinite(st)), args
        lon, lat, vals = _read_csv(tmp_path / f"prog_h_t{0:020.8f}.csv")
        assert 9000 < vals.min() < vals.max() < 11000


@pytest.mark.parametrize("robert", [0, 1])
def test_sh_example_galewsky_initial_state_matches_oracle(gpu, oracle_mod, tmp_path, robert):
    """Scenario Q1 (BenchmarkGalewsky.hpp:18-243) as sh_example sets it up: the
    balanced height, the bump and the jet (in prog_u in both forms, as
    AppSWE.hpp:199-206) against the oracle's restatement of BenchmarkGalewsky
    with adaptive quadrature (oracle/galewsky.py), compared as spectra.  R60
    E20 rounds to zero steps, so the checkpoint holds the initial state."""
    from oracle import galewsky as G

    st, out = _run_cli(["T63", "P0", "N1", f"S{robert}", "R60", "E20", "O1e9", "V0", "Q1"], tmp_path)
    g = oracle_mod.Grid(63)
    ho, uo, vo = G.initial_state(g.lat, g.nphi, 6.37122e6, 9.80616, 7.292e-5)
    n = g.nlm
    assert rel_l2(st[:n], g.spat_to_SH(ho)) < 1e-12
    assert rel_l2(st[n:2 * n], g.spat_to_SH(uo)) < 1e-12
    assert np.abs(st[2 * n:]).max() == 0.0


def test_sh_example_checkpoint_resume(gpu, tmp_path):
    """C<file> resumes from a D<file> dump: 5 + 5 steps equal 10 steps bitwise."""
    base = ["T31", "P0", "N1", "R120", "O1e9", "Q10"]
    full, _ = _run_cli(base + ["E1200"], tmp_path)
    half, _ = _run_cli(base + ["E600"], tmp_path)
    ck = tmp_path / "half.bin"
    half.tofile(ck)
    again, out = _run_cli(base + ["E600", f"C{ck}"], tmp_path)
    assert "resumed from" in out
    assert np.array_equal(again, full)
    bad = tmp_path / "short.bin"
    half[:10].tofile(bad)
    r = subprocess.run([os.path.join(PKG, "sh_example"), *base, "E600", f"C{bad}"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode != 0 and "checkpoint" in r.stderr


def test_sh_example_rejects_bad_usage(gpu):
    exe = os.path.join(PKG, "sh_example")
    assert subprocess.run([exe], capture_output=True).returncode != 0
    assert subprocess.run([exe, "T31", "P1", "R1", "E1"], capture_output=True).returncode != 0
    r = subprocess.run([exe, "T31", "P0", "N1", "S0", "M32", "R100", "E100"], capture_output=True, text=True)
    assert r.returncode != 0 and "linear" in r.stderr
