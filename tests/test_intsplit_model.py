"""The integer-split (Ozaki) model of the Legendre contractions
(oracle/intsplit.py), the arithmetic of the library's kind::i8 tensor-core
kernels, against the FP64 oracle: with 4 balanced signed digits and 4 product
groups (10 int8 products) the synthesis of spectra with (l+1)^-1.5 decay is
within 2e-8 relative L2 of FP64 and the analysis within 5e-9 (the split-TF32
form reaches 2.6e-7), with 3 groups within 5e-6; every exact integer group sum
stays inside int32, and the kernels' digit word (v + 0x808080) ^ 0x808080
holds exactly the balanced digits."""
import numpy as np
import pytest
import scipy.special as sp

from oracle import intsplit
from tests.helpers import random_spec, rel_l2


def _plm(g, T):
    nh = g.nlat // 2
    th = np.arccos(np.asarray(g.mu)[:nh])
    cache = {}

    def P(m):
        if m not in cache:
            cache[m] = np.nan_to_num(np.array([sp.sph_harm_y(l, m, th, 0.0).real for l in range(m, T + 1)]))
        return cache[m]

    return P, nh


@pytest.mark.parametrize("L", [31, 63])
def test_intsplit_synthesis_accuracy(oracle_mod, L):
    g = oracle_mod.Grid(L)
    assert np.all(np.diff(np.asarray(g.mu)) < 0)  # northern latitudes first
    P, nh = _plm(g, L + 1)  # the library's tables reach degree L + 1
    spec = random_spec(L, 4, seed=L + 3)
    ref = g.SH_to_spat(spec)  # [b][nphi][nlat]
    for G, tol in ((4, 2e-8), (3, 5e-6)):
        F, gmax = intsplit.synthesis(P, nh, g.nlat, L, spec, G)
        assert gmax < 2 ** 31
        # longitude synthesis of F as the library's ring stage does it
        nphi = g.nphi
        lam = 2 * np.pi * np.arange(nphi) / nphi
        ms = np.arange(L + 1)
        E = np.exp(1j * np.outer(lam, ms))  # nphi x (L+1)
        w = np.where(ms == 0, 1.0, 2.0)
        grid = np.einsum("pm,bmj->bpj", E * w, F).real
        assert rel_l2(grid, ref) < tol, (G, rel_l2(grid, ref))


def test_intsplit_matmul_is_exact_integer_arithmetic():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((40, 300)) * np.exp(rng.uniform(-20, 5, (40, 1)))
    B = rng.standard_normal((300, 6))
    C, gmax = intsplit.matmul(A, B, 7)  # every digit product kept: only v's rounding remains
    assert gmax < 2 ** 31
    assert rel_l2(C, A @ B) < 1e-8
    C4, _ = intsplit.matmul(A, B, 4)
    assert rel_l2(C4, A @ B) < 1e-8


def test_digit_word_holds_the_balanced_digits():
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-1, 1, 20000) * (128 / 129), [0.0, 128 / 129 - 1e-12, -(128 / 129) + 1e-12]])
    e = np.zeros(1, np.int64)
    d = intsplit.digits(x[:, None], e, 1)
    assert all(np.all((q >= -128) & (q <= 127)) for q in d)
    v = np.rint(x * 2.0 ** 31).astype(np.int64)
    assert np.array_equal(d[0][:, 0] * 2 ** 24 + d[1][:, 0] * 2 ** 16 + d[2][:, 0] * 2 ** 8 + d[3][:, 0], v)
    w = intsplit.digit_word(v)
    as_i8 = lambda b: ((b.astype(np.int64) + 128) & 255) - 128
    for k, s in enumerate((24, 16, 8, 0)):
        assert np.array_equal(as_i8((w >> s) & 255), d[k][:, 0])


@pytest.mark.parametrize("L", [31, 63])
def test_intsplit_analysis_accuracy(oracle_mod, L):
    g = oracle_mod.Grid(L)
    P, nh = _plm(g, L + 1)
    spec = random_spec(L, 3, seed=L + 5)
    grid = g.SH_to_spat(spec)
    ref = g.spat_to_SH(grid)
    nphi = g.nphi
    F = (2 * np.pi / nphi) * np.fft.fft(grid, axis=1)[:, : L + 1, :]  # [b][m][j]
    out, gmax = intsplit.analysis(P, nh, g.nlat, L, F, np.asarray(g.w), 4)
    assert gmax < 2 ** 31
    assert rel_l2(out, ref) < 5e-9, rel_l2(out, ref)
