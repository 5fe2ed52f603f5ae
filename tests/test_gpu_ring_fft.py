"""Longitude stage (ring FFTs) of the transforms at every compile-time ring
length of the automatic grids (96 ... 3072) against numpy's FFT.

The Legendre stage is the same on both sides (sph_legendre_synthesis /
sph_legendre_analysis feed numpy), so the comparison isolates the ring
kernels: the FFT passes, the two-rings-per-complex-sequence packing, the
radix-3 stage fused with the tile load (analysis) or store (synthesis), and
the masks of never-written Fourier rows.  pad = 1 gives the grid an odd
leading dimension, which takes the 8-byte path instead of 16-byte chunks.
"""
import numpy as np
import pytest
import torch

from tests.helpers import random_spec, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [31, 63, 127, 255, 511, 1023])
@pytest.mark.parametrize("pad", [0, 1])
def test_ring_stage_vs_numpy(gpu, L, pad):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph, _ptr, _stream

    s = Sph(L)
    nb = 2
    N, nlat, nspat = s.nphi, s.nlat, s.nphi * s.nlat
    assert N == 3 * (L + 1)
    ld = nspat + pad
    spec = torch.from_numpy(random_spec(L, nb, seed=L + pad)).cuda()
    four = torch.empty(nb, L + 1, nlat, dtype=torch.complex128, device="cuda")
    s.legendre_synthesis(spec, four)
    F = four.cpu().numpy()
    # grid = Re F_0 + sum_{m >= 1} 2 Re(F_m e^{i m lambda})
    X = np.zeros((nb, N, nlat), complex)
    X[:, 0, :] = F[:, 0, :].real
    X[:, 1 : L + 1, :] = 2.0 * F[:, 1:, :]
    ref = (N * np.fft.ifft(X, axis=1)).real

    buf = torch.zeros(nb * ld, dtype=torch.float64, device="cuda")
    capi.check(capi.lib().sph_SH_to_spat(s.h, _ptr(spec), _ptr(buf), nb, 0, ld, _stream()))
    got = np.stack([buf[b * ld : b * ld + nspat].cpu().numpy().reshape(N, nlat) for b in range(nb)])
    assert rel_l2(got, ref) < 1e-13

    # analysis: spectra of the same grid through numpy's FFT and the library's
    grid = torch.from_numpy(ref).cuda()
    for b in range(nb):
        buf[b * ld : b * ld + nspat] = grid[b].reshape(-1)
    out = torch.empty(nb, s.nlm, dtype=torch.complex128, device="cuda")
    capi.check(capi.lib().sph_spat_to_SH(s.h, _ptr(buf), _ptr(out), nb, ld, 0, _stream()))
    Fn = (2.0 * np.pi / N) * np.fft.fft(ref, axis=1)[:, : L + 1, :]
    want = torch.empty_like(out)
    s.legendre_analysis(torch.from_numpy(np.ascontiguousarray(Fn)).cuda(), want)
    assert rel_l2(out.cpu().numpy(), want.cpu().numpy()) < 1e-13
