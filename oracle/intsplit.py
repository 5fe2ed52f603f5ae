"""TEST INFRASTRUCTURE ONLY (the oracle): numpy model of an integer-split
(Ozaki-scheme) evaluation of the Legendre contractions, the arithmetic of a
tensor-core form that keeps its sums exact in int32 instead of folding FP32
partial sums into FP64.

A dense product C = A B (A: rows x K, B: K x columns) is evaluated as
  1. every row i of A is scaled by 2^-ea_i and every column j of B by 2^-eb_j,
     powers of two chosen so that the scaled entries lie in [-1, 1);
  2. each scaled operand is cut into S slices of 7 bits: x = sum_s q_s 2^-7(s+1)
     with integers q_s in [-127, 127] (round to nearest, remainder carried to
     the next slice);
  3. the slice products q_s(A) q_t(B) with s + t < S are summed EXACTLY in
     integers, grouped by k = s + t (S groups);
  4. C_ij = 2^(ea_i + eb_j) sum_k 2^-7(k+2) G_k,ij in FP64.
Step 3 is exact as long as every group sum stays below 2^31 in magnitude
(int32 accumulators): |G_k| <= (k + 1) 127^2 K.

The Legendre synthesis of one order m and parity is such a product with
A = P_l^m(mu_j) (rows: northern latitudes j, K: degrees l of that parity) and
B = the spectra (columns: fields, real and imaginary parts); the analysis
uses A = P^T (rows: degrees) and B = the Gauss-weighted north +/- south
Fourier sums (K: latitudes).  `synthesis` below evaluates the whole real
synthesis of a batch of packed spectra this way, for comparison with the FP64
transforms.
"""
from __future__ import annotations

import numpy as np

BITS = 7
QMAX = 127


def split(M: np.ndarray, S: int, axis: int):
    """Power-of-two scaling along `axis` (1: per row, 0: per column) and S
    integer slices; returns (list of int64 arrays, exponents)."""
    mx = np.max(np.abs(M), axis=axis, keepdims=True)
    e = np.where(mx > 0, np.floor(np.log2(np.where(mx > 0, mx, 1.0))) + 1.0, 0.0)
    R = M * np.exp2(-e)
    out = []
    for s in range(S):
        q = np.clip(np.rint(R * 2.0 ** (BITS * (s + 1))), -QMAX, QMAX)
        out.append(q.astype(np.int64))
        R = R - q * 2.0 ** (-BITS * (s + 1))
    return out, e


def matmul(A: np.ndarray, B: np.ndarray, S: int):
    """C = A B by the integer split; also returns the largest |group sum| so
    that callers can check the int32 bound."""
    As, ea = split(A, S, 1)
    Bs, eb = split(B, S, 0)
    C = np.zeros((A.shape[0], B.shape[1]))
    gmax = 0
    for k in range(S):
        G = np.zeros((A.shape[0], B.shape[1]), np.int64)
        for s in range(k + 1):
            G += As[s] @ Bs[k - s]
        gmax = max(gmax, int(np.abs(G).max()) if G.size else 0)
        C += G.astype(np.float64) * 2.0 ** (-BITS * (k + 2))
    return C * np.exp2(ea) * np.exp2(eb), gmax


def synthesis(P, nh: int, nlat: int, L: int, spec: np.ndarray, S: int):
    """Fourier coefficients F[b][m][j] (j over all nlat latitudes, north first)
    of packed real spectra spec[b][nlm] of degree L.  P(m) returns the
    (L - m + 1) x nh array P_l^m(mu_j) of the northern latitudes.  Returns
    (F, largest group sum)."""
    nb = spec.shape[0]
    F = np.zeros((nb, L + 1, nlat), complex)
    gmax = 0
    for m in range(L + 1):
        Pm = P(m)
        base = m * (2 * L - m + 1) // 2 + m  # packed index of (l = m, m)
        x = spec[:, base: base + L - m + 1]  # [b][l - m]
        B = np.concatenate([x.real.T, x.imag.T], axis=1)  # K x 2 nb
        eo = []
        for par in (0, 1):
            A = Pm[par::2].T  # nh x K_par
            if A.shape[1] == 0:
                eo.append(np.zeros((nh, 2 * nb)))
                continue
            C, g = matmul(A, B[par::2], S)
            gmax = max(gmax, g)
            eo.append(C)
        north = eo[0] + eo[1]
        south = eo[0] - eo[1]
        F[:, m, :nh] = (north[:, :nb] + 1j * north[:, nb:]).T
        F[:, m, nlat - nh:] = (south[:, :nb] + 1j * south[:, nb:]).T[:, ::-1]
    return F, gmax


def analysis(P, nh: int, nlat: int, L: int, F: np.ndarray, w: np.ndarray, S: int):
    """Packed real spectra spec[b][nlm] from Fourier coefficients F[b][m][j]
    (analysis convention F_m = (2 pi / nphi) sum_i f e^{-i m lambda_i}) with
    the Gauss weights w[j] of the northern latitudes: per m and parity the
    product of P^T (rows: degrees) with the weighted north +/- south sums
    (K: latitudes).  Returns (spec, largest group sum)."""
    nb = F.shape[0]
    nlm = (L + 1) * (L + 2) // 2
    spec = np.zeros((nb, nlm), complex)
    gmax = 0
    for m in range(L + 1):
        Pm = P(m)
        north = F[:, m, :nh]
        south = F[:, m, nlat - nh:][:, ::-1]
        base = m * (2 * L - m + 1) // 2 + m
        for par in (0, 1):
            A = Pm[par::2]  # K_par x nh: rows are degrees l = m + par + 2k
            if A.shape[0] == 0:
                continue
            G = (north + south) if par == 0 else (north - south)
            G = G * w[None, :nh]
            B = np.concatenate([G.real.T, G.imag.T], axis=1)  # nh x 2 nb
            C, g = matmul(A, B, S)
            gmax = max(gmax, g)
            spec[:, base + par: base + L - m + 1: 2] = (C[:, :nb] + 1j * C[:, nb:]).T
    return spec, gmax
