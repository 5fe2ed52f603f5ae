"""TEST INFRASTRUCTURE ONLY (the oracle): numpy model of the integer-split
(Ozaki-scheme) Legendre contractions of the library's mixed-precision form,
the arithmetic of its tcgen05.mma kind::i8 kernels, so that the kernels can be
held to this model to the rounding of their final FP64 combination and the
model to the FP64 oracle.

A dense product C = A B (A: rows x K, B: K x columns) is evaluated as
  1. every row i of A is scaled by 2^-ea_i and every column j of B by 2^-eb_j,
     with ea, eb the binary (frexp) exponents of (1 + 2^-7) times the largest
     magnitude, so that the scaled entries a satisfy |a| < 128/129;
  2. each scaled entry is rounded to v = rint(a 2^31) and written in balanced
     base 256: v = d0 2^24 + d1 2^16 + d2 2^8 + d3 with every digit in
     [-128, 127] (the kernels form the four digits as the bytes of
     (v + 0x808080) ^ 0x808080), so a ~ d0 2^-7 + d1 2^-15 + d2 2^-23 + d3 2^-31
     (digit s weighs 2^-(7 + 8 s));
  3. the digit products d_s(A) d_t(B) with s + t < G are summed EXACTLY in
     integers, grouped by g = s + t (G int32 accumulators; the kernels issue one
     signed kind::i8 MMA per product).  The dropped products are zero-mean, so
     G = 4 (10 products) is within a factor of about two of keeping them all;
  4. C_ij = 2^(ea_i + eb_j - 14) (((G_0 + G_1 2^-8) + G_2 2^-16) + ...) in
     FP64, in that order.
Step 3 is exact while every group sum stays below 2^31 in magnitude:
|G_g| <= (g + 1) 128^2 K for the 4 digit planes.

The Legendre stages use it per order m and parity:
  synthesis  A = P_l^m(mu_j) (rows: northern latitudes j, K: degrees of the
             parity), B = the spectra (columns: fields x re/im); the row
             exponent of latitude j is taken over all degrees of order m up to
             the table degree (both parities), the column exponent over all
             degrees of the column (both parities);
  analysis   A = P_l^m(mu_j) w_j (rows: degrees, K: latitudes; the Gauss weight
             folded into the table), B = the north +/- south Fourier sums; the
             row exponent is the row's own, the column exponent that of
             max_j (|north_j| + |south_j|), which bounds both parities.
"""
from __future__ import annotations

import numpy as np

VBITS = 31


def exponents(M: np.ndarray, axis: int) -> np.ndarray:
    """frexp exponent of (1 + 2^-7) times the largest magnitude along `axis`
    (0 where all zero)."""
    mx = np.max(np.abs(M), axis=axis) if M.size else np.zeros(M.shape[1 - axis])
    return np.where(mx > 0, np.frexp(mx * (1.0 + 2.0 ** -7))[1], 0).astype(np.int64)


def digits(M: np.ndarray, e: np.ndarray, axis: int):
    """The four balanced digit planes d0..d3 (int64 arrays with values in
    [-128, 127]) of v = rint(M 2^-e 2^31), e broadcast along `axis` (1: one
    exponent per row, 0: one per column)."""
    k = (VBITS - (e[:, None] if axis == 1 else e[None, :])).astype(np.int64)
    # M 2^k in one step: 2^k alone overflows for rows of tiny magnitude
    v = np.rint(np.ldexp(M, np.broadcast_to(k, M.shape))).astype(np.int64)
    out = []
    for _ in range(3):
        d = ((v + 128) & 255) - 128
        out.append(d)
        v = (v - d) >> 8
    out.append(v)
    return out[::-1]


def digit_word(v: np.ndarray) -> np.ndarray:
    """The kernels' form of the four digits of int32 values v: the word
    (v + 0x808080) ^ 0x808080, whose bytes 3, 2, 1, 0 read as int8 are d0..d3."""
    w = (np.asarray(v, np.int64) + 0x808080) & 0xFFFFFFFF
    return (w ^ 0x808080).astype(np.uint32)


def matmul_scaled(A, ea, B, eb, groups: int = 4):
    """C = A B by the byte split with given row / column exponents; returns
    (C, largest |group sum|)."""
    Ad, Bd = digits(A, ea, 1), digits(B, eb, 0)
    acc = np.zeros((A.shape[0], B.shape[1]))
    gmax = 0
    for g in range(groups):
        G = np.zeros((A.shape[0], B.shape[1]), np.int64)
        for s in range(max(0, g - 3), min(g, 3) + 1):
            G += Ad[s] @ Bd[g - s]
        gmax = max(gmax, int(np.abs(G).max()) if G.size else 0)
        acc = acc + G.astype(np.float64) * 2.0 ** (-8 * g)
    return np.ldexp(acc, (ea[:, None] + eb[None, :] - 14).astype(np.int64)), gmax


def matmul(A, B, groups: int = 4):
    """C = A B with per-row / per-column exponents of A and B themselves."""
    return matmul_scaled(A, exponents(A, 1), B, exponents(B, 0), groups)


def synthesis(P, nh: int, nlat: int, L: int, spec: np.ndarray, groups: int = 4):
    """Fourier coefficients F[b][m][j] (all nlat latitudes, north first) of
    packed real spectra spec[b][nlm] of degree L.  P(m) returns the
    (T - m + 1) x nh array P_l^m(mu_j), l = m..T, of the northern latitudes,
    T >= L the degree of the library's table.  Returns (F, largest group sum)."""
    nb = spec.shape[0]
    F = np.zeros((nb, L + 1, nlat), complex)
    gmax = 0
    for m in range(L + 1):
        Pm = P(m)
        ea = exponents(Pm, 0)  # per latitude, over all degrees of the table
        base = m * (2 * L - m + 1) // 2 + m  # packed index of (l = m, m)
        x = spec[:, base: base + L - m + 1]  # [b][l - m]
        B = np.concatenate([x.real.T, x.imag.T], axis=1)  # K x 2 nb
        eb = exponents(B, 0)
        eo = []
        for par in (0, 1):
            A = Pm[par: L - m + 1: 2].T  # nh x K_par
            if A.shape[1] == 0:
                eo.append(np.zeros((nh, 2 * nb)))
                continue
            C, g = matmul_scaled(A, ea, B[par::2], eb, groups)
            gmax = max(gmax, g)
            eo.append(C)
        north = eo[0] + eo[1]
        south = eo[0] - eo[1]
        F[:, m, :nh] = (north[:, :nb] + 1j * north[:, nb:]).T
        F[:, m, nlat - nh:] = (south[:, :nb] + 1j * south[:, nb:]).T[:, ::-1]
    return F, gmax


def analysis(P, nh: int, nlat: int, L: int, F: np.ndarray, w: np.ndarray, groups: int = 4):
    """Packed real spectra spec[b][nlm] of degree L from Fourier coefficients
    F[b][m][j] (analysis convention F_m = (2 pi / nphi) sum_i f e^{-i m lambda_i})
    with the Gauss weights w[j] of the northern latitudes folded into the
    table.  Returns (spec, largest group sum)."""
    nb = F.shape[0]
    nlm = (L + 1) * (L + 2) // 2
    spec = np.zeros((nb, nlm), complex)
    gmax = 0
    for m in range(L + 1):
        Pw = P(m)[: L - m + 1] * w[None, :nh]
        north = F[:, m, :nh]
        south = F[:, m, nlat - nh:][:, ::-1]
        bound = np.concatenate([(np.abs(north.real) + np.abs(south.real)).T,
                                (np.abs(north.imag) + np.abs(south.imag)).T], axis=1)
        eb = exponents(bound, 0)
        base = m * (2 * L - m + 1) // 2 + m
        for par in (0, 1):
            A = Pw[par::2]  # K_par x nh: rows are degrees l = m + par + 2k
            if A.shape[0] == 0:
                continue
            G = (north + south) if par == 0 else (north - south)
            B = np.concatenate([G.real.T, G.imag.T], axis=1)  # nh x 2 nb
            C, g = matmul_scaled(A, exponents(A, 1), B, eb, groups)
            gmax = max(gmax, g)
            spec[:, base + par: base + L - m + 1: 2] = (C[:, :nb] + 1j * C[:, nb:]).T
    return spec, gmax

