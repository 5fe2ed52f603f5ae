// Host-side assembly of the pole-independent REXI band matrices and the
// N-compact block layout (shared by rexi.cu and its CPU unit test).
// Components follow SPHSolverComplex::solver_component_rexi_* with a unit
// scalar (SPHSolverComplex.hpp:88-420); rows store the five even offsets
// -4,-2,0,+2,+4 (index (offset+4)/2).
#pragma once

#include <complex>
#include <cstdlib>
#include <vector>

#include "identities.cuh"

namespace sphgpu {

using cd = std::complex<double>;

// N-compact row of (n, m): blocks m = -L..L contiguous, n = |m|..L (SPHConfig.hpp:136-156)
__host__ __device__ inline int block_off(int L, int m) {
    return m < 0 ? ((L + m) * (L + m + 1)) / 2 : (L * (L + 1)) / 2 + (m * (2 * L - m + 3)) / 2;
}
__host__ __device__ inline int brow(int L, int n, int m) { return block_off(L, m) + n - (m < 0 ? -m : m); }

// Components as SPHSolverComplex::solver_component_rexi_* with unit scalar;
// rows store the five even offsets -4,-2,0,+2,+4 (index (off+4)/2); entries that
// fall outside the m-block are dropped, as the band conversion of
// BandedMatrixSolver.hpp:346-368 drops them.
struct BandTable {
    int L, halo;
    std::vector<cd> a;  // [row][5]
    BandTable(int L_) : L(L_), a((size_t)(L_ + 1) * (L_ + 1) * 5) {}
    void add(int n, int m, int rel, cd v) {
        if (n < m) return;  // reference guard (SPHMatrixComplex.hpp:198)
        const int n2 = n + rel;
        const int am = m < 0 ? -m : m;
        if (n2 < 0 || n2 < am || n2 > L) return;
        if (rel & 1) return;  // odd offsets never occur in the REXI matrices
        a[(size_t)brow(L, n, m) * 5 + (rel + 4) / 2] += v;
    }
};

static void comp_z2(BandTable& t, cd s) {
    const int L = t.L;
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) {
            t.add(n, m, -2, s * idA(n - 2, m));
            t.add(n, m, 0, s * idB(n, m));
            t.add(n, m, +2, s * idC(n + 2, m));
        }
}
static void comp_z3(BandTable& t, cd s) {
    const int L = t.L;
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) {
            t.add(n, m, -4, s * (idA(n - 2, m) * idA(n - 4.0, m)));
            t.add(n, m, -2, s * (idA(n - 2, m) * idB(n - 2, m) + idB(n, m) * idA(n - 2, m)));
            t.add(n, m, 0, s * (idA(n - 2, m) * idC(n, m) + idB(n, m) * idB(n, m) + idC(n + 2, m) * idA(n, m)));
            t.add(n, m, +2, s * (idB(n, m) * idC(n + 2, m) + idC(n + 2, m) * idB(n + 2, m)));
            t.add(n, m, +4, s * (idC(n + 2, m) * idC(n + 4, m)));
        }
}
static void comp_z4robert(BandTable& t, cd s, double r) {
    const int L = t.L;
    for (int m = -L; m <= L; m++) {
        const cd fac = 1.0 / (r * r) * s * cd(0, m);
        for (int n = std::abs(m); n <= L; n++) {
            t.add(n, m, -2, -fac * idA(n - 2, m));
            t.add(n, m, 0, -fac * idB(n, m) + fac);
            t.add(n, m, +2, -fac * idC(n + 2, m));
        }
    }
}
static void comp_z5robert(BandTable& t, cd s, double r, bool fix) {
    const int L = t.L;
    const int o0 = fix ? -4 : -2, o2 = fix ? 0 : -2, o3 = fix ? 2 : -2, o4 = fix ? 4 : -2;
    for (int m = -L; m <= L; m++) {
        const cd fac = 1.0 / (r * r) * s * cd(0, m);
        for (int n = std::abs(m); n <= L; n++) {
            t.add(n, m, o0, -fac * (idA(n - 2, m) * idA(n - 4, m)));
            t.add(n, m, -2, -fac * (idA(n - 2, m) * idB(n - 2, m) + idB(n, m) * idA(n - 2, m)) + fac * idA(n - 2, m));
            t.add(n, m, o2, -fac * (idA(n - 2, m) * idC(n, m) + idB(n, m) * idB(n, m) + idC(n + 2, m) * idA(n, m)) +
                               fac * idB(n, m));
            t.add(n, m, o3, -fac * (idB(n, m) * idC(n + 2, m) + idC(n + 2, m) * idB(n + 2, m)) + fac * idC(n + 2, m));
            t.add(n, m, o4, -fac * (idC(n + 2, m) * idC(n + 4, m)));
        }
    }
}
static void comp_z6robert(BandTable& t, cd s_, double r) {
    const int L = t.L;
    for (int m = -L; m <= L; m++) {
        const cd s = 1.0 / (r * r) * s_ * (double)m;
        for (int n = std::abs(m); n <= L; n++) {
            const double gr = idG(n - 1, m) * idR(n - 2, m);
            const double gs = idG(n - 1, m) * idS(n, m) + idH(n + 1, m) * idR(n, m);
            const double hs = idH(n + 1, m) * idS(n + 2, m);
            t.add(n, m, -2, s * gr);
            t.add(n, m, 0, s * gs);
            t.add(n, m, +2, s * hs);
            t.add(n, m, -4, s * (-idA(n - 4, m) * gr));
            t.add(n, m, -2, s * (-idB(n - 2, m) * gr));
            t.add(n, m, 0, s * (-idC(n + 0, m) * gr));
            t.add(n, m, -2, s * (-idA(n - 2, m) * gs));
            t.add(n, m, 0, s * (-idB(n + 0, m) * gs));
            t.add(n, m, +2, s * (-idC(n + 2, m) * gs));
            t.add(n, m, 0, s * (-idA(n + 0, m) * hs));
            t.add(n, m, +2, s * (-idB(n + 2, m) * hs));
            t.add(n, m, +4, s * (-idC(n + 4, m) * hs));
        }
    }
}
// The non-Robert components of SWERexiSPH (SPHSolverComplex.hpp:221-234,
// 263-280, 319-335): z4 = grad_j(mu) grad_i(phi) is diagonal (i m / r^2),
// z5 = grad_j(mu) mu^2 grad_i(phi) is i m / r^2 times the mu^2 band, z6 =
// grad_j(mu) mu grad_j(phi) uses the D, E, R, S identities; all offsets even.
static void comp_z4(BandTable& t, cd s, double r) {
    const int L = t.L;
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) t.add(n, m, 0, 1.0 / (r * r) * s * cd(0, m));
}
static void comp_z5(BandTable& t, cd s, double r) {
    const int L = t.L;
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) {
            const cd fac = 1.0 / (r * r) * s * cd(0, m);
            t.add(n, m, -2, fac * idA(n - 2, m));
            t.add(n, m, 0, fac * idB(n + 0, m));
            t.add(n, m, +2, fac * idC(n + 2, m));
        }
}
static void comp_z6(BandTable& t, cd s, double r) {
    const int L = t.L;
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) {
            t.add(n, m, -2, -1.0 / (r * r) * s * (idD(n - 1, m) * idR(n - 2, m) + (idE(n, m) - 3.0) * idA(n - 2, m)));
            t.add(n, m, 0, -1.0 / (r * r) * s * (1.0 + idD(n - 1, m) * idS(n, m) + (idE(n, m) - 3.0) * idB(n, m)));
            t.add(n, m, +2, -1.0 / (r * r) * s * (idE(n, m) - 3.0) * idC(n + 2, m));
        }
}
static void comp_z7(BandTable& t, cd s, double r) {
    const int L = t.L;
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) t.add(n, m, 0, -1.0 / (r * r) * s * (double)n * ((double)n + 1.0));
}
static void comp_z8(BandTable& t, cd s, double r) {
    const int L = t.L;
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) {
            t.add(n, m, 0, 1.0 / (r * r) * s * 2.0);
            const double fac = -1.0 / (r * r) * ((double)m * m - (double)n * (n + 1.0));
            t.add(n, m, -2, s * fac * idA(n - 2, m));
            t.add(n, m, 0, s * fac * idB(n, m));
            t.add(n, m, +2, s * fac * idC(n + 2, m));
        }
}

}  // namespace sphgpu
