// Host-only shim around sph_swe_b200/csrc/rexi_tables.h for the CPU unit test
// of the REXI band-matrix assembly (compiled by tests/test_rexi_host.py).
#include "../sph_swe_b200/csrc/rexi_tables.h"
#include "../sph_swe_b200/csrc/rexi_lane.h"

#include <cstring>
#include <vector>

using namespace sphgpu;

// Host run of rexi_lane (the per-pole arithmetic of the CUDA kernel) for one
// pole over all m-blocks.  Tables and vectors in the kernel's layouts:
// cphi [4][nc][5], cvel [nc][3], coef [nc][4], V [18][nc] (complex, block rows).
// out: [3][nc] complex, unscaled phi, u, v.  Returns 0, or 1 on a zero pivot.
extern "C" int shim_rexi_pole(int L, int coriolis, double r, double T, double P, double a_re, double a_im,
                              const double* cphi, const double* cvel, const double* coef, const double* V,
                              double* out) {
    const int nc = (L + 1) * (L + 1);
    RexiDev d{};
    d.L = L;
    d.npoles = 1;
    d.ngroups = 1;
    d.ncplx = nc;
    d.coriolis = coriolis;
    d.r = r;
    d.ir = 1.0 / r;
    d.T = T;
    d.P = P;
    d.Cphi = reinterpret_cast<const double2*>(cphi);
    d.Cvel = reinterpret_cast<const double2*>(cvel);
    d.coef = coef;
    d.V = reinterpret_cast<const double2*>(V);
    std::vector<double2> phi(L + 1), ra(L + 1), rb(L + 1);
    double2* o = reinterpret_cast<double2*>(out);
    int rc = 0;
    for (int m = -L; m <= L; m++) {
        const bool ok = rexi_lane<512>(d, m, make_double2(a_re, a_im), phi.data(), ra.data(), rb.data());
        if (!ok) rc = 1;
        const int base = block_off(L, m), N = L + 1 - (m < 0 ? -m : m);
        for (int i = 0; i < N; i++) {
            o[base + i] = phi[i];
            o[nc + base + i] = ra[i];
            o[2 * nc + base + i] = rb[i];
        }
    }
    return rc;
}

// The same pole with the banded systems factored once into stored planes
// (rexi_factor_lane) and solved from them (rexi_lane<.., STORED>), as the
// CUDA kernels do when the factors are kept between steps.
extern "C" int shim_rexi_pole_stored(int L, int coriolis, double r, double T, double P, double a_re, double a_im,
                                     const double* cphi, const double* cvel, const double* coef, const double* V,
                                     double* out) {
    const int nc = (L + 1) * (L + 1);
    RexiDev d{};
    d.L = L;
    d.npoles = 1;
    d.ngroups = 1;
    d.ncplx = nc;
    d.coriolis = coriolis;
    d.r = r;
    d.ir = 1.0 / r;
    d.T = T;
    d.P = P;
    d.Cphi = reinterpret_cast<const double2*>(cphi);
    d.Cvel = reinterpret_cast<const double2*>(cvel);
    d.coef = coef;
    d.V = reinterpret_cast<const double2*>(V);
    std::vector<double2> fphi((size_t)7 * nc), fvel((size_t)4 * nc);
    std::vector<signed char> pphi(nc, -1), pvel(nc, -1);
    d.fphi = fphi.data();
    d.pphi = pphi.data();
    d.fvel = fvel.data();
    d.pvel = pvel.data();
    d.plane = nc;
    d.lanes = 1;
    const double2 a = make_double2(a_re, a_im);
    int rc = 0;
    for (int m = -L; m <= L; m++)
        if (coriolis && !rexi_factor_lane(d, m, a, 0)) rc = 1;
    // every row of every block has its pivot offset (0..H) written exactly once
    for (int i = 0; i < nc && coriolis; i++)
        if (pphi[i] < 0 || pphi[i] > 2 || pvel[i] < 0 || pvel[i] > 1) rc = 2;
    std::vector<double2> phi(L + 1), ra(L + 1), rb(L + 1);
    double2* o = reinterpret_cast<double2*>(out);
    for (int m = -L; m <= L; m++) {
        rexi_lane<512, false, true>(d, m, a, phi.data(), ra.data(), rb.data(), 0);
        const int base = block_off(L, m), N = L + 1 - (m < 0 ? -m : m);
        for (int i = 0; i < N; i++) {
            o[base + i] = phi[i];
            o[nc + base + i] = ra[i];
            o[2 * nc + base + i] = rb[i];
        }
    }
    return rc;
}

extern "C" int shim_block_row(int L, int n, int m) { return brow(L, n, m); }

// comp: 2 z2, 3 z3, 4 z4robert, 5 z5robert, 6 z6robert, 7 z7, 8 z8; out: ncplx*5 complex
extern "C" void shim_component(int L, int comp, double s_re, double s_im, double r, int fix, double* out) {
    BandTable t(L);
    const cd s(s_re, s_im);
    switch (comp) {
        case 2: comp_z2(t, s); break;
        case 3: comp_z3(t, s); break;
        case 4: comp_z4robert(t, s, r); break;
        case 5: comp_z5robert(t, s, r, fix != 0); break;
        case 6: comp_z6robert(t, s, r); break;
        case 7: comp_z7(t, s, r); break;
        case 8: comp_z8(t, s, r); break;
        case 14: comp_z4(t, s, r); break;
        case 15: comp_z5(t, s, r); break;
        case 16: comp_z6(t, s, r); break;
        default: break;
    }
    std::memcpy(out, (const void*)t.a.data(), sizeof(cd) * t.a.size());
}
