// Exercises SPHDataComplex / SPHOperatorsComplex of include/sph_swe/sph_swe.hpp:
// reads two complex spectra x, y (complex128, layout n*n+n+m, degree L) from
// argv[2], applies the operators and writes the results (spectral: complex128
// (L+1)^2; grid: complex128 nphi*nlat) in a fixed order to argv[3].
// tests/test_gpu_cpp.py compares every block with the oracle.
#include <sph_swe/sph_swe.hpp>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>

using namespace sph_swe;

static void put_spec(std::ofstream& f, const SPHDataComplex& x) {
    const auto v = x.spec_to_host();
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(cplx)));
}
static void put_spat(std::ofstream& f, const SPHDataComplex& x) {
    const auto v = x.spat_to_host();
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(cplx)));
}
static void put_real_spat(std::ofstream& f, const SPHData& x) {
    const auto v = x.spat_to_host();
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

int main(int argc, char** argv) {
    if (argc < 4) return 1;
    const int L = std::atoi(argv[1]);
    try {
        SPHConfig cfg;
        int nphi = 0, nlat = 0;
        cfg.setupAutoPhysicalSpace(L, L, &nphi, &nlat);
        std::printf("%d %d %d\n", nphi, nlat, cfg.cplx_spec_num_elems);
        std::vector<cplx> hx(cfg.cplx_spec_num_elems), hy(cfg.cplx_spec_num_elems);
        {
            std::ifstream in(argv[2], std::ios::binary);
            in.read(reinterpret_cast<char*>(hx.data()), (std::streamsize)(hx.size() * sizeof(cplx)));
            in.read(reinterpret_cast<char*>(hy.data()), (std::streamsize)(hy.size() * sizeof(cplx)));
        }
        SPHDataComplex x(&cfg), y(&cfg);
        x.spec_from_host(hx);
        y.spec_from_host(hy);
        using Op = SPHOperatorsComplex;
        std::ofstream out(argv[3], std::ios::binary);
        put_spec(out, Op::diff_lon(x));                                             // 0
        put_spec(out, Op::spec_one_minus_mu_squared_diff_lat_mu(x));                // 1
        put_spec(out, Op::mu(x));                                                   // 2
        put_spec(out, Op::mu2(x));                                                  // 3
        put_spec(out, Op::laplace(x));                                              // 4
        put_spat(out, Op::grad_lon(x));                                             // 5 grid
        put_spat(out, Op::grad_lat(x));                                             // 6 grid
        put_spat(out, Op::div_lat(x));                                              // 7 grid
        put_spec(out, x.spec_solve_helmholtz(cplx(1.5, 0.5), cplx(2.0e-3, 1.0e-3), 3.0));  // 8
        put_spec(out, Op::robert_vort(x, y));                                       // 9
        put_spat(out, Op::robert_div(x, y));                                        // 10 grid
        put_spat(out, Op::diff_lat_mu(x));                                          // 11 grid
        // real <-> complex through the grid (SPHDataComplex.hpp:93-175)
        SPHData re(&cfg), im(&cfg);
        x.spat_RealToSPHData(re);
        x.spat_ImagToSPHData(im);
        put_real_spat(out, re);                                                     // 12 real grid
        put_real_spat(out, im);                                                     // 13 real grid
        SPHDataComplex z(&cfg);
        z = re;
        put_spec(out, z);                                                           // 14
        SPHDataComplex w(&cfg);
        w.spat_fromSPHData(im);
        put_spat(out, w);                                                           // 15 grid
        SPHData q = re;
        q.request_data_spectral();
        q.data_spat_valid = false;  // spectral only: the conversion must synthesise
        const SPHDataComplex c(q);
        put_spat(out, c);                                                           // 16 grid
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    return 0;
}
