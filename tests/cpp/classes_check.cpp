// Exercises the C++ class surface of include/sph_swe/sph_swe.hpp: reads two
// spectral fields x, y (complex128, packed layout of degree L) from argv[2],
// applies the operators and writes their results (spectral: complex128 nlm;
// grid: double nphi*nlat) in a fixed order to argv[3].  tests/test_gpu_cpp.py
// compares every block with the oracle.
#include <sph_swe/sph_swe.hpp>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>

using namespace sph_swe;

static void put_spec(std::ofstream& f, const SPHData& x) {
    const auto v = x.spec_to_host();
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(cplx)));
}
static void put_spat(std::ofstream& f, const SPHData& x) {
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
        std::printf("%d %d %d %d\n", nphi, nlat, cfg.spec_num_elems, cfg.cplx_spec_num_elems);
        std::vector<cplx> hx(cfg.spec_num_elems), hy(cfg.spec_num_elems);
        {
            std::ifstream in(argv[2], std::ios::binary);
            in.read(reinterpret_cast<char*>(hx.data()), (std::streamsize)(hx.size() * sizeof(cplx)));
            in.read(reinterpret_cast<char*>(hy.data()), (std::streamsize)(hy.size() * sizeof(cplx)));
        }
        SPHData x(&cfg), y(&cfg);
        x.spec_update_lambda([&](int n, int m, cplx& o) { o = hx[cfg.getArrayIndexByModes(n, m)]; });
        y.spec_update_lambda([&](int n, int m, cplx& o) { o = hy[cfg.getArrayIndexByModes(n, m)]; });
        std::ofstream out(argv[3], std::ios::binary);
        put_spec(out, SPHOperators::diff_lon(x));                        // 0
        put_spec(out, SPHOperators::spec_one_minus_mu_squared_diff_lat_mu(x));  // 1
        put_spec(out, SPHOperators::mu(x));                              // 2
        put_spec(out, SPHOperators::mu2(x));                             // 3
        put_spec(out, SPHOperators::laplace(x));                         // 4
        put_spat(out, SPHOperators::grad_lon(x));                        // 5 grid
        put_spat(out, SPHOperators::grad_lat(x));                        // 6 grid
        put_spat(out, SPHOperators::div_lat(x));                         // 7 grid
        put_spec(out, x * 123.0);                                        // 8
        put_spec(out, x + 100.0);                                        // 9
        put_spec(out, x + y - y * 2.0);                                  // 10
        put_spat(out, x * y);                                            // 11 grid product
        put_spec(out, x.spec_solve_helmholtz(1.5, 2.0e-3, 3.0));        // 12
        put_spec(out, SPHOperators::vort(x, y));                         // 13
        put_spec(out, SPHOperators::div(x, y));                          // 14
        SPHData g(&cfg);
        g.spat_update_lambda_gaussian_grid([](double lon, double mu, double& o) { o = mu * std::cos(lon) + 2.0; });
        put_spec(out, g);                                                // 15
        put_spat(out, SPHOperators::diff_lat_mu(x));                     // 16 grid
        put_spat(out, SPHOperators::robert_div_lon(x));                  // 17 grid
        put_spat(out, SPHOperators::robert_div_lat(x));                  // 18 grid
        put_spec(out, SPHOperators::robert_grad_lat(x));                 // 19
        put_spec(out, SPHOperators::robert_grad_lon(x));                 // 20
        std::printf("nan %d absmax %.17g\n", (int)x.isAnyNaNorInf(), x.spat_reduce_abs_max());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    return 0;
}
