// Exercises the per-pole REXI classes SWERexiSPHRobert and SWERexiSPH of
// include/sph_swe/sph_swe.hpp the way AppSWE::run uses them (AppSWE.hpp:381-523):
// one object per pole, solve for (g h, u, v), sum over the poles, h = sum / g;
// and, for comparison, one step of SWERexi over all poles at once.
// argv: L, output file, form (1 Robert, the default; 0 non-Robert).  Writes
// h, u, v of the pole loop, then h, u, v of SWERexi (complex128, packed
// layout); prints nlm and the pole count.
#include <sph_swe/sph_swe.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

using namespace sph_swe;

static void put_spec(std::ofstream& f, const SPHData& x) {
    const auto v = x.spec_to_host();
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(cplx)));
}

int main(int argc, char** argv) {
    if (argc < 3) return 1;
    const int L = std::atoi(argv[1]);
    const bool robert = argc < 4 || std::atoi(argv[3]) != 0;
    try {
        SPHConfig cfg;
        cfg.setupAutoPhysicalSpace(L, L, nullptr, nullptr);
        SWEParameters p;
        p.earth_radius = 6.371e6;
        p.viscosity2 = 0.0;
        p.use_nonlinear_equations = false;
        p.use_robert_functions = robert;
        const double tau = 3600.0;
        // the 500 m bump at (30N, 60E), sigma = 0.1 a, on h0 = 1e4; rest state
        SPHData h(&cfg), u(&cfg), v(&cfg);
        const double lat0 = 30.0 * M_PI / 180.0, lon0 = 60.0 * M_PI / 180.0;
        h.spat_update_lambda_gaussian_grid([&](double lon, double mu, double& o) {
            const double ph = std::asin(mu);
            const double c = std::sin(ph) * std::sin(lat0) + std::cos(ph) * std::cos(lat0) * std::cos(lon - lon0);
            const double d = std::acos(std::max(-1.0, std::min(1.0, c)));
            o = 1e4 + 500.0 * std::exp(-(d / 0.1) * (d / 0.1));
        });
        u.spat_set_zero();
        v.spat_set_zero();
        REXI rexi;
        rexi.setup(0.2, 16, 0, false);
        std::printf("%d %zu\n", cfg.spec_num_elems, rexi.alpha.size());

        std::vector<SWERexiSPHRobert> rpoles(robert ? rexi.alpha.size() : 0);
        std::vector<SWERexiSPH> npoles(robert ? 0 : rexi.alpha.size());
        std::vector<SWERexiSPHPole*> poles;
        for (auto& q : rpoles) poles.push_back(&q);
        for (auto& q : npoles) poles.push_back(&q);
        for (size_t k = 0; k < poles.size(); k++)
            poles[k]->setup(&cfg, rexi.alpha[k], rexi.beta_re[k], p.earth_radius, p.coriolis_omega,
                            p.h0 * p.gravitation, tau);
        SPHOperatorsComplex op;
        const SPHData phi0 = h * p.gravitation;
        SPHData acc_phi(&cfg), acc_u(&cfg), acc_v(&cfg), t_phi, t_u, t_v;
        acc_phi.spec_set_zero();
        acc_u.spec_set_zero();
        acc_v.spec_set_zero();
        for (auto* pole : poles) {
            pole->solve(phi0, u, v, t_phi, t_u, t_v, op);
            acc_phi += t_phi;
            acc_u += t_u;
            acc_v += t_v;
        }
        std::ofstream out(argv[2], std::ios::binary);
        put_spec(out, acc_phi * (1.0 / p.gravitation));
        put_spec(out, acc_u);
        put_spec(out, acc_v);
        SWERexi all(&cfg, p, rexi, tau, robert);
        all.run(h, u, v, 1);
        put_spec(out, h);
        put_spec(out, u);
        put_spec(out, v);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    return 0;
}
