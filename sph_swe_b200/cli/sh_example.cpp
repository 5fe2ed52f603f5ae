// sh_example: the reference's command-line driver (main.cpp:37-210, AppSWE.hpp)
// on top of libsphgpu.so through the C++ class surface of sph_swe.hpp.
//
//   sh_example T<n> P0 N<0|1> M<rexiM> H<h> I<halfpoles> X<added modes> R<dt> S<robert>
//              Q<scenario> E<tend> V<visc> O<outdt> F<omega> W<M> [K<precision>] [C<file>] [D<file>]
//   sh_example <n> [<m> [<nlon> <nlat>]] <flags...>
//
// Same single-letter flags and defaults as the reference (SimVars.hpp:14-79);
// as in the reference, a trailing T<k> after the first argument is ignored.
// New values and letters: N2 selects the full nonlinear equations in
// vorticity-divergence form with Robert velocities on the grid (the reference
// has no such form; the state is then h, vorticity, divergence), K selects the
// precision form (0 FP64, 1 mixed), C<file> resumes from a checkpoint written
// by D<file>, and D<file>
// writes the final spectral state [h | u | v] (complex128, packed layout) to a
// file.  Programs: P0 (shallow-water run); the reference's test programs
// P1..P5 are not part of this driver.
// Scenarios: Q0 the reference's Gaussian bump (AppSWE.hpp:99-128), Q1 the
// Galewsky barotropic jet with its height bump (BenchmarkGalewsky.hpp:18-243:
// zonal jet between pi/7 and pi/2 - pi/7, depth in gradient-wind balance
// integrated ring by ring with the reference's area mean), Q10 the 500 m bump
// at (30N, 60E) with sigma = 0.1 a of the plain-method configuration.  With
// Robert variables the velocity state is U, V = u cos(phi), v cos(phi); with N2
// it is the vorticity and divergence.
// Output as the reference's AppSWE::write_output (AppSWE.hpp:60-95): at t = 0,
// every O seconds of simulated time and at the end, the grids of h, u, v and
// the vorticity as CSV files prog_{h,u,v,eta}_t<hours>.csv (longitude 0 in the
// middle for Q0); with N2: prog_h, prog_eta (vorticity), prog_div.  O <= 0
// means every half hour.
#include <sph_swe/sph_swe.hpp>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <iostream>
#include <vector>
#include <string>

using namespace sph_swe;

namespace {

struct Vars {
    int n = -1, m = -1, nlon = 0, nlat = 0;
    int program = 0;
    int nonlinear = 1;
    int rexi_M = 128;
    bool use_rexi = false;
    double rexi_h = 0.2;
    bool half_poles = true;
    double dt = 0.0;
    int robert = 0;
    int scenario = 0;
    double tend = -1.0;
    double visc = 1e5;
    double out_dt = 0.2;
    double omega = 7.292e-5;
    double gravity = 9.80616;
    double radius = 6.37122e6;
    double h0 = 10000.0;
    int precision = SPH_PREC_FP64;
    int rexi_ext = 0;  // X<k>: REXI at truncation L + k (rexi_use_extended_modes)
    std::string dump;
    std::string resume;
};

int parse(int argc, char** argv, Vars& v) {
    if (argc < 2) {
        std::cerr << "Usage: " << argv[0] << " T[n] [flags]\n   OR: " << argv[0] << " [n] [m] [nlon nlat] [flags]\n";
        return -1;
    }
    int first_flag = 2;
    if (argv[1][0] == 'T') {
        v.n = v.m = std::atoi(argv[1] + 1);
    } else {
        v.n = std::atoi(argv[1]);
        v.m = v.n;
        int i = 2;
        if (argc > i && std::isdigit((unsigned char)argv[i][0])) v.m = std::atoi(argv[i++]);
        if (argc > i + 1 && std::isdigit((unsigned char)argv[i][0]) && std::isdigit((unsigned char)argv[i + 1][0])) {
            v.nlon = std::atoi(argv[i++]);
            v.nlat = std::atoi(argv[i++]);
        }
        first_flag = i;
    }
    for (int i = first_flag; i < argc; i++) {
        const char* a = argv[i] + 1;
        switch (argv[i][0]) {
            case 'F': v.omega = std::atof(a); break;
            case 'P': v.program = std::atoi(a); break;
            case 'N': v.nonlinear = std::atoi(a); break;
            case 'M': v.rexi_M = std::atoi(a); v.use_rexi = v.rexi_M > 0; break;
            case 'H': v.rexi_h = std::atof(a); break;
            case 'I': v.half_poles = std::atoi(a) != 0; break;
            case 'R': v.dt = std::atof(a); break;
            case 'S': v.robert = std::atoi(a); break;
            case 'Q': v.scenario = std::atoi(a); break;
            case 'E': v.tend = std::atof(a); break;
            case 'V': v.visc = std::atof(a); break;
            case 'O': v.out_dt = std::atof(a); break;
            case 'W': v.rexi_M = std::atoi(a); break;
            case 'K': v.precision = std::atoi(a); break;
            case 'X': v.rexi_ext = std::atoi(a); break;
            case 'D': v.dump = a; break;
            case 'C': v.resume = a; break;
            default: break;  // unknown letters (and a trailing T<k>) are ignored, as in the reference
        }
    }
    return 0;
}

// Gauss-Legendre rule of n points on [-1, 1] (Newton on P_n)
void gauss_rule(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int k = 0; k < (n + 1) / 2; k++) {
        double z = std::cos(M_PI * (k + 0.75) / (n + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int i = 2; i <= n; i++) {
                const double p2 = ((2.0 * i - 1.0) * z * p1 - (i - 1.0) * p0) / i;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-15) break;
        }
        x[k] = -z;
        x[n - 1 - k] = z;
        w[k] = w[n - 1 - k] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// depth on the rings lat[j] (j = 0 north) in gradient-wind balance with the
// zonal flow u(phi): g dh/dphi = -a u (2 Omega sin(phi) + u tan(phi) / a),
// integrated from the south pole ring by ring (24-point Gauss rule per
// interval) and shifted to the area mean h_avg with the reference's
// ring-interval area terms (BenchmarkGalewsky.hpp:101-218)
std::vector<double> balanced_height(const double* lat, int nlat, const std::function<double(double)>& u, double a,
                                    double g, double om, double h_avg) {
    std::vector<double> gx, gw;
    gauss_rule(24, gx, gw);
    auto integ = [&](double lo, double hi) {
        const double mid = 0.5 * (lo + hi), half = 0.5 * (hi - lo);
        double sum = 0.0;
        for (int i = 0; i < 24; i++) {
            const double phi = mid + half * gx[i], uu = u(phi);
            sum += gw[i] * a * uu * (2.0 * om * std::sin(phi) + std::tan(phi) / a * uu);
        }
        return half * sum;
    };
    std::vector<double> edges;
    edges.push_back(-0.5 * M_PI);
    for (int j = nlat - 1; j >= 0; j--) edges.push_back(lat[j]);
    edges.push_back(0.5 * M_PI);
    std::vector<double> hg(edges.size() - 1);
    double acc = 0.0, hsum = 0.0, area = 0.0;
    for (size_t k = 0; k + 1 < edges.size(); k++) {
        acc -= integ(edges[k], edges[k + 1]);
        hg[k] = acc;
        const double mterm = (std::sin(edges[k + 1]) - std::sin(edges[k])) * 2.0 * M_PI;
        hsum += hg[k] * mterm;
        area += mterm;
    }
    const double shift = h_avg - hsum / g / area;
    std::vector<double> h(nlat);
    for (int j = 0; j < nlat; j++) h[j] = hg[nlat - 1 - j] / g + shift;
    return h;
}

void initial_state(const Vars& v, SPHConfig& cfg, SPHData& h, SPHData& u, SPHData& w) {
    if (v.scenario == 1) {
        // BenchmarkGalewsky.hpp:18-36 (constants), 59-71 (jet), 221-229 (bump)
        const double phi0 = M_PI / 7.0, phi1 = 0.5 * M_PI - phi0, umax = 80.0;
        const double en = std::exp(-4.0 / ((phi1 - phi0) * (phi1 - phi0)));
        auto ujet = [&](double phi) {
            return (phi <= phi0 || phi >= phi1) ? 0.0 : umax / en * std::exp(1.0 / ((phi - phi0) * (phi - phi1)));
        };
        const std::vector<double> hr =
            balanced_height(cfg.lat, cfg.spat_num_lat, ujet, v.radius, v.gravity, v.omega, v.h0);
        const double phi2 = M_PI / 4.0, alpha = 1.0 / 3.0, beta = 1.0 / 15.0, hhat = 120.0;
        std::vector<double> hg((size_t)cfg.spat_num_elems), ug((size_t)cfg.spat_num_elems);
        for (int i = 0; i < cfg.spat_num_lon; i++) {
            const double lam = 2.0 * M_PI * i / cfg.spat_num_lon;
            for (int j = 0; j < cfg.spat_num_lat; j++) {
                const double phi = cfg.lat[j];
                const size_t k = (size_t)i * cfg.spat_num_lat + j;
                hg[k] = hr[j] + hhat * std::cos(phi) * std::exp(-std::pow((lam - M_PI) / alpha, 2.0)) *
                                    std::exp(-std::pow((phi2 - phi) / beta, 2.0));
                // the reference stores the jet itself in prog_u also in the Robert
                // form (AppSWE.hpp:199-206); only the vorticity-divergence form
                // (N2) takes the Robert velocity u cos(phi) for its vector analysis
                ug[k] = ujet(phi) * (v.nonlinear == 2 ? std::cos(phi) : 1.0);
            }
        }
        h.spat_from_host(hg);
        u.spat_from_host(ug);
        w.spat_set_zero();
        if (v.nonlinear == 2) {
            // vorticity-divergence state from the Robert velocities (exact vector analysis)
            SPHData z(&cfg), d(&cfg);
            u.request_data_physical();
            w.request_data_physical();
            check(sph_vec_spat_to_SH(cfg.handle(), u.data_spat, w.data_spat, reinterpret_cast<double*>(z.data_spec),
                                     reinterpret_cast<double*>(d.data_spec), 1, 1, cfg.s()),
                  "sph_vec_spat_to_SH");
            z.mark_spectral();
            d.mark_spectral();
            u = z * (1.0 / v.radius);
            w = d * (1.0 / v.radius);
        }
        return;
    }
    if (v.scenario == 10) {
        const double lat0 = M_PI / 6.0, lon0 = M_PI / 3.0;
        h.spat_update_lambda_gaussian_grid([&](double lon, double mu, double& o) {
            const double phi = std::asin(mu);
            const double c = std::sin(phi) * std::sin(lat0) + std::cos(phi) * std::cos(lat0) * std::cos(lon - lon0);
            const double d = std::acos(std::fmax(-1.0, std::fmin(1.0, c)));
            o = v.h0 + 500.0 * std::exp(-(d / 0.1) * (d / 0.1));
        });
    } else {
        // AppSWE::setup_initial_conditions_gaussian (AppSWE.hpp:99-128)
        const double clat = M_PI / 3.0, clon = M_PI / 3.0, fac = 10.0;
        h.spat_update_lambda_gaussian_grid([&](double lon, double mu, double& o) {
            const double phi = std::asin(mu);
            const double d = std::acos(std::sin(phi) * std::sin(clat) + std::cos(phi) * std::cos(clat) * std::cos(lon - clon));
            o = std::exp(-d * d * fac) * 0.1 * v.h0 + v.h0;
        });
    }
    u.spat_set_zero();
    w.spat_set_zero();
}

}  // namespace

int main(int argc, char** argv) {
    Vars v;
    if (parse(argc, argv, v)) return 1;
    if (v.program != 0) {
        std::cerr << "program P" << v.program << " (reference test program) is not part of this driver\n";
        return 1;
    }
    if (v.dt <= 0.0 || v.tend <= 0.0) {
        std::cerr << "need a time step R<dt> > 0 and an end time E<t> > 0\n";
        return 1;
    }
    try {
        SPHConfig cfg;
        int nphi = v.nlon, nlat = v.nlat;
        if (nphi > 0 && nlat > 0)
            cfg.setup(v.m, v.n, nphi, nlat, v.precision);
        else
            cfg.setupAutoPhysicalSpace(v.m, v.n, &nphi, &nlat, v.precision);
        std::printf("Using T=%d on %d x %d (nlat x nphi), precision %s\n", v.n, nlat, nphi,
                    v.precision == SPH_PREC_MIXED ? "mixed" : "fp64");
        std::printf(" + gravity %g, radius %g, h0 %g, omega %g, viscosity %g, nonlinear %d, robert %d\n", v.gravity,
                    v.radius, v.h0, v.omega, v.visc, v.nonlinear, v.robert);
        std::printf(" + scenario %d, dt %g, end %g, REXI %d (M %d, h %g, half %d)\n", v.scenario, v.dt, v.tend,
                    (int)v.use_rexi, v.rexi_M, v.rexi_h, (int)v.half_poles);

        SPHData h(&cfg), u(&cfg), w(&cfg);
        if (!v.resume.empty()) {
            // checkpoint written by D<file>: the three spectral fields, packed layout
            std::ifstream f(v.resume, std::ios::binary);
            std::vector<cplx> buf((size_t)cfg.spec_num_elems);
            for (SPHData* x : {&h, &u, &w}) {
                f.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)(buf.size() * sizeof(cplx)));
                if (!f) throw std::runtime_error("checkpoint " + v.resume + " does not hold T" + std::to_string(v.n) +
                                                 " spectra of [h | u | v]");
                x->spec_from_host(buf);
            }
            std::printf(" + resumed from %s\n", v.resume.c_str());
        } else {
            initial_state(v, cfg, h, u, w);
        }
        h.request_data_spectral();
        u.request_data_spectral();
        w.request_data_spectral();

        SWEParameters p;
        p.earth_radius = v.radius;
        p.gravitation = v.gravity;
        p.coriolis_omega = v.omega;
        p.h0 = v.h0;
        p.viscosity2 = v.visc;
        p.use_nonlinear_equations = v.nonlinear != 0;
        p.use_robert_functions = v.robert != 0;
        p.use_vort_div_form = v.nonlinear == 2;

        const long long nsteps = (long long)std::llround(v.tend / v.dt);
        const double out_dt = v.out_dt > 0.0 ? v.out_dt : 1800.0;
        double next_out = 0.0;
        // AppSWE::write_output (AppSWE.hpp:60-95)
        auto write_output = [&](double t) {
            char name[128];
            const bool shifted = v.scenario == 0;
            auto put = [&](const char* field, const SPHData& x, const char* title) {
                std::snprintf(name, sizeof name, "prog_%s_t%020.8f.csv", field, t / 3600.0);
                x.spat_write_file(name, title, 8, shifted);
                return std::string(name);
            };
            const std::string fh = put("h", h, "");
            std::printf("%s (min: %g, max: %g)\n", fh.c_str(), h.spat_reduce_min(), h.spat_reduce_max());
            if (v.nonlinear == 2) {
                std::printf("%s\n", put("eta", u, "vorticity").c_str());
                std::printf("%s\n", put("div", w, "divergence").c_str());
            } else {
                std::printf("%s\n", put("u", u, "").c_str());
                std::printf("%s\n", put("v", w, "").c_str());
                const SPHData eta = SPHOperators::vort(u, w) * (1.0 / v.radius);
                std::printf("%s\n", put("eta", eta, shifted ? "vorticity, lon pi shifted" : "").c_str());
            }
        };
        // steps until the next output time (as the reference: output when t >= next_out)
        auto steps_to_output = [&](long long done) {
            const double t = done * v.dt;
            if (t >= next_out) {
                write_output(t);
                next_out += out_dt;
                if (next_out < t) next_out = t;
            }
            const long long k = (long long)std::ceil((next_out - t) / v.dt - 1e-9);
            return std::max<long long>(1, std::min(k, nsteps - done));
        };
        const auto t0 = std::chrono::steady_clock::now();
        long long done = 0;
        if (v.use_rexi) {
            if (v.nonlinear) throw std::runtime_error("REXI integrates the linear equations (N0)");
            REXI rexi;
            rexi.setup(v.rexi_h, v.rexi_M, 0, v.half_poles);
            std::printf(" + REXI poles: %zu\n", rexi.alpha.size());
            if (v.rexi_ext > 0) {
                // AppSWE.hpp:338-350, 434-445, 524-535: every step copies the state up to
                // truncation L + X, integrates there and copies it back down
                SPHConfig cfg_ext;
                cfg_ext.setupAdditionalModes(&cfg, v.rexi_ext, v.rexi_ext, v.precision);
                std::printf(" + REXI additional modes: %d (T%d on %d x %d)\n", v.rexi_ext, cfg_ext.spec_n_max,
                            cfg_ext.spat_num_lat, cfg_ext.spat_num_lon);
                // SWERexiSPH (S0) or SWERexiSPHRobert (S1) for every pole (AppSWE.hpp:368-414)
                SWERexi stepper(&cfg_ext, p, rexi, v.dt, v.robert != 0, false, v.precision);
                SPHData he(&cfg_ext), ue(&cfg_ext), we(&cfg_ext);
                while (done < nsteps) {
                    const long long k = steps_to_output(done);
                    for (long long i = 0; i < k; i++) {
                        h.spec_copyToDifferentModes(he);
                        u.spec_copyToDifferentModes(ue);
                        w.spec_copyToDifferentModes(we);
                        stepper.run(he, ue, we, 1);
                        he.spec_copyToDifferentModes(h);
                        ue.spec_copyToDifferentModes(u);
                        we.spec_copyToDifferentModes(w);
                    }
                    done += k;
                }
            } else {
                SWERexi stepper(&cfg, p, rexi, v.dt, v.robert != 0, false, v.precision);
                while (done < nsteps) {
                    const long long k = steps_to_output(done);
                    stepper.run(h, u, w, (int)k);
                    done += k;
                }
            }
        } else {
            SWERK4 stepper(&cfg, p);
            while (done < nsteps) {
                const long long k = steps_to_output(done);
                stepper.run(h, u, w, v.dt, (int)k);
                done += k;
            }
        }
        write_output(done * v.dt);
        cuda_check(cudaDeviceSynchronize(), "sync");
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("steps %lld  wall %.3f s  (%.1f steps/s incl. output)\n", done, secs, done / secs);
        if (!v.dump.empty()) {
            std::ofstream f(v.dump, std::ios::binary);
            for (const SPHData* x : {&h, &u, &w}) {
                const auto s = x->spec_to_host();
                f.write(reinterpret_cast<const char*>(s.data()), (std::streamsize)(s.size() * sizeof(cplx)));
            }
            std::printf("state written to %s\n", v.dump.c_str());
        }
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 2;
    }
    return 0;
}
