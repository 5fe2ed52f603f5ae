// sh_example: the reference's command-line driver (main.cpp:37-210, AppSWE.hpp)
// on top of libsphgpu.so through the C++ class surface of sph_swe.hpp.
//
//   sh_example T<n> P0 N<0|1> M<rexiM> H<h> I<halfpoles> R<dt> S<robert>
//              Q<scenario> E<tend> V<visc> O<outdt> F<omega> W<M> [K<precision>] [D<file>]
//   sh_example <n> [<m> [<nlon> <nlat>]] <flags...>
//
// Same single-letter flags and defaults as the reference (SimVars.hpp:14-79);
// as in the reference, a trailing T<k> after the first argument is ignored.
// New values and letters: N2 selects the full nonlinear equations in
// vorticity-divergence form with Robert velocities on the grid (the reference
// has no such form; the state is then h, vorticity, divergence), K selects the
// precision form (0 FP64, 1 mixed) and D<file>
// writes the final spectral state [h | u | v] (complex128, packed layout) to a
// file.  Programs: P0 (shallow-water run); the reference's test programs
// P1..P5 are not part of this driver.
// Scenarios: Q0 the reference's Gaussian bump (AppSWE.hpp:99-128), Q10 the
// 500 m bump at (30N, 60E) with sigma = 0.1 a of the plain-method configuration.
// Initial velocities are zero; with Robert variables the state is U, V.
#include <sph_swe/sph_swe.hpp>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
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
    std::string dump;
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
            case 'D': v.dump = a; break;
            default: break;  // unknown letters (and a trailing T<k>) are ignored, as in the reference
        }
    }
    return 0;
}

void initial_state(const Vars& v, SPHData& h, SPHData& u, SPHData& w) {
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
        initial_state(v, h, u, w);
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
        const long long out_every = v.out_dt > 0.0 ? std::max<long long>(1, std::llround(v.out_dt / v.dt)) : nsteps;
        const auto t0 = std::chrono::steady_clock::now();
        long long done = 0;
        if (v.use_rexi) {
            if (!v.robert) throw std::runtime_error("REXI needs the Robert formulation (S1)");
            if (v.nonlinear) throw std::runtime_error("REXI integrates the linear equations (N0)");
            REXI rexi;
            rexi.setup(v.rexi_h, v.rexi_M, 0, v.half_poles);
            std::printf(" + REXI poles: %zu\n", rexi.alpha.size());
            SWERexiRobert stepper(&cfg, p, rexi, v.dt, false, v.precision);
            while (done < nsteps) {
                const int k = (int)std::min(out_every, nsteps - done);
                stepper.run(h, u, w, k);
                done += k;
                std::printf("t = %g  h in [%.6f, %.6f]\n", done * v.dt, h.spat_reduce_min(), h.spat_reduce_max());
            }
        } else {
            SWERK4 stepper(&cfg, p);
            while (done < nsteps) {
                const int k = (int)std::min(out_every, nsteps - done);
                stepper.run(h, u, w, v.dt, k);
                done += k;
                std::printf("t = %g  h in [%.6f, %.6f]\n", done * v.dt, h.spat_reduce_min(), h.spat_reduce_max());
            }
        }
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
