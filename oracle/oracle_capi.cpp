// TEST INFRASTRUCTURE ONLY — C entry points of the oracle, loaded by the
// tests (ctypes), smoke() and the bench's cpu_baseline leg.  Never part of the
// product path.  Complex arrays are interleaved (re, im) doubles.
#include "sph_oracle.hpp"

#include <cstring>
#include <exception>
#include <memory>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

namespace {
inline cplx* C(double* p) { return reinterpret_cast<cplx*>(p); }
inline const cplx* C(const double* p) { return reinterpret_cast<const cplx*>(p); }

Field real_from_spat(const Grid* g, const double* spat) {
    Field f(g);
    std::memcpy(f.spat.data(), spat, sizeof(double) * g->nspat);
    f.spat_valid = true;
    return f;
}
Field real_from_spec(const Grid* g, const double* spec) {
    Field f(g);
    std::memcpy((void*)f.spec.data(), spec, sizeof(cplx) * g->nlm);
    f.spec_valid = true;
    return f;
}
CField cplx_from_spat(const Grid* g, const double* spat) {
    CField f(g);
    std::memcpy((void*)f.spat.data(), spat, sizeof(cplx) * g->nspat);
    f.spat_valid = true;
    return f;
}
CField cplx_from_spec(const Grid* g, const double* spec) {
    CField f(g);
    std::memcpy((void*)f.spec.data(), spec, sizeof(cplx) * g->ncplx);
    f.spec_valid = true;
    return f;
}
}  // namespace

extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void orc_auto_grid(int L, int* nlat, int* nphi) { auto_grid(L, nlat, nphi); }

void* orc_grid_new(int L, int nlat, int nphi) {
    try {
        Grid* g = new Grid();
        g->setup(L, nlat, nphi);
        return g;
    } catch (...) {
        return nullptr;
    }
}

void orc_grid_free(void* g) { delete static_cast<Grid*>(g); }

// out: L, nlat, nphi, nlm, ncplx
void orc_grid_info(const void* gp, int* out) {
    const Grid* g = static_cast<const Grid*>(gp);
    out[0] = g->L; out[1] = g->nlat; out[2] = g->nphi; out[3] = g->nlm; out[4] = g->ncplx;
}

void orc_grid_arrays(const void* gp, double* mu, double* w, double* cosphi, double* lat) {
    const Grid* g = static_cast<const Grid*>(gp);
    for (int j = 0; j < g->nlat; j++) { mu[j] = g->mu[j]; w[j] = g->w[j]; cosphi[j] = g->cosphi[j]; lat[j] = g->lat[j]; }
}

// P_l^m(mu_j), j < nlat/2; returns the value or NaN outside the table
double orc_plm(const void* gp, int l, int m, int j) {
    const Grid* g = static_cast<const Grid*>(gp);
    if (m < 0 || m > g->L + 1 || l < m || l > g->L + 1 || j < 0 || j >= g->nh) return __builtin_nan("");
    return g->P(l, m, j);
}

void orc_spat_to_SH(const void* gp, const double* spat, double* spec, int batch) {
    const Grid* g = static_cast<const Grid*>(gp);
    for (int b = 0; b < batch; b++) g->spat_to_SH(spat + (size_t)b * g->nspat, C(spec) + (size_t)b * g->nlm);
}

void orc_SH_to_spat(const void* gp, const double* spec, double* spat, int batch) {
    const Grid* g = static_cast<const Grid*>(gp);
    for (int b = 0; b < batch; b++) g->SH_to_spat(C(spec) + (size_t)b * g->nlm, spat + (size_t)b * g->nspat);
}

// degree-lmax variants (lmax = L or L+1), packed with (m*(2*lmax-m+1))/2+n
void orc_spat_to_SH_l(const void* gp, const double* spat, double* spec, int lmax) {
    const Grid* g = static_cast<const Grid*>(gp);
    g->spat_to_SH(spat, C(spec), lmax);
}
void orc_SH_to_spat_l(const void* gp, const double* spec, double* spat, int lmax) {
    const Grid* g = static_cast<const Grid*>(gp);
    g->SH_to_spat(C(spec), spat, lmax);
}

void orc_cplx_spat_to_SH(const void* gp, const double* spat, double* spec, int batch) {
    const Grid* g = static_cast<const Grid*>(gp);
    for (int b = 0; b < batch; b++) g->cplx_spat_to_SH(C(spat) + (size_t)b * g->nspat, C(spec) + (size_t)b * g->ncplx);
}

void orc_cplx_SH_to_spat(const void* gp, const double* spec, double* spat, int batch) {
    const Grid* g = static_cast<const Grid*>(gp);
    for (int b = 0; b < batch; b++) g->cplx_SH_to_spat(C(spec) + (size_t)b * g->ncplx, C(spat) + (size_t)b * g->nspat);
}

// Real operators, applied through the lazy field semantics.  in_kind: 0 grid
// input (nspat doubles), 1 spectral input (nlm complex).  Output is returned
// in the representation the operator leaves valid: *out_kind = 0 grid, 1 spec.
// op: 0 diff_lon, 1 (1-mu^2)d/dmu, 2 mu, 3 mu2, 4 laplace, 5 grad_lon,
//     6 grad_lat, 7 div_lat, 8 diff_lat_mu, 9 robert_div_lon, 10 robert_div_lat,
//     11 spec_truncate, 12 x*123, 13 x+100, 14 identity
int orc_real_op(const void* gp, int op, int in_kind, const double* in, double* out, int* out_kind) {
    const Grid* g = static_cast<const Grid*>(gp);
    try {
        Field x = in_kind == 0 ? real_from_spat(g, in) : real_from_spec(g, in);
        Field y(g);
        switch (op) {
            case 0: y = Ops::diff_lon(x); break;
            case 1: y = Ops::spec_one_minus_mu_squared_diff_lat_mu(x); break;
            case 2: y = Ops::mu(x); break;
            case 3: y = Ops::mu2(x); break;
            case 4: y = Ops::laplace(x); break;
            case 5: y = Ops::grad_lon(x); break;
            case 6: y = Ops::grad_lat(x); break;
            case 7: y = Ops::div_lat(x); break;
            case 8: y = Ops::diff_lat_mu(x); break;
            case 9: y = Ops::robert_div_lon(x); break;
            case 10: y = Ops::robert_div_lat(x); break;
            case 11: { x.request_spec(); Field t(g); g->SH_to_spat(x.spec.data(), t.spat.data()); t.spat_valid = true; t.request_spec(); y = t; break; }
            case 12: y = x * 123.0; break;
            case 13: y = x + 100.0; break;
            case 14: y = x; break;
            default: return 1;
        }
        if (y.spat_valid) { std::memcpy(out, y.spat.data(), sizeof(double) * g->nspat); *out_kind = 0; }
        else { std::memcpy(out, y.spec.data(), sizeof(cplx) * g->nlm); *out_kind = 1; }
        return 0;
    } catch (...) {
        return 2;
    }
}

// Complex operators, same conventions (grid: nspat complex, spec: ncplx complex).
// op: 0 diff_lon, 1 (1-mu^2)d/dmu, 2 mu, 3 mu2, 4 laplace, 5 grad_lon,
//     6 grad_lat, 7 div_lat, 14 identity
int orc_cplx_op(const void* gp, int op, int in_kind, const double* in, double* out, int* out_kind) {
    const Grid* g = static_cast<const Grid*>(gp);
    try {
        CField x = in_kind == 0 ? cplx_from_spat(g, in) : cplx_from_spec(g, in);
        CField y(g);
        switch (op) {
            case 0: y = OpsC::diff_lon(x); break;
            case 1: y = OpsC::spec_one_minus_mu_squared_diff_lat_mu(x); break;
            case 2: y = OpsC::mu(x); break;
            case 3: y = OpsC::mu2(x); break;
            case 4: y = OpsC::laplace(x); break;
            case 5: y = OpsC::grad_lon(x); break;
            case 6: y = OpsC::grad_lat(x); break;
            case 7: y = OpsC::div_lat(x); break;
            case 14: y = x; break;
            default: return 1;
        }
        if (y.spat_valid) { std::memcpy(out, (const void*)y.spat.data(), sizeof(cplx) * g->nspat); *out_kind = 0; }
        else { std::memcpy(out, (const void*)y.spec.data(), sizeof(cplx) * g->ncplx); *out_kind = 1; }
        return 0;
    } catch (...) {
        return 2;
    }
}

// LAPACK zgbsv semantics (A(i,j) at ab[(kl+ku+i-j) + j*ldab], 0-based)
int orc_zgbsv(int n, int kl, int ku, double* ab, int ldab, int* ipiv, double* b) {
    return gbsv(n, kl, ku, C(ab), ldab, ipiv, C(b));
}

// Build an SPHSolverComplex from components and either solve (mode 0) or
// apply (mode 1) it to a complex spectral vector.
// comp ids: 0 scalar_phi, 1 mu_phi, 2 one_minus_mu_mu_diff_mu_phi, 3 z1, 4 z2,
// 5 z3, 6 z4, 7 z4robert, 8 z5, 9 z5robert, 10 z6, 11 z6robert, 12 z7, 13 z8
int orc_solver(const void* gp, int halo, int ncomp, const int* comp, const double* scal, double r, int fix_z5,
               int mode, const double* rhs, double* out) {
    const Grid* g = static_cast<const Grid*>(gp);
    try {
        SolverC s;
        s.setup(g, halo);
        s.fix_z5robert = fix_z5 != 0;
        for (int k = 0; k < ncomp; k++) {
            const cplx v(scal[2 * k], scal[2 * k + 1]);
            switch (comp[k]) {
                case 0: s.scalar_phi(v); break;
                case 1: s.mu_phi(v); break;
                case 2: s.one_minus_mu_mu_diff_mu_phi(); break;
                case 3: s.z1(v, r); break;
                case 4: s.z2(v, r); break;
                case 5: s.z3(v, r); break;
                case 6: s.z4(v, r); break;
                case 7: s.z4robert(v, r); break;
                case 8: s.z5(v, r); break;
                case 9: s.z5robert(v, r); break;
                case 10: s.z6(v, r); break;
                case 11: s.z6robert(v, r); break;
                case 12: s.z7(v, r); break;
                case 13: s.z8(v, r); break;
                default: return 1;
            }
        }
        CField x = cplx_from_spec(g, rhs);
        CField y = mode == 0 ? s.solve(x) : s.apply(x);
        std::memcpy(out, (const void*)y.spec.data(), sizeof(cplx) * g->ncplx);
        return 0;
    } catch (...) {
        return 2;
    }
}

// raw band rows of a solver (N-compact order, 2*halo+1 per row), for checks of
// the assembled matrix
int orc_solver_rows(const void* gp, int halo, int ncomp, const int* comp, const double* scal, double r, int fix_z5,
                    double* out_rows) {
    const Grid* g = static_cast<const Grid*>(gp);
    SolverC s;
    s.setup(g, halo);
    s.fix_z5robert = fix_z5 != 0;
    for (int k = 0; k < ncomp; k++) {
        const cplx v(scal[2 * k], scal[2 * k + 1]);
        switch (comp[k]) {
            case 0: s.scalar_phi(v); break;
            case 1: s.mu_phi(v); break;
            case 2: s.one_minus_mu_mu_diff_mu_phi(); break;
            case 3: s.z1(v, r); break;
            case 4: s.z2(v, r); break;
            case 5: s.z3(v, r); break;
            case 6: s.z4(v, r); break;
            case 7: s.z4robert(v, r); break;
            case 8: s.z5(v, r); break;
            case 9: s.z5robert(v, r); break;
            case 10: s.z6(v, r); break;
            case 11: s.z6robert(v, r); break;
            case 12: s.z7(v, r); break;
            case 13: s.z8(v, r); break;
            default: return 1;
        }
    }
    std::memcpy(out_rows, (const void*)s.rows.data(), sizeof(cplx) * s.rows.size());
    return 0;
}

// REXI coefficients; returns the number of poles written (<= cap), or -1
int orc_rexi_coeffs(double h, int M, int L, int half, double* alpha, double* beta_re, double* beta_im, int cap) {
    try {
        Rexi r;
        r.setup(h, M, L, half != 0);
        const int n = (int)r.alpha.size();
        if (n > cap) return -1;
        std::memcpy(alpha, (const void*)r.alpha.data(), sizeof(cplx) * n);
        std::memcpy(beta_re, (const void*)r.beta_re.data(), sizeof(cplx) * n);
        std::memcpy(beta_im, (const void*)r.beta_im.data(), sizeof(cplx) * n);
        return n;
    } catch (...) {
        return -1;
    }
}

// SWE parameters: p[0]=a, p[1]=g, p[2]=omega, p[3]=h0, p[4]=visc, p[5]=dt
static SWEParams make_params(const double* p, int nonlinear, int robert) {
    SWEParams s;
    s.a = p[0]; s.g = p[1]; s.omega = p[2]; s.h0 = p[3]; s.visc = p[4]; s.dt = p[5];
    s.nonlinear = nonlinear; s.robert = robert;
    return s;
}

// One tendency evaluation (spectral in, spectral out)
int orc_swe_tendency(const void* gp, const double* p, int nonlinear, int robert, const double* h, const double* u,
                     const double* v, double* ht, double* ut, double* vt) {
    const Grid* g = static_cast<const Grid*>(gp);
    try {
        SWEParams s = make_params(p, nonlinear, robert);
        Field fdata(g);
        fdata.spat_update_lambda_gaussian_grid([](double, double mu, double& d) { d = mu; });
        Field H = real_from_spec(g, h), U = real_from_spec(g, u), V = real_from_spec(g, v);
        Field Ht(g), Ut(g), Vt(g);
        swe_tendency(s, fdata, H, U, V, Ht, Ut, Vt);
        Ht.request_spec(); Ut.request_spec(); Vt.request_spec();
        std::memcpy(ht, (const void*)Ht.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(ut, (const void*)Ut.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(vt, (const void*)Vt.spec.data(), sizeof(cplx) * g->nlm);
        return 0;
    } catch (...) {
        return 2;
    }
}

// nsteps RK4 steps of the SWE (AppSWE::run RK branch); state spectral in/out.
// Returns 0, 3 if a non-finite value appeared, 2 on other errors.
int orc_swe_run(const void* gp, const double* p, int nonlinear, int robert, double* h, double* u, double* v,
                int nsteps) {
    const Grid* g = static_cast<const Grid*>(gp);
    try {
        SWEParams s = make_params(p, nonlinear, robert);
        Field fdata(g);
        fdata.spat_update_lambda_gaussian_grid([](double, double mu, double& d) { d = mu; });
        Field H = real_from_spec(g, h), U = real_from_spec(g, u), V = real_from_spec(g, v);
        int rc = 0;
        for (int k = 0; k < nsteps; k++) {
            swe_rk4_step(s, fdata, H, U, V, s.dt);
            if (H.isAnyNaNorInf()) { rc = 3; break; }
        }
        H.request_spec(); U.request_spec(); V.request_spec();
        std::memcpy(h, (const void*)H.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(u, (const void*)U.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(v, (const void*)V.spec.data(), sizeof(cplx) * g->nlm);
        return rc;
    } catch (...) {
        return 2;
    }
}

// One pole of SWERexiSPH[Robert]::setup + solve: inputs phi0 = g h, u, v (real
// spectral), outputs the real spectra of Re(I_c(beta * x)).  alpha, beta are
// the raw pole coefficients (divided by tau inside setup).
int orc_rexi_pole(const void* gp, const double* p, int robert, int coriolis, int fix_z5, const double* alpha,
                  const double* beta, const double* phi0, const double* u, const double* v, double* ophi, double* ou,
                  double* ov) {
    const Grid* g = static_cast<const Grid*>(gp);
    try {
        RexiSWE s;
        s.setup(g, cplx(alpha[0], alpha[1]), cplx(beta[0], beta[1]), p[0], p[2], p[3] * p[1], p[5],
                coriolis != 0 && p[2] != 0, robert != 0, fix_z5 != 0);
        Field P = real_from_spec(g, phi0), U = real_from_spec(g, u), V = real_from_spec(g, v);
        Field a(g), b(g), c(g);
        s.solve(P, U, V, a, b, c);
        a.request_spec(); b.request_spec(); c.request_spec();
        std::memcpy(ophi, (const void*)a.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(ou, (const void*)b.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(ov, (const void*)c.spec.data(), sizeof(cplx) * g->nlm);
        return 0;
    } catch (...) {
        return 2;
    }
}

// nsteps REXI steps (AppSWE::run REXI branch, extended modes off); state h,u,v
// spectral in/out.  p as orc_swe_run (p[5] = tau).  Returns number of poles
// used (>0) or <0 on error.
int orc_rexi_run(const void* gp, const double* p, int robert, int coriolis, double rexi_h, int rexi_M, int half,
                 int fix_z5, double* h, double* u, double* v, int nsteps) {
    const Grid* g = static_cast<const Grid*>(gp);
    try {
        SWEParams s = make_params(p, 0, robert);
        Rexi rx;
        rx.setup(rexi_h, rexi_M, 0, half != 0);
        const int np = (int)rx.alpha.size();
        std::vector<std::unique_ptr<RexiSWE>> solvers(np);
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 0; i < np; i++) {
            solvers[i].reset(new RexiSWE());
            solvers[i]->setup(g, rx.alpha[i], rx.beta_re[i], s.a, s.omega, s.h0 * s.g, s.dt, coriolis != 0 && s.omega != 0,
                              robert != 0, fix_z5 != 0);
        }
        Field H = real_from_spec(g, h), U = real_from_spec(g, u), V = real_from_spec(g, v);
        for (int k = 0; k < nsteps; k++) {
            Field phi_r = H * s.g;
            Field u_r = U, v_r = V;
            Field acc_phi(g), acc_u(g), acc_v(g);
            acc_phi.spat_set_zero(); acc_u.spat_set_zero(); acc_v.spat_set_zero();
            // poles are independent: solve in parallel, accumulate in pole order
            std::vector<std::unique_ptr<Field>> out(3 * np);
            phi_r.request_spat(); u_r.request_spat(); v_r.request_spat();
#pragma omp parallel for schedule(dynamic, 1)
            for (int i = 0; i < np; i++) {
                Field a(phi_r), b(u_r), c(v_r);
                out[3 * i].reset(new Field(g));
                out[3 * i + 1].reset(new Field(g));
                out[3 * i + 2].reset(new Field(g));
                solvers[i]->solve(a, b, c, *out[3 * i], *out[3 * i + 1], *out[3 * i + 2]);
                out[3 * i]->request_spec(); out[3 * i + 1]->request_spec(); out[3 * i + 2]->request_spec();
            }
            for (int i = 0; i < np; i++) {
                acc_phi += *out[3 * i];
                acc_u += *out[3 * i + 1];
                acc_v += *out[3 * i + 2];
            }
            H = acc_phi * (1.0 / s.g);
            U = acc_u;
            V = acc_v;
            if (s.visc != 0) {
                const double sc = s.visc * s.dt;
                H = H.spec_solve_helmholtz(1.0, -sc, s.a);
                U = U.spec_solve_helmholtz(1.0, -sc, s.a);
                V = V.spec_solve_helmholtz(1.0, -sc, s.a);
            }
        }
        H.request_spec(); U.request_spec(); V.request_spec();
        std::memcpy(h, (const void*)H.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(u, (const void*)U.spec.data(), sizeof(cplx) * g->nlm);
        std::memcpy(v, (const void*)V.spec.data(), sizeof(cplx) * g->nlm);
        return np;
    } catch (...) {
        return -2;
    }
}

}  // extern "C"
