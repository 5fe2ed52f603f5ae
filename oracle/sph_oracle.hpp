// TEST INFRASTRUCTURE ONLY — the oracle.
//
// A plain C++17 / OpenMP / FP64 CPU restatement of the spectral shallow-water
// algorithm of schreiberx/sph_swe, written from the mathematics.  It is the
// checker for the CUDA library (tests, smoke, and the bench's cpu_baseline leg)
// and is never linked into, loaded by, or called from the product path.
//
// The reference delegates its transforms to SHTNS 2.6.6-r535 (+FFTW 3.3.4) and
// its banded solves to LAPACK 3.6.1 zgbsv; none of these are present here.  The
// oracle restates their published algorithms:
//   * Gauss-Legendre quadrature (Newton iteration on P_n, Tricomi start),
//   * orthonormal associated Legendre functions with Condon-Shortley phase
//     (SHTNS "sht_orthonormal" without SHT_NO_CS_PHASE; SPHConfig.hpp:338),
//   * a mixed-radix Stockham FFT,
//   * banded LU with partial pivoting following LAPACK zgbtf2/zgbtrs.
// Pinning: against scipy.special.roots_legendre / sph_harm_y, numpy.fft,
// scipy.linalg.lapack.zgbsv and the analytic known-answer tests of the
// reference's P1/P4 programs (AppTestSPHOperators.hpp, AppTestSPHSolverComplex.hpp).
//
// Conventions follow the reference (file:line relative to its src/ tree):
//   grid index      i_lon*nlat + j_lat, j=0 nearest the north pole
//                   (SPHConfig.hpp:344,390 SHT_THETA_CONTIGUOUS; SPHData.hpp:645-666)
//   real spectral   m-major, n contiguous: (m*(2L-m+1))/2 + n   (SPHConfig.hpp:106-116)
//   complex spectral n*n+n+m                                      (SPHConfig.hpp:120-130)
//   real synthesis  f = sum_l Q_l0 Y_l0 + 2 Re sum_{m>0} Q_lm Y_lm
//   complex         Y_l^{-m} = (-1)^m conj(Y_l^m)
#pragma once

#include <complex>
#include <vector>
#include <functional>
#include <cstddef>
#include <cmath>

namespace orc {

using cplx = std::complex<double>;

// ---------------------------------------------------------------- FFT
struct FFTPlan {
    int n = 0;
    std::vector<int> radices;
    std::vector<cplx> tw;  // exp(-2 pi i t / n), t = 0..n-1
    void init(int n);
    // in-place complex DFT, sign -1 (forward) or +1 (backward, unnormalised)
    void exec(cplx* x, cplx* work, int sign) const;
};

// ---------------------------------------------------------------- grid
struct Grid {
    int L = 0;            // lmax == mmax
    int nlat = 0, nphi = 0, nh = 0;
    int nlm = 0;          // (L+1)(L+2)/2
    int ncplx = 0;        // (L+1)^2
    int nspat = 0;
    std::vector<double> mu, w, cosphi, lat;   // per latitude
    // P_l^m(mu_j) for j < nh, l = m..L+1: plm[poff[m] + (l-m)*nh + j]
    std::vector<double> plm;
    std::vector<size_t> poff;
    FFTPlan fft;

    void setup(int L, int nlat, int nphi);
    inline int idx(int n, int m) const { return ((m * (2 * L - m + 1)) >> 1) + n; }
    inline int cidx(int n, int m) const { return n * n + n + m; }
    inline double P(int l, int m, int j) const { return plm[poff[m] + (size_t)(l - m) * nh + j]; }

    // transforms (batched over independent fields, contiguous)
    void spat_to_SH(const double* spat, cplx* spec, int lmax_out = -1) const;
    void SH_to_spat(const cplx* spec, double* spat, int lmax_in = -1) const;
    void cplx_spat_to_SH(const cplx* spat, cplx* spec) const;
    void cplx_SH_to_spat(const cplx* spec, cplx* spat) const;

    // Fourier-level helpers: F[m*nlat+j], m=0..lmax
    void ring_analysis(const double* spat, cplx* F, int mmax) const;
    void ring_synthesis(const cplx* F, double* spat, int mmax) const;
    void legendre_analysis(const cplx* F, cplx* spec, int lmax) const;   // spec: packed for lmax
    void legendre_synthesis(const cplx* spec, cplx* F, int lmax) const;
};

// automatic grid choice for a quadratic (3/2) rule, as SHTNS shtns_set_grid_auto
// with nl_order=2 (SPHConfig.hpp:366-399): nphi = smallest 7-smooth >= 3L+1,
// nlat = (3L)/2+1 rounded up to even.
void auto_grid(int L, int* nlat, int* nphi);

// ---------------------------------------------------------------- identities
// SPHIdentities.hpp:17-103 (R, S, A, B, C, D, E, G, H; double arguments)
struct Id {
    static double R(double k, double m);
    static double S(double k, double m);
    static double A(double k, double m) { double n = k + 2.0; return R(n - 1, m) * R(n - 2, m); }
    static double B(double n, double m) { return R(n - 1, m) * S(n, m) + S(n + 1, m) * R(n, m); }
    static double C(double k, double m) { double n = k - 2.0; return S(n + 1, m) * S(n + 2, m); }
    static double D(double k, double m) { double n = k + 1; return (2.0 * n + 1.0) * std::sqrt((n * n - m * m) / (4.0 * n * n - 1.0)); }
    static double E(double n, double) { return -n; }
    static double G(double n, double m) { n = n + 1; return D(n - 1, m) + E(n, m) * R(n - 1, m); }
    static double H(double n, double m) { n = n - 1; return E(n, m) * S(n + 1, m); }
};

// ---------------------------------------------------------------- lazy fields
// Restates SPHData's dual representation (SPHData.hpp:28-227): exactly one of
// the representations is valid after a request, the other is dropped.
class Field {
public:
    const Grid* g;
    mutable std::vector<cplx> spec;
    mutable std::vector<double> spat;
    mutable bool spec_valid = false, spat_valid = false;

    explicit Field(const Grid* g_);
    Field(const Field& o);
    Field& operator=(const Field& o);

    void request_spec() const;
    void request_spat() const;

    Field operator+(const Field& o) const;
    Field& operator+=(const Field& o);
    Field& operator-=(const Field& o);
    Field operator-(const Field& o) const;
    Field operator-() const;
    Field operator*(const Field& o) const;       // grid product
    Field operator*(double v) const;
    const Field& operator*=(double v) const;
    const Field& operator*=(const cplx& v) const;
    Field operator/(double v) const;
    Field operator+(double v) const;             // adds v*sqrt(4 pi) to (0,0)

    cplx spec_get(int n, int m) const;
    void spec_set_zero();
    void spat_set_zero();
    void spat_update_lambda(const std::function<void(double, double, double&)>& f);           // (lon, lat)
    void spat_update_lambda_gaussian_grid(const std::function<void(double, double, double&)>& f);   // (lon, mu)
    void spat_update_lambda_cogaussian_grid(const std::function<void(double, double, double&)>& f); // (lon, cos phi)
    void spec_update_lambda(const std::function<void(int, int, cplx&)>& f);
    Field spec_solve_helmholtz(double a, double b, double r) const;
    bool isAnyNaNorInf() const;
};
inline Field operator*(double v, const Field& f) { return f * v; }

class CField {
public:
    const Grid* g;
    mutable std::vector<cplx> spec;
    mutable std::vector<cplx> spat;
    mutable bool spec_valid = false, spat_valid = false;

    explicit CField(const Grid* g_);
    CField(const CField& o);
    CField(const Field& o);                      // promotion through the grid
    CField& operator=(const CField& o);
    CField& operator=(const Field& o);

    void request_spec() const;
    void request_spat() const;

    void spat_RealToSPHData(Field& out) const;
    void spat_fromSPHData(const Field& in);

    CField operator+(const CField& o) const;
    CField& operator+=(const CField& o);
    CField& operator-=(const CField& o);
    CField operator-(const CField& o) const;
    CField operator-() const;
    CField operator*(const CField& o) const;     // grid product (full grid; see defect note)
    CField operator*(double v) const;
    CField operator*(const cplx& v) const;
    const CField& operator*=(double v) const;
    const CField& operator*=(const cplx& v) const;
    CField operator/(double v) const;
    CField operator+(double v) const;
    CField operator+(const cplx& v) const;

    cplx spec_get(int n, int m) const;
    void spat_set_zero();
    void spat_update_lambda(const std::function<void(double, double, cplx&)>& f);
    void spat_update_lambda_gaussian_grid(const std::function<void(double, double, cplx&)>& f);
    void spat_update_lambda_cogaussian_grid(const std::function<void(double, double, cplx&)>& f);
    void spec_update_lambda(const std::function<void(int, int, cplx&)>& f);
    CField spec_solve_helmholtz(const cplx& a, const cplx& b, double r) const;
};
inline CField operator*(double v, const CField& f) { return f * v; }
inline CField operator*(const cplx& v, const CField& f) { return f * v; }
inline CField operator+(double v, const CField& f) { return f + v; }
inline CField operator+(const cplx& v, const CField& f) { return f + v; }

// ---------------------------------------------------------------- operators
// SPHOperators.hpp
struct Ops {
    static Field diff_lon(const Field& x);
    static Field spec_one_minus_mu_squared_diff_lat_mu(const Field& x);
    static Field mu(const Field& x);
    static Field mu2(const Field& x);
    static Field grad_lon(const Field& x);
    static Field grad_lat(const Field& x);
    static Field div_lon(const Field& x) { return grad_lon(x); }
    static Field div_lat(const Field& x);
    static Field diff_lat_mu(const Field& x);
    static Field laplace(const Field& x);
    static Field vort(const Field& lon, const Field& lat) { return grad_lon(lat) - grad_lat(lon); }
    static Field div(const Field& lon, const Field& lat) { return div_lon(lon) + div_lat(lat); }
    static Field robert_div_lon(const Field& x);
    static Field robert_div_lat(const Field& x);
    static Field robert_grad_lon(const Field& x) { return diff_lon(x); }
    static Field robert_grad_lat(const Field& x) { return spec_one_minus_mu_squared_diff_lat_mu(x); }
};

// SPHOperatorsComplex.hpp
struct OpsC {
    static CField diff_lon(const CField& x);
    static CField spec_one_minus_mu_squared_diff_lat_mu(const CField& x);
    static CField mu(const CField& x);
    static CField mu2(const CField& x);
    static CField grad_lon(const CField& x);
    static CField grad_lat(const CField& x);
    static CField div_lon(const CField& x) { return grad_lon(x); }
    static CField div_lat(const CField& x);
    static CField laplace(const CField& x);
    static CField vort(const CField& lon, const CField& lat) { return grad_lon(lat) - grad_lat(lon); }
    static CField div(const CField& lon, const CField& lat) { return div_lon(lon) + div_lat(lat); }
    static CField robert_grad_lon(const CField& x) { return diff_lon(x); }
    static CField robert_grad_lat(const CField& x) { return spec_one_minus_mu_squared_diff_lat_mu(x); }
    static CField robert_vort(const CField& lon, const CField& lat) { return robert_grad_lon(lat) - robert_grad_lat(lon); }
    static CField robert_div(const CField& lon, const CField& lat);
};

// ---------------------------------------------------------------- banded LU
// LAPACK zgbsv semantics: LU with partial pivoting of an n x n band matrix
// with kl sub- and ku super-diagonals in LAPACK GB storage (ldab >= 2kl+ku+1,
// A(i,j) at ab[(kl+ku+i-j) + j*ldab], 0-based), then forward/back solve.
// Returns info (0 ok, k>0 zero pivot at column k).
int gbsv(int n, int kl, int ku, cplx* ab, int ldab, int* ipiv, cplx* b);

// ---------------------------------------------------------------- REXI solver
// SPHSolverComplex.hpp + SPHMatrixComplex.hpp + BandedMatrixSolver.hpp
class SolverC {
public:
    const Grid* g = nullptr;
    int halo = 0, ndiag = 0;
    bool fix_z5robert = false;
    std::vector<cplx> rows;       // (L+1)^2 rows in N-compact order, ndiag each
    void setup(const Grid* g, int halo);
    size_t ncompact(int n, int m) const;
    cplx* row(int n, int m) { return &rows[ncompact(n, m) * ndiag]; }
    void add(cplx* row, int n, int m, int rel, const cplx& v);

    void scalar_phi(const cplx& v);
    void mu_phi(const cplx& s = 1.0);
    void one_minus_mu_mu_diff_mu_phi();
    void z1(const cplx& s, double r) { scalar_phi(s); }
    void z2(const cplx& s, double r);
    void z3(const cplx& s, double r);
    void z4(const cplx& s, double r);
    void z4robert(const cplx& s, double r);
    void z5(const cplx& s, double r);
    void z5robert(const cplx& s, double r);
    void z6(const cplx& s, double r);
    void z6robert(const cplx& s, double r);
    void z7(const cplx& s, double r);
    void z8(const cplx& s, double r);
    CField solve(const CField& rhs) const;
    CField apply(const CField& x) const;
};

// ---------------------------------------------------------------- REXI coefficients
// REXI.hpp:52-131, GaussianApproximation.hpp:38-81, ExponentialApproximation.hpp:49-124
struct Rexi {
    std::vector<cplx> alpha, beta_re, beta_im;
    void setup(double h, int M, int L = 0, bool half = true);
    cplx approx_e_ix(double x) const;
};

// SWERexiSPH.hpp / SWERexiSPHRobert.hpp
class RexiSWE {
public:
    bool robert = true;
    const Grid* g = nullptr;
    SolverC phi_solver, vel_solver;
    cplx alpha, beta;
    bool coriolis = true;
    double tau = 0, r = 0, ir = 0, omega = 0, two_omega = 0, avg_geopot = 0;
    void setup(const Grid* g, const cplx& alpha, const cplx& beta, double radius, double omega,
               double avg_geopot, double tau, bool coriolis, bool robert, bool fix_z5robert);
    void solve(const Field& phi0, const Field& u0, const Field& v0, Field& o_phi, Field& o_u, Field& o_v) const;
};

// ---------------------------------------------------------------- SWE app
struct SWEParams {
    double a = 6.37122e6, g = 9.80616, omega = 7.292e-5, h0 = 1e4, visc = 0.0, dt = 120.0;
    // nonlinear: 0 linear, 1 the reference's nonlinear advective form (robert
    // ignored); the vorticity-divergence form is restated in oracle/vortdiv.py
    int nonlinear = 1, robert = 0;
};

// AppSWE::p_run_euler_timestep_update (AppSWE.hpp:574-659)
void swe_tendency(const SWEParams& p, const Field& fdata, const Field& h, const Field& u, const Field& v,
                  Field& h_t, Field& u_t, Field& v_t);
// TimesteppingRK RK4 (TimesteppingRK.hpp:310-392)
void swe_rk4_step(const SWEParams& p, const Field& fdata, Field& h, Field& u, Field& v, double dt);

}  // namespace orc
