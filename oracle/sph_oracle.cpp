// TEST INFRASTRUCTURE ONLY — the oracle (see sph_oracle.hpp for scope and pinning).
#include "sph_oracle.hpp"

#include <algorithm>
#include <cassert>
#include <cstring>
#include <stdexcept>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const double PI = 3.14159265358979323846264338327950288;

// ============================================================ FFT
void FFTPlan::init(int n_) {
    n = n_;
    radices.clear();
    int r = n;
    while (r % 4 == 0) { radices.push_back(4); r /= 4; }
    while (r % 2 == 0) { radices.push_back(2); r /= 2; }
    for (int p = 3; r > 1; p += 2) {
        while (r % p == 0) { radices.push_back(p); r /= p; }
    }
    tw.resize(n);
    for (int t = 0; t < n; t++) {
        // exp(-2 pi i t/n), argument reduced to [0, pi/4]-ish accuracy by symmetric evaluation
        long double a = -2.0L * (long double)PI * (long double)t / (long double)n;
        tw[t] = cplx((double)std::cos(a), (double)std::sin(a));
    }
}

// Stockham auto-sort, decimation in time.  Pass with radix R over sub-length Ls:
// out[(j-k)*R + k + s*Ls] = sum_r x[j + r*n/R] * w^(r*k*n/(Ls*R)) * w^(r*s*n/R), k = j mod Ls.
void FFTPlan::exec(cplx* x, cplx* work, int sign) const {
    cplx* src = x;
    cplx* dst = work;
    int Ls = 1;
    cplx v[64], o[64];
    for (int R : radices) {
        const int nR = n / R;
        const int tstep = n / (Ls * R);
        for (int j = 0; j < nR; j++) {
            const int k = j % Ls;
            for (int r = 0; r < R; r++) {
                cplx t = tw[(size_t)((long long)r * k * tstep % n)];
                if (sign > 0) t = std::conj(t);
                v[r] = src[j + r * nR] * t;
            }
            for (int s = 0; s < R; s++) {
                cplx acc = 0;
                for (int r = 0; r < R; r++) {
                    cplx t = tw[(size_t)((long long)r * s * nR % n)];
                    if (sign > 0) t = std::conj(t);
                    acc += v[r] * t;
                }
                o[s] = acc;
            }
            const int base = (j - k) * R + k;
            for (int s = 0; s < R; s++) dst[base + s * Ls] = o[s];
        }
        std::swap(src, dst);
        Ls *= R;
    }
    if (src != x) std::memcpy(x, src, sizeof(cplx) * n);
}

// ============================================================ grid
static bool smooth7(int n) {
    for (int p : {2, 3, 5, 7}) while (n % p == 0) n /= p;
    return n == 1;
}

void auto_grid(int L, int* nlat, int* nphi) {
    int np = 3 * L + 1;
    while (!smooth7(np)) np++;
    int nl = (3 * L) / 2 + 1;
    if (nl & 1) nl++;
    *nlat = nl;
    *nphi = np;
}

static void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const int nh = (n + 1) / 2;
    for (int k = 0; k < nh; k++) {
        double z = std::cos(PI * (k + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int i = 2; i <= n; i++) {
                double p2 = ((2.0 * i - 1.0) * z * p1 - (i - 1.0) * p0) / i;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) <= 1e-16 * std::fabs(z) + 1e-300) {
                if (it > 0) break;
            }
        }
        // derivative at the converged node
        double p0 = 1.0, p1 = z;
        for (int i = 2; i <= n; i++) {
            double p2 = ((2.0 * i - 1.0) * z * p1 - (i - 1.0) * p0) / i;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        x[k] = z;
        x[n - 1 - k] = -z;
        double wk = 2.0 / ((1.0 - z * z) * dp * dp);
        w[k] = wk;
        w[n - 1 - k] = wk;
    }
}

// Orthonormal P_l^m(x) with CS phase for m = 0..mmax, l = m..lmax, with a
// power-of-two exponent carried along so that sin^m(theta) cannot underflow
// before the l-recurrence grows it back.
static void plm_at(int mmax, int lmax, double x, const std::vector<size_t>& poff, int nh, int j, double* plm) {
    const double s = std::sqrt((1.0 - x) * (1.0 + x));
    const double BIG = std::ldexp(1.0, 600), SMALL = std::ldexp(1.0, -600);
    double pmm = std::sqrt(1.0 / (4.0 * PI));
    int e = 0;
    for (int m = 0; m <= mmax; m++) {
        if (m > 0) {
            pmm *= -std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * s;
            if (std::fabs(pmm) < SMALL && pmm != 0.0) { pmm *= BIG; e -= 600; }
        }
        double* col = plm + poff[m] + j;
        double p0 = pmm;
        int el = e;
        col[0] = std::ldexp(p0, el);
        if (m + 1 > lmax) continue;
        double p1 = x * std::sqrt(2.0 * m + 3.0) * p0;
        col[(size_t)nh] = std::ldexp(p1, el);
        for (int l = m + 2; l <= lmax; l++) {
            double ll = l, mm = m;
            double a = std::sqrt((4.0 * ll * ll - 1.0) / (ll * ll - mm * mm));
            double b = std::sqrt(((ll - 1.0) * (ll - 1.0) - mm * mm) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0));
            double p2 = a * (x * p1 - b * p0);
            p0 = p1;
            p1 = p2;
            if (el < 0 && std::fabs(p1) > BIG) { p0 *= SMALL; p1 *= SMALL; el += 600; }
            col[(size_t)(l - m) * nh] = std::ldexp(p1, el);
        }
    }
}

void Grid::setup(int L_, int nlat_, int nphi_) {
    L = L_;
    if (nlat_ <= 0 || nphi_ <= 0) auto_grid(L, &nlat_, &nphi_);
    nlat = nlat_;
    nphi = nphi_;
    if (nlat % 2) throw std::runtime_error("nlat must be even");
    nh = nlat / 2;
    nlm = (L + 1) * (L + 2) / 2;
    ncplx = (L + 1) * (L + 1);
    nspat = nlat * nphi;
    gauss_legendre(nlat, mu, w);
    cosphi.resize(nlat);
    lat.resize(nlat);
    for (int j = 0; j < nlat; j++) {
        cosphi[j] = std::sqrt((1.0 - mu[j]) * (1.0 + mu[j]));
        lat[j] = 0.5 * PI - std::acos(mu[j]);
    }
    const int mmax = L + 1, lmax = L + 1;
    poff.resize(mmax + 2);
    size_t off = 0;
    for (int m = 0; m <= mmax; m++) {
        poff[m] = off;
        off += (size_t)(lmax - m + 1) * nh;
    }
    poff[mmax + 1] = off;
    plm.assign(off, 0.0);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nh; j++) plm_at(mmax, lmax, mu[j], poff, nh, j, plm.data());
    fft.init(nphi);
}

void Grid::ring_analysis(const double* spat, cplx* F, int mmax) const {
    const int N = nphi;
    const double scale = 2.0 * PI / N;
#pragma omp parallel
    {
        std::vector<cplx> z(N), wk(N);
#pragma omp for schedule(static)
        for (int jp = 0; jp < nh; jp++) {
            const int j = 2 * jp;
            for (int i = 0; i < N; i++) z[i] = cplx(spat[(size_t)i * nlat + j], spat[(size_t)i * nlat + j + 1]);
            fft.exec(z.data(), wk.data(), -1);
            for (int m = 0; m <= mmax; m++) {
                cplx a = z[m], b = std::conj(z[(N - m) % N]);
                cplx X = 0.5 * (a + b);
                cplx Y = cplx(0, -0.5) * (a - b);
                if (m > L) { X = 0; Y = 0; }
                F[(size_t)m * nlat + j] = X * scale;
                F[(size_t)m * nlat + j + 1] = Y * scale;
            }
        }
    }
}

void Grid::ring_synthesis(const cplx* F, double* spat, int mmax) const {
    const int N = nphi;
    const int mm = std::min(mmax, std::min(L, (N - 1) / 2));
#pragma omp parallel
    {
        std::vector<cplx> z(N), wk(N);
#pragma omp for schedule(static)
        for (int jp = 0; jp < nh; jp++) {
            const int j = 2 * jp;
            std::fill(z.begin(), z.end(), cplx(0));
            z[0] = cplx(F[j].real(), F[j + 1].real());
            for (int m = 1; m <= mm; m++) {
                cplx X = F[(size_t)m * nlat + j], Y = F[(size_t)m * nlat + j + 1];
                z[m] = X + cplx(0, 1) * Y;
                z[N - m] = std::conj(X) + cplx(0, 1) * std::conj(Y);
            }
            fft.exec(z.data(), wk.data(), +1);
            for (int i = 0; i < N; i++) {
                spat[(size_t)i * nlat + j] = z[i].real();
                spat[(size_t)i * nlat + j + 1] = z[i].imag();
            }
        }
    }
}

// packed layout for degree lmax: (m*(2*lmax-m+1))/2 + n, m = 0..lmax
static inline size_t pidx(int lmax, int n, int m) { return (size_t)((m * (2 * lmax - m + 1)) >> 1) + n; }

void Grid::legendre_analysis(const cplx* F, cplx* spec, int lmax) const {
    const int mtop = std::min(lmax, L);
#pragma omp parallel for schedule(dynamic, 1)
    for (int m = 0; m <= lmax; m++) {
        if (m > mtop) { spec[pidx(lmax, m, m)] = 0; continue; }
        std::vector<cplx> S(nh), A(nh);
        const cplx* Fm = F + (size_t)m * nlat;
        for (int j = 0; j < nh; j++) {
            S[j] = (Fm[j] + Fm[nlat - 1 - j]) * w[j];
            A[j] = (Fm[j] - Fm[nlat - 1 - j]) * w[j];
        }
        for (int l = m; l <= lmax; l++) {
            const double* p = &plm[poff[m] + (size_t)(l - m) * nh];
            const std::vector<cplx>& src = ((l - m) & 1) ? A : S;
            double re = 0, im = 0;
            for (int j = 0; j < nh; j++) { re += p[j] * src[j].real(); im += p[j] * src[j].imag(); }
            spec[pidx(lmax, l, m)] = cplx(re, im);
        }
    }
}

void Grid::legendre_synthesis(const cplx* spec, cplx* F, int lmax) const {
    const int mtop = std::min(lmax, L);
#pragma omp parallel for schedule(dynamic, 1)
    for (int m = 0; m <= mtop; m++) {
        cplx* Fm = F + (size_t)m * nlat;
        for (int j = 0; j < nh; j++) {
            double er = 0, ei = 0, orr = 0, oi = 0;
            for (int l = m; l <= lmax; l++) {
                const double p = plm[poff[m] + (size_t)(l - m) * nh + j];
                const cplx q = spec[pidx(lmax, l, m)];
                if ((l - m) & 1) { orr += p * q.real(); oi += p * q.imag(); }
                else { er += p * q.real(); ei += p * q.imag(); }
            }
            Fm[j] = cplx(er + orr, ei + oi);
            Fm[nlat - 1 - j] = cplx(er - orr, ei - oi);
        }
    }
}

void Grid::spat_to_SH(const double* spat, cplx* spec, int lmax_out) const {
    const int lm = lmax_out < 0 ? L : lmax_out;
    std::vector<cplx> F((size_t)(lm + 1) * nlat);
    ring_analysis(spat, F.data(), std::min(lm, L));
    legendre_analysis(F.data(), spec, lm);
}

void Grid::SH_to_spat(const cplx* spec, double* spat, int lmax_in) const {
    const int lm = lmax_in < 0 ? L : lmax_in;
    std::vector<cplx> F((size_t)(lm + 1) * nlat);
    legendre_synthesis(spec, F.data(), lm);
    ring_synthesis(F.data(), spat, std::min(lm, L));
}

void Grid::cplx_spat_to_SH(const cplx* spat, cplx* spec) const {
    const int N = nphi;
    const double scale = 2.0 * PI / N;
    std::vector<cplx> F((size_t)(2 * L + 1) * nlat);
#pragma omp parallel
    {
        std::vector<cplx> z(N), wk(N);
#pragma omp for schedule(static)
        for (int j = 0; j < nlat; j++) {
            for (int i = 0; i < N; i++) z[i] = spat[(size_t)i * nlat + j];
            fft.exec(z.data(), wk.data(), -1);
            for (int m = -L; m <= L; m++) F[(size_t)(m + L) * nlat + j] = z[((m % N) + N) % N] * scale;
        }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int m = -L; m <= L; m++) {
        const int am = std::abs(m);
        const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
        const cplx* Fm = &F[(size_t)(m + L) * nlat];
        std::vector<cplx> S(nh), A(nh);
        for (int j = 0; j < nh; j++) {
            S[j] = (Fm[j] + Fm[nlat - 1 - j]) * (w[j] * sg);
            A[j] = (Fm[j] - Fm[nlat - 1 - j]) * (w[j] * sg);
        }
        for (int l = am; l <= L; l++) {
            const double* p = &plm[poff[am] + (size_t)(l - am) * nh];
            const std::vector<cplx>& src = ((l - am) & 1) ? A : S;
            double re = 0, im = 0;
            for (int j = 0; j < nh; j++) { re += p[j] * src[j].real(); im += p[j] * src[j].imag(); }
            spec[cidx(l, m)] = cplx(re, im);
        }
    }
}

void Grid::cplx_SH_to_spat(const cplx* spec, cplx* spat) const {
    const int N = nphi;
    std::vector<cplx> F((size_t)(2 * L + 1) * nlat);
#pragma omp parallel for schedule(dynamic, 1)
    for (int m = -L; m <= L; m++) {
        const int am = std::abs(m);
        const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
        cplx* Fm = &F[(size_t)(m + L) * nlat];
        for (int j = 0; j < nh; j++) {
            cplx e = 0, o = 0;
            for (int l = am; l <= L; l++) {
                const double p = plm[poff[am] + (size_t)(l - am) * nh + j] * sg;
                if ((l - am) & 1) o += p * spec[cidx(l, m)];
                else e += p * spec[cidx(l, m)];
            }
            Fm[j] = e + o;
            Fm[nlat - 1 - j] = e - o;
        }
    }
#pragma omp parallel
    {
        std::vector<cplx> z(N), wk(N);
#pragma omp for schedule(static)
        for (int j = 0; j < nlat; j++) {
            std::fill(z.begin(), z.end(), cplx(0));
            for (int m = -L; m <= L; m++) z[((m % N) + N) % N] += F[(size_t)(m + L) * nlat + j];
            fft.exec(z.data(), wk.data(), +1);
            for (int i = 0; i < N; i++) spat[(size_t)i * nlat + j] = z[i];
        }
    }
}

// ============================================================ identities
double Id::R(double k, double m) {
    double n = k + 1;
    if (n < 0) return 0;
    if (n < std::fabs(m)) return 0;
    if (n * n - m * m < 0) return 0;
    return std::sqrt((n * n - m * m) / (4.0 * n * n - 1.0));
}

double Id::S(double k, double m) {
    double n = k - 1;
    if (n < 0) return 0;
    if (n < std::fabs(m)) return 0;
    if (n * n - m * m < 0) return 0;
    return std::sqrt(((n + 1.0) * (n + 1.0) - m * m) / ((2.0 * n + 1.0) * (2.0 * n + 3.0)));
}

// ============================================================ Field (real)
Field::Field(const Grid* g_) : g(g_), spec(g_->nlm), spat(g_->nspat) {}
Field::Field(const Field& o) : g(o.g), spec(o.g->nlm), spat(o.g->nspat) { *this = o; }
Field& Field::operator=(const Field& o) {
    if (o.spat_valid) spat = o.spat;
    if (o.spec_valid) spec = o.spec;
    spec_valid = o.spec_valid;
    spat_valid = o.spat_valid;
    return *this;
}
void Field::request_spec() const {
    if (spec_valid) return;
    assert(spat_valid);
    g->spat_to_SH(spat.data(), spec.data());
    spat_valid = false;
    spec_valid = true;
}
void Field::request_spat() const {
    if (spat_valid) return;
    assert(spec_valid);
    g->SH_to_spat(spec.data(), spat.data());
    spec_valid = false;
    spat_valid = true;
}
#define SPEC_OUT(out) out.spec_valid = true; out.spat_valid = false
Field Field::operator+(const Field& o) const {
    request_spec(); o.request_spec();
    Field out(g);
    for (int i = 0; i < g->nlm; i++) out.spec[i] = spec[i] + o.spec[i];
    SPEC_OUT(out);
    return out;
}
Field& Field::operator+=(const Field& o) {
    request_spec(); o.request_spec();
    for (int i = 0; i < g->nlm; i++) spec[i] += o.spec[i];
    spec_valid = true; spat_valid = false;
    return *this;
}
Field& Field::operator-=(const Field& o) {
    request_spec(); o.request_spec();
    for (int i = 0; i < g->nlm; i++) spec[i] -= o.spec[i];
    spec_valid = true; spat_valid = false;
    return *this;
}
Field Field::operator-(const Field& o) const {
    request_spec(); o.request_spec();
    Field out(g);
    for (int i = 0; i < g->nlm; i++) out.spec[i] = spec[i] - o.spec[i];
    SPEC_OUT(out);
    return out;
}
Field Field::operator-() const {
    request_spec();
    Field out(g);
    for (int i = 0; i < g->nlm; i++) out.spec[i] = -spec[i];
    SPEC_OUT(out);
    return out;
}
Field Field::operator*(const Field& o) const {
    request_spat(); o.request_spat();
    Field out(g);
    for (int i = 0; i < g->nspat; i++) out.spat[i] = o.spat[i] * spat[i];
    out.spec_valid = false; out.spat_valid = true;
    return out;
}
Field Field::operator*(double v) const {
    request_spec();
    Field out(g);
    for (int i = 0; i < g->nlm; i++) out.spec[i] = spec[i] * v;
    SPEC_OUT(out);
    return out;
}
const Field& Field::operator*=(double v) const {
    request_spec();
    for (int i = 0; i < g->nlm; i++) spec[i] *= v;
    return *this;
}
const Field& Field::operator*=(const cplx& v) const {
    request_spec();
    for (int i = 0; i < g->nlm; i++) spec[i] *= v;
    return *this;
}
Field Field::operator/(double v) const {
    request_spec();
    Field out(g);
    for (int i = 0; i < g->nlm; i++) out.spec[i] = spec[i] / v;
    SPEC_OUT(out);
    return out;
}
Field Field::operator+(double v) const {
    request_spec();
    Field out(*this);
    out.spec[0] += v * std::sqrt(4.0 * PI);
    SPEC_OUT(out);
    return out;
}
cplx Field::spec_get(int n, int m) const {
    if (n < 0 || m < 0 || n > g->L || m > g->L || m > n) return 0;
    return spec[g->idx(n, m)];
}
void Field::spec_set_zero() {
    std::fill(spec.begin(), spec.end(), cplx(0));
    spat_valid = false; spec_valid = true;
}
void Field::spat_set_zero() {
    std::fill(spat.begin(), spat.end(), 0.0);
    spat_valid = true; spec_valid = false;
}
void Field::spat_update_lambda(const std::function<void(double, double, double&)>& f) {
    if (spec_valid) request_spat();
    for (int i = 0; i < g->nphi; i++) {
        double lon = ((double)i / (double)g->nphi) * 2.0 * PI;
        for (int j = 0; j < g->nlat; j++) f(lon, g->lat[j], spat[(size_t)i * g->nlat + j]);
    }
    spat_valid = true; spec_valid = false;
}
void Field::spat_update_lambda_gaussian_grid(const std::function<void(double, double, double&)>& f) {
    if (spec_valid) request_spat();
    for (int i = 0; i < g->nphi; i++) {
        double lon = ((double)i / (double)g->nphi) * 2.0 * PI;
        for (int j = 0; j < g->nlat; j++) f(lon, g->mu[j], spat[(size_t)i * g->nlat + j]);
    }
    spat_valid = true; spec_valid = false;
}
void Field::spat_update_lambda_cogaussian_grid(const std::function<void(double, double, double&)>& f) {
    if (spec_valid) request_spat();
    for (int i = 0; i < g->nphi; i++) {
        double lon = ((double)i / (double)g->nphi) * 2.0 * PI;
        for (int j = 0; j < g->nlat; j++) f(lon, g->cosphi[j], spat[(size_t)i * g->nlat + j]);
    }
    spat_valid = true; spec_valid = false;
}
void Field::spec_update_lambda(const std::function<void(int, int, cplx&)>& f) {
    if (spat_valid) request_spec();
    for (int m = 0; m <= g->L; m++)
        for (int n = m; n <= g->L; n++) f(n, m, spec[g->idx(n, m)]);
    spat_valid = false; spec_valid = true;
}
Field Field::spec_solve_helmholtz(double a, double b_, double r) const {
    Field out(*this);
    const double b = b_ / (r * r);
    out.spec_update_lambda([&](int n, int, cplx& d) { d /= (a + (-b * (double)n * ((double)n + 1.0))); });
    return out;
}
bool Field::isAnyNaNorInf() const {
    // SPHData.hpp:560-569 scans data_spat without a request (defect); here the
    // check runs on whichever representation is valid.
    if (spat_valid) {
        for (double x : spat) if (!std::isfinite(x)) return true;
        return false;
    }
    for (const cplx& x : spec) if (!std::isfinite(x.real()) || !std::isfinite(x.imag())) return true;
    return false;
}

// ============================================================ CField (complex)
CField::CField(const Grid* g_) : g(g_), spec(g_->ncplx), spat(g_->nspat) {}
CField::CField(const CField& o) : g(o.g), spec(o.g->ncplx), spat(o.g->nspat) { *this = o; }
CField::CField(const Field& o) : g(o.g), spec(o.g->ncplx), spat(o.g->nspat) { spat_fromSPHData(o); }
CField& CField::operator=(const CField& o) {
    if (o.spat_valid) spat = o.spat;
    if (o.spec_valid) spec = o.spec;
    spec_valid = o.spec_valid;
    spat_valid = o.spat_valid;
    return *this;
}
CField& CField::operator=(const Field& o) { spat_fromSPHData(o); return *this; }
void CField::request_spec() const {
    if (spec_valid) return;
    assert(spat_valid);
    g->cplx_spat_to_SH(spat.data(), spec.data());
    spat_valid = false; spec_valid = true;
}
void CField::request_spat() const {
    if (spat_valid) return;
    assert(spec_valid);
    g->cplx_SH_to_spat(spec.data(), spat.data());
    spec_valid = false; spat_valid = true;
}
void CField::spat_RealToSPHData(Field& out) const {
    request_spat();
    for (int i = 0; i < g->nspat; i++) out.spat[i] = spat[i].real();
    out.spec_valid = false; out.spat_valid = true;
}
void CField::spat_fromSPHData(const Field& in) {
    in.request_spat();
    for (int i = 0; i < g->nspat; i++) spat[i] = in.spat[i];
    spec_valid = false; spat_valid = true;
}
CField CField::operator+(const CField& o) const {
    request_spec(); o.request_spec();
    CField out(g);
    for (int i = 0; i < g->ncplx; i++) out.spec[i] = spec[i] + o.spec[i];
    SPEC_OUT(out);
    return out;
}
CField& CField::operator+=(const CField& o) {
    request_spec(); o.request_spec();
    for (int i = 0; i < g->ncplx; i++) spec[i] += o.spec[i];
    spec_valid = true; spat_valid = false;
    return *this;
}
CField& CField::operator-=(const CField& o) {
    request_spec(); o.request_spec();
    for (int i = 0; i < g->ncplx; i++) spec[i] -= o.spec[i];
    spec_valid = true; spat_valid = false;
    return *this;
}
CField CField::operator-(const CField& o) const {
    request_spec(); o.request_spec();
    CField out(g);
    for (int i = 0; i < g->ncplx; i++) out.spec[i] = spec[i] - o.spec[i];
    SPEC_OUT(out);
    return out;
}
CField CField::operator-() const {
    request_spec();
    CField out(g);
    for (int i = 0; i < g->ncplx; i++) out.spec[i] = -spec[i];
    SPEC_OUT(out);
    return out;
}
// SPHDataComplex.hpp:321-340 bounds its loop by cplx_spec_num_elems (defect: only
// the first (L+1)^2 grid points are multiplied, the rest of the output is left
// uninitialised).  The oracle multiplies the full grid.
CField CField::operator*(const CField& o) const {
    request_spat(); o.request_spat();
    CField out(g);
    for (int i = 0; i < g->nspat; i++) out.spat[i] = o.spat[i] * spat[i];
    out.spec_valid = false; out.spat_valid = true;
    return out;
}
CField CField::operator*(double v) const {
    request_spec();
    CField out(g);
    for (int i = 0; i < g->ncplx; i++) out.spec[i] = spec[i] * v;
    SPEC_OUT(out);
    return out;
}
CField CField::operator*(const cplx& v) const {
    request_spec();
    CField out(g);
    for (int i = 0; i < g->ncplx; i++) out.spec[i] = spec[i] * v;
    SPEC_OUT(out);
    return out;
}
const CField& CField::operator*=(double v) const {
    request_spec();
    for (int i = 0; i < g->ncplx; i++) spec[i] *= v;
    return *this;
}
const CField& CField::operator*=(const cplx& v) const {
    request_spec();
    for (int i = 0; i < g->ncplx; i++) spec[i] *= v;
    return *this;
}
CField CField::operator/(double v) const {
    request_spec();
    CField out(g);
    for (int i = 0; i < g->ncplx; i++) out.spec[i] = spec[i] / v;
    SPEC_OUT(out);
    return out;
}
CField CField::operator+(double v) const {
    request_spec();
    CField out(*this);
    out.spec[0] += v * std::sqrt(4.0 * PI);
    SPEC_OUT(out);
    return out;
}
CField CField::operator+(const cplx& v) const {
    CField out(*this);
    out.request_spec();
    out.spec[0] += v * std::sqrt(4.0 * PI);
    return out;
}
cplx CField::spec_get(int n, int m) const {
    if (n < 0 || n > g->L || std::abs(m) > g->L || std::abs(m) > n) return 0;
    return spec[g->cidx(n, m)];
}
void CField::spat_set_zero() {
    std::fill(spat.begin(), spat.end(), cplx(0));
    spat_valid = true; spec_valid = false;
}
void CField::spat_update_lambda(const std::function<void(double, double, cplx&)>& f) {
    if (spec_valid) request_spat();
    for (int i = 0; i < g->nphi; i++) {
        double lon = ((double)i / (double)g->nphi) * 2.0 * PI;
        for (int j = 0; j < g->nlat; j++) f(lon, g->lat[j], spat[(size_t)i * g->nlat + j]);
    }
    spat_valid = true; spec_valid = false;
}
void CField::spat_update_lambda_gaussian_grid(const std::function<void(double, double, cplx&)>& f) {
    if (spec_valid) request_spat();
    for (int i = 0; i < g->nphi; i++) {
        double lon = ((double)i / (double)g->nphi) * 2.0 * PI;
        for (int j = 0; j < g->nlat; j++) f(lon, g->mu[j], spat[(size_t)i * g->nlat + j]);
    }
    spat_valid = true; spec_valid = false;
}
void CField::spat_update_lambda_cogaussian_grid(const std::function<void(double, double, cplx&)>& f) {
    if (spec_valid) request_spat();
    for (int i = 0; i < g->nphi; i++) {
        double lon = ((double)i / (double)g->nphi) * 2.0 * PI;
        for (int j = 0; j < g->nlat; j++) f(lon, g->cosphi[j], spat[(size_t)i * g->nlat + j]);
    }
    spat_valid = true; spec_valid = false;
}
void CField::spec_update_lambda(const std::function<void(int, int, cplx&)>& f) {
    if (spat_valid) request_spec();
    for (int n = 0; n <= g->L; n++)
        for (int m = -n; m <= n; m++) f(n, m, spec[g->cidx(n, m)]);
    spat_valid = false; spec_valid = true;
}
CField CField::spec_solve_helmholtz(const cplx& a, const cplx& b_, double r) const {
    CField out(*this);
    const cplx b = b_ / (r * r);
    out.spec_update_lambda([&](int n, int, cplx& d) { d /= (a + (-b * (double)n * ((double)n + 1.0))); });
    return out;
}

// ============================================================ real operators
Field Ops::diff_lon(const Field& x) {
    x.request_spec();
    Field out(x.g);
    const Grid* g = x.g;
    for (int m = 0; m <= g->L; m++)
        for (int n = m; n <= g->L; n++) out.spec[g->idx(n, m)] = x.spec[g->idx(n, m)] * cplx(0, m);
    SPEC_OUT(out);
    return out;
}
Field Ops::spec_one_minus_mu_squared_diff_lat_mu(const Field& x) {
    x.request_spec();
    Field out(x.g);
    const Grid* g = x.g;
    for (int m = 0; m <= g->L; m++)
        for (int n = m; n <= g->L; n++)
            out.spec[g->idx(n, m)] = ((-n + 1.0) * Id::R(n - 1, m)) * x.spec_get(n - 1, m) +
                                      ((n + 2.0) * Id::S(n + 1, m)) * x.spec_get(n + 1, m);
    SPEC_OUT(out);
    return out;
}
Field Ops::mu(const Field& x) {
    x.request_spec();
    Field out(x.g);
    const Grid* g = x.g;
    for (int m = 0; m <= g->L; m++)
        for (int n = m; n <= g->L; n++)
            out.spec[g->idx(n, m)] = Id::R(n - 1, m) * x.spec_get(n - 1, m) + Id::S(n + 1, m) * x.spec_get(n + 1, m);
    SPEC_OUT(out);
    return out;
}
Field Ops::mu2(const Field& x) {
    x.request_spec();
    Field out(x.g);
    const Grid* g = x.g;
    for (int m = 0; m <= g->L; m++)
        for (int n = m; n <= g->L; n++)
            out.spec[g->idx(n, m)] = +Id::A(n - 2, m) * x.spec_get(n - 2, m) + Id::B(n + 0, m) * x.spec_get(n + 0, m) +
                                      Id::C(n + 2, m) * x.spec_get(n + 2, m);
    SPEC_OUT(out);
    return out;
}
Field Ops::grad_lon(const Field& x) {
    x.request_spec();
    Field out = diff_lon(x);
    out.request_spat();
    out.spat_update_lambda_gaussian_grid([](double, double mu, double& d) { d /= std::sqrt(1.0 - mu * mu); });
    return out;
}
Field Ops::grad_lat(const Field& x) {
    Field out = spec_one_minus_mu_squared_diff_lat_mu(x);
    out.request_spat();
    out.spat_update_lambda_gaussian_grid([](double, double mu, double& d) { d /= std::sqrt(1.0 - mu * mu); });
    return out;
}
Field Ops::div_lat(const Field& x) {
    Field out(x);
    out.spat_update_lambda_cogaussian_grid([](double, double c, double& d) { d *= c; });
    out = grad_lat(out);
    out.spat_update_lambda_cogaussian_grid([](double, double c, double& d) { d /= c; });
    return out;
}
Field Ops::diff_lat_mu(const Field& x) {
    Field out = spec_one_minus_mu_squared_diff_lat_mu(x);
    out.spat_update_lambda_gaussian_grid([](double, double mu, double& d) { d /= (1.0 - mu * mu); });
    return out;
}
Field Ops::laplace(const Field& x) {
    x.request_spec();
    Field out(x);
    out.spec_update_lambda([](int n, int, cplx& d) { d *= -(double)n * ((double)n + 1.0); });
    return out;
}
Field Ops::robert_div_lon(const Field& x) {
    Field out = diff_lon(x);
    out.spat_update_lambda_cogaussian_grid([](double, double c, double& d) { d /= c * c; });
    return out;
}
Field Ops::robert_div_lat(const Field& x) {
    Field out = spec_one_minus_mu_squared_diff_lat_mu(x);
    out.spat_update_lambda_cogaussian_grid([](double, double c, double& d) { d /= c * c; });
    return out;
}

// ============================================================ complex operators
CField OpsC::diff_lon(const CField& x) {
    x.request_spec();
    CField out(x.g);
    const Grid* g = x.g;
    for (int n = 0; n <= g->L; n++)
        for (int m = -n; m <= n; m++) out.spec[g->cidx(n, m)] = x.spec[g->cidx(n, m)] * cplx(0, m);
    SPEC_OUT(out);
    return out;
}
CField OpsC::spec_one_minus_mu_squared_diff_lat_mu(const CField& x) {
    x.request_spec();
    CField out(x.g);
    const Grid* g = x.g;
    for (int n = 0; n <= g->L; n++)
        for (int m = -n; m <= n; m++)
            out.spec[g->cidx(n, m)] = ((-n + 1.0) * Id::R(n - 1, m)) * x.spec_get(n - 1, m) +
                                       ((n + 2.0) * Id::S(n + 1, m)) * x.spec_get(n + 1, m);
    SPEC_OUT(out);
    return out;
}
CField OpsC::mu(const CField& x) {
    x.request_spec();
    CField out(x.g);
    const Grid* g = x.g;
    for (int n = 0; n <= g->L; n++)
        for (int m = -n; m <= n; m++)
            out.spec[g->cidx(n, m)] = Id::R(n - 1, m) * x.spec_get(n - 1, m) + Id::S(n + 1, m) * x.spec_get(n + 1, m);
    SPEC_OUT(out);
    return out;
}
CField OpsC::mu2(const CField& x) {
    x.request_spec();
    CField out(x.g);
    const Grid* g = x.g;
    for (int n = 0; n <= g->L; n++)
        for (int m = -n; m <= n; m++)
            out.spec[g->cidx(n, m)] = +Id::A(n - 2, m) * x.spec_get(n - 2, m) + Id::B(n + 0, m) * x.spec_get(n + 0, m) +
                                       Id::C(n + 2, m) * x.spec_get(n + 2, m);
    SPEC_OUT(out);
    return out;
}
CField OpsC::grad_lon(const CField& x) {
    CField out = diff_lon(x);
    out.spat_update_lambda_gaussian_grid([](double, double mu, cplx& d) { d /= std::sqrt(1.0 - mu * mu); });
    return out;
}
CField OpsC::grad_lat(const CField& x) {
    CField out = spec_one_minus_mu_squared_diff_lat_mu(x);
    out.request_spat();
    out.spat_update_lambda_gaussian_grid([](double, double mu, cplx& d) { d /= std::sqrt(1.0 - mu * mu); });
    return out;
}
CField OpsC::div_lat(const CField& x) {
    CField out(x);
    out.spat_update_lambda_cogaussian_grid([](double, double c, cplx& d) { d *= c; });
    out = grad_lat(out);
    // SPHOperatorsComplex.hpp:327-333 divides by cos(phi) from the latitude angle
    out.spat_update_lambda([](double, double phi, cplx& d) { d /= std::cos(phi); });
    return out;
}
CField OpsC::laplace(const CField& x) {
    x.request_spec();
    CField out(x);
    out.spec_update_lambda([](int n, int, cplx& d) { d *= -(double)n * ((double)n + 1.0); });
    return out;
}
CField OpsC::robert_div(const CField& lon, const CField& lat) {
    CField out = diff_lon(lon) + spec_one_minus_mu_squared_diff_lat_mu(lat);
    out.spat_update_lambda_cogaussian_grid([](double, double c, cplx& d) { d /= c * c; });
    return out;
}

// ============================================================ banded LU (zgbtf2 + zgbtrs)
static inline double cabs1(const cplx& z) { return std::fabs(z.real()) + std::fabs(z.imag()); }

int gbsv(int n, int kl, int ku, cplx* ab, int ldab, int* ipiv, cplx* b) {
    if (n <= 0) return 0;
    const int kv = ku + kl;
    // 1-based accessor into GB storage
    auto AB = [&](int i, int j) -> cplx& { return ab[(size_t)(i - 1) + (size_t)(j - 1) * ldab]; };
    auto B = [&](int i) -> cplx& { return b[i - 1]; };
    int info = 0;
    for (int j = ku + 2; j <= std::min(kv, n); j++)
        for (int i = kv - j + 2; i <= kl; i++) AB(i, j) = 0;
    int ju = 1;
    for (int j = 1; j <= n; j++) {
        if (j + kv <= n)
            for (int i = 1; i <= kl; i++) AB(i, j + kv) = 0;
        const int km = std::min(kl, n - j);
        int jp = 1;
        double best = cabs1(AB(kv + 1, j));
        for (int t = 2; t <= km + 1; t++) {
            double v = cabs1(AB(kv + t, j));
            if (v > best) { best = v; jp = t; }
        }
        ipiv[j - 1] = jp + j - 1;
        if (AB(kv + jp, j) != cplx(0)) {
            ju = std::max(ju, std::min(j + ku + jp - 1, n));
            if (jp != 1) {
                for (int c = 0; c <= ju - j; c++) std::swap(AB(kv + jp - c, j + c), AB(kv + 1 - c, j + c));
            }
            if (km > 0) {
                const cplx rp = cplx(1.0) / AB(kv + 1, j);
                for (int i = 1; i <= km; i++) AB(kv + 1 + i, j) *= rp;
                for (int c = 1; c <= ju - j; c++) {
                    const cplx y = AB(kv + 1 - c, j + c);
                    if (y != cplx(0))
                        for (int i = 1; i <= km; i++) AB(kv + 1 + i - c, j + c) -= AB(kv + 1 + i, j) * y;
                }
            }
        } else if (info == 0) {
            info = j;
        }
    }
    if (info != 0) return info;
    // forward: L with row interchanges
    if (kl > 0) {
        for (int j = 1; j <= n - 1; j++) {
            const int lm = std::min(kl, n - j);
            const int l = ipiv[j - 1];
            if (l != j) std::swap(B(l), B(j));
            const cplx bj = B(j);
            for (int i = 1; i <= lm; i++) B(j + i) -= AB(kv + 1 + i, j) * bj;
        }
    }
    // backward: U (kl+ku super-diagonals)
    for (int j = n; j >= 1; j--) {
        if (B(j) != cplx(0)) {
            B(j) /= AB(kv + 1, j);
            const cplx t = B(j);
            for (int i = std::max(1, j - kv); i <= j - 1; i++) B(i) -= t * AB(kv + 1 + i - j, j);
        }
    }
    return 0;
}

// ============================================================ SolverC
void SolverC::setup(const Grid* g_, int halo_) {
    g = g_;
    halo = halo_;
    ndiag = 2 * halo + 1;
    rows.assign((size_t)g->ncplx * ndiag, cplx(0));
}
// rows of block m (m = -L..L) are contiguous, n = |m|..L (SPHConfig.hpp:136-156)
size_t SolverC::ncompact(int n, int m) const {
    const int L = g->L;
    size_t off;
    if (m < 0) off = (size_t)(L + m) * (L + m + 1) / 2;
    else off = (size_t)L * (L + 1) / 2 + (size_t)m * (2 * L - m + 3) / 2;
    return off + (size_t)(n - std::abs(m));
}
// SPHMatrixComplex.hpp:181-206 (guard compares against m, not |m|; entries that
// fall outside the block are stored and later ignored by the band conversion)
void SolverC::add(cplx* row, int n, int m, int rel, const cplx& v) {
    if (n < m) return;
    const int n2 = n + rel;
    if (n2 < 0 || n2 < m || n2 > g->L) return;
    row[rel + halo] += v;
}
#define FOR_ROWS for (int m = -g->L; m <= g->L; m++) for (int n = std::abs(m); n <= g->L; n++)
void SolverC::scalar_phi(const cplx& v) { FOR_ROWS { add(row(n, m), n, m, 0, v); } }
void SolverC::mu_phi(const cplx& s) {
    FOR_ROWS {
        cplx* r = row(n, m);
        add(r, n, m, -1, Id::R(n - 1, m) * s);
        add(r, n, m, +1, Id::S(n + 1, m) * s);
    }
}
void SolverC::one_minus_mu_mu_diff_mu_phi() {
    FOR_ROWS {
        cplx* r = row(n, m);
        add(r, n, m, -1, (-(double)n + 1.0) * Id::R(n - 1, m));
        add(r, n, m, +1, ((double)n + 2.0) * Id::S(n + 1, m));
    }
}
void SolverC::z2(const cplx& s, double) {
    FOR_ROWS {
        cplx* r = row(n, m);
        add(r, n, m, -2, s * Id::A(n - 2, m));
        add(r, n, m, 0, s * Id::B(n, m));
        add(r, n, m, +2, s * Id::C(n + 2, m));
    }
}
void SolverC::z3(const cplx& s, double) {
    using I = Id;
    FOR_ROWS {
        cplx* r = row(n, m);
        add(r, n, m, -4, s * (I::A(n - 2, m) * I::A(n - 4.0, m)));
        add(r, n, m, -2, s * (I::A(n - 2, m) * I::B(n - 2, m) + I::B(n, m) * I::A(n - 2, m)));
        add(r, n, m, 0, s * (I::A(n - 2, m) * I::C(n, m) + I::B(n, m) * I::B(n, m) + I::C(n + 2, m) * I::A(n, m)));
        add(r, n, m, +2, s * (I::B(n, m) * I::C(n + 2, m) + I::C(n + 2, m) * I::B(n + 2, m)));
        add(r, n, m, +4, s * (I::C(n + 2, m) * I::C(n + 4, m)));
    }
}
void SolverC::z4(const cplx& s, double r_) {
    FOR_ROWS { add(row(n, m), n, m, 0, 1.0 / (r_ * r_) * s * cplx(0, m)); }
}
void SolverC::z4robert(const cplx& s, double r_) {
    for (int m = -g->L; m <= g->L; m++) {
        const cplx fac = 1.0 / (r_ * r_) * s * cplx(0, m);
        for (int n = std::abs(m); n <= g->L; n++) {
            cplx* r = row(n, m);
            add(r, n, m, -2, -fac * Id::A(n - 2, m));
            add(r, n, m, 0, -fac * Id::B(n, m) + fac);
            add(r, n, m, +2, -fac * Id::C(n + 2, m));
        }
    }
}
void SolverC::z5(const cplx& s, double r_) {
    FOR_ROWS {
        const cplx fac = 1.0 / (r_ * r_) * s * cplx(0, m);
        cplx* r = row(n, m);
        add(r, n, m, -2, fac * Id::A(n - 2, m));
        add(r, n, m, 0, fac * Id::B(n + 0, m));
        add(r, n, m, +2, fac * Id::C(n + 2, m));
    }
}
void SolverC::z5robert(const cplx& s, double r_) {
    using I = Id;
    for (int m = -g->L; m <= g->L; m++) {
        const cplx fac = 1.0 / (r_ * r_) * s * cplx(0, m);
        for (int n = std::abs(m); n <= g->L; n++) {
            cplx* r = row(n, m);
            // SPHSolverComplex.hpp:305-309 places all five terms at offset -2;
            // fix_z5robert puts them at -4,-2,0,+2,+4.
            const int o[5] = {fix_z5robert ? -4 : -2, -2, fix_z5robert ? 0 : -2, fix_z5robert ? 2 : -2, fix_z5robert ? 4 : -2};
            add(r, n, m, o[0], -fac * (I::A(n - 2, m) * I::A(n - 4, m)));
            add(r, n, m, o[1], -fac * (I::A(n - 2, m) * I::B(n - 2, m) + I::B(n, m) * I::A(n - 2, m)) + fac * I::A(n - 2, m));
            add(r, n, m, o[2], -fac * (I::A(n - 2, m) * I::C(n, m) + I::B(n, m) * I::B(n, m) + I::C(n + 2, m) * I::A(n, m)) + fac * I::B(n, m));
            add(r, n, m, o[3], -fac * (I::B(n, m) * I::C(n + 2, m) + I::C(n + 2, m) * I::B(n + 2, m)) + fac * I::C(n + 2, m));
            add(r, n, m, o[4], -fac * (I::C(n + 2, m) * I::C(n + 4, m)));
        }
    }
}
void SolverC::z6(const cplx& s, double r_) {
    using I = Id;
    FOR_ROWS {
        cplx* r = row(n, m);
        add(r, n, m, -2, -1.0 / (r_ * r_) * s * (I::D(n - 1, m) * I::R(n - 2, m) + (I::E(n, m) - 3.0) * I::A(n - 2, m)));
        add(r, n, m, 0, -1.0 / (r_ * r_) * s * (1.0 + I::D(n - 1, m) * I::S(n, m) + (I::E(n, m) - 3.0) * I::B(n, m)));
        add(r, n, m, +2, -1.0 / (r_ * r_) * s * (I::E(n, m) - 3.0) * I::C(n + 2, m));
    }
}
void SolverC::z6robert(const cplx& s_, double r_) {
    using I = Id;
    for (int m = -g->L; m <= g->L; m++) {
        const cplx s = 1.0 / (r_ * r_) * s_ * (double)m;
        for (int n = std::abs(m); n <= g->L; n++) {
            cplx* r = row(n, m);
            const double gr = I::G(n - 1, m) * I::R(n - 2, m);
            const double gs = I::G(n - 1, m) * I::S(n, m) + I::H(n + 1, m) * I::R(n, m);
            const double hs = I::H(n + 1, m) * I::S(n + 2, m);
            add(r, n, m, -2, s * gr);
            add(r, n, m, 0, s * gs);
            add(r, n, m, +2, s * hs);
            add(r, n, m, -4, s * (-I::A(n - 4, m) * gr));
            add(r, n, m, -2, s * (-I::B(n - 2, m) * gr));
            add(r, n, m, 0, s * (-I::C(n + 0, m) * gr));
            add(r, n, m, -2, s * (-I::A(n - 2, m) * gs));
            add(r, n, m, 0, s * (-I::B(n + 0, m) * gs));
            add(r, n, m, +2, s * (-I::C(n + 2, m) * gs));
            add(r, n, m, 0, s * (-I::A(n + 0, m) * hs));
            add(r, n, m, +2, s * (-I::B(n + 2, m) * hs));
            add(r, n, m, +4, s * (-I::C(n + 4, m) * hs));
        }
    }
}
void SolverC::z7(const cplx& s, double r_) {
    FOR_ROWS { add(row(n, m), n, m, 0, -1.0 / (r_ * r_) * s * (double)n * ((double)n + 1.0)); }
}
void SolverC::z8(const cplx& s, double r_) {
    FOR_ROWS {
        cplx* r = row(n, m);
        add(r, n, m, 0, 1.0 / (r_ * r_) * s * 2.0);
        const double fac = -1.0 / (r_ * r_) * ((double)m * m - (double)n * (n + 1.0));
        add(r, n, m, -2, s * fac * Id::A(n - 2, m));
        add(r, n, m, 0, s * fac * Id::B(n, m));
        add(r, n, m, +2, s * fac * Id::C(n + 2, m));
    }
}
CField SolverC::apply(const CField& x) const {
    x.request_spec();
    CField out(g);
    for (int n = 0; n <= g->L; n++)
        for (int m = -n; m <= n; m++) {
            const cplx* r = &rows[ncompact(n, m) * ndiag];
            cplx acc = 0;
            for (int d = 0; d < ndiag; d++) {
                const int n2 = n + d - halo;
                if (n2 < 0 || n2 < std::abs(m) || n2 > g->L) continue;
                acc += r[d] * x.spec_get(n2, m);
            }
            out.spec[g->cidx(n, m)] = acc;
        }
    SPEC_OUT(out);
    return out;
}
CField SolverC::solve(const CField& rhs) const {
    rhs.request_spec();
    CField out(g);
    const int L = g->L;
    const int ldab = 3 * halo + 1;
    std::vector<cplx> ab((size_t)ldab * (L + 1));
    std::vector<cplx> b(L + 1);
    std::vector<int> ipiv(L + 1);
    for (int m = -L; m <= L; m++) {
        const int am = std::abs(m);
        const int N = L + 1 - am;
        const cplx* blk = &rows[ncompact(am, m) * ndiag];
        std::fill(ab.begin(), ab.end(), cplx(0));
        for (int i = 0; i < N; i++)
            for (int d = 0; d < ndiag; d++) {
                const int j = i + d - halo;
                if (j < 0 || j >= N) continue;
                ab[(size_t)(2 * halo + i - j) + (size_t)j * ldab] = blk[(size_t)i * ndiag + d];
            }
        for (int i = 0; i < N; i++) b[i] = rhs.spec[g->cidx(am + i, m)];
        int info = gbsv(N, halo, halo, ab.data(), ldab, ipiv.data(), b.data());
        if (info != 0) throw std::runtime_error("banded solve: singular matrix");
        for (int i = 0; i < N; i++) out.spec[g->cidx(am + i, m)] = b[i];
    }
    SPEC_OUT(out);
    return out;
}

// ============================================================ REXI coefficients
// Gaussian-approximation weights a_l (L=11) and mean mu of
// T. Haut, T. Babb, P. Martinsson, B. Wingate, "A high-order time-parallel
// scheme for solving wave propagation problems via the direct construction of
// an approximate time-evolution operator", IMA J. Numer. Anal. 36 (2016);
// the same table as GaussianApproximation.hpp:51-81.
static const double GA_MU = -4.315321510875024;
static const double GA_A[23][2] = {
    {-1.0845749544592896e-7, 2.77075431662228e-8},
    {1.858753344202957e-8, -9.105375434750162e-7},
    {3.6743713227243024e-6, 7.073284346322969e-7},
    {-2.7990058083347696e-6, 0.0000112564827639346},
    {0.000014918577548849352, -0.0000316278486761932},
    {-0.0010751767283285608, -0.00047282220513073084},
    {0.003816465653840016, 0.017839810396560574},
    {0.12124105653274578, -0.12327042473830248},
    {-0.9774980792734348, -0.1877130220537587},
    {1.3432866123333178, 3.2034715228495942},
    {4.072408546157305, -6.123755543580666},
    {-9.442699917778205, 0.},
    {4.072408620272648, 6.123755841848161},
    {1.3432860877712938, -3.2034712658530275},
    {-0.9774985292598916, 0.18771238018072134},
    {0.1212417070363373, 0.12326987628935386},
    {0.0038169724770333343, -0.017839242222443888},
    {-0.0010756025812659208, 0.0004731874917343858},
    {0.000014713754789095218, 0.000031358475831136815},
    {-2.659323898804944e-6, -0.000011341571201752273},
    {3.6970377676364553e-6, -6.517457477594937e-7},
    {3.883933649142257e-9, 9.128496023863376e-7},
    {-1.0816457995911385e-7, -2.954309729192276e-8}};

void Rexi::setup(double h, int M, int L_, bool half) {
    const int L = (L_ == 0) ? 11 : L_;
    if (L != 11) throw std::runtime_error("only L=11 Gaussian approximation is available");
    const int N = M + L;
    alpha.assign(2 * N + 1, cplx(0));
    beta_re.assign(2 * N + 1, cplx(0));
    beta_im.assign(2 * N + 1, cplx(0));
    // b_m = e^{h^2} e^{-i m h} (ExponentialApproximation.hpp:122)
    std::vector<cplx> b(2 * M + 1);
    for (int m = -M; m <= M; m++) b[m + M] = std::exp(h * h) * std::exp(-cplx(0, 1) * ((double)m * h));
    for (int l = -L; l <= L; l++)
        for (int m = -M; m <= M; m++) {
            const int n = l + m;
            const cplx a(GA_A[l + L][0], GA_A[l + L][1]);
            alpha[n + N] = h * (cplx(GA_MU, 0) + cplx(0, n));
            beta_re[n + N] += b[m + M].real() * h * a;
            beta_im[n + N] += b[m + M].imag() * h * a;
        }
    if (half) {
        alpha.resize(N + 1);
        beta_re.resize(N + 1);
        beta_im.resize(N + 1);
        for (int i = 0; i < N; i++) { beta_re[i] *= 2.0; beta_im[i] *= 2.0; }
    }
}

cplx Rexi::approx_e_ix(double x) const {
    double re = 0, im = 0;
    for (size_t n = 0; n < alpha.size(); n++) {
        const cplx d = cplx(0, x) + alpha[n];
        re += (beta_re[n] / d).real();
        im += (beta_im[n] / d).real();
    }
    return cplx(re, im);
}

// ============================================================ REXI SWE solver
void RexiSWE::setup(const Grid* g_, const cplx& a_, const cplx& b_, double radius, double omega_,
                    double avg_geopot_, double tau_, bool coriolis_, bool robert_, bool fix_z5) {
    g = g_;
    robert = robert_;
    coriolis = coriolis_;
    tau = tau_;
    alpha = a_ / tau;
    beta = b_ / tau;
    r = radius;
    ir = 1.0 / r;
    omega = omega_;
    two_omega = 2.0 * omega;
    avg_geopot = avg_geopot_;
    phi_solver.setup(g, 4);
    phi_solver.fix_z5robert = fix_z5;
    const cplx A = alpha;
    const double T = two_omega, P = avg_geopot;
    phi_solver.z1((A * A) * (A * A), r);
    if (coriolis) {
        phi_solver.z2(2.0 * T * T * A * A, r);
        phi_solver.z3((T * T) * (T * T), r);
        if (robert) {
            phi_solver.z4robert(-P * A * T, r);
            phi_solver.z5robert(P / A * T * T * T, r);
            phi_solver.z6robert(P * 2.0 * T * T, r);
        } else {
            phi_solver.z4(-P * A * T, r);
            phi_solver.z5(P / A * T * T * T, r);
            phi_solver.z6(P * 2.0 * T * T, r);
        }
    }
    phi_solver.z7(-P * A * A, r);
    if (coriolis) phi_solver.z8(-P * T * T, r);
    vel_solver.setup(g, 2);
    vel_solver.z1(A * A, r);
    if (coriolis) vel_solver.z2(T * T, r);
}

void RexiSWE::solve(const Field& i_phi0, const Field& i_u0, const Field& i_v0, Field& o_phi, Field& o_u, Field& o_v) const {
    using op = OpsC;
    CField mu(g);
    mu.spat_update_lambda_gaussian_grid([](double, double m, cplx& d) { d = m; });
    CField phi0(i_phi0);
    CField u0(i_u0);
    CField v0(i_v0);
    const cplx a = alpha;
    const double T = two_omega, P = avg_geopot;
    CField div0 = robert ? ir * op::robert_div(u0, v0) : ir * op::div(u0, v0);
    CField eta0 = robert ? ir * op::robert_vort(u0, v0) : ir * op::vort(u0, v0);
    CField phi(g), u(g), v(g);
    if (coriolis) {
        CField lat_mu = robert ? op::robert_grad_lat(mu) : op::grad_lat(mu);
        CField Fc_k = T * ir * lat_mu * (-(a * a * u0 - T * T * op::mu2(u0)) + 2.0 * a * T * op::mu(v0));
        CField foo = P * (div0 - T * (1.0 / a) * op::mu(eta0)) + (a * CField(i_phi0) + T * T * (1.0 / a) * op::mu2(CField(i_phi0)));
        CField rhs = a * a * foo + T * T * op::mu2(foo) + (P / a) * Fc_k;
        phi = phi_solver.solve(rhs);
        CField A_ = u0 + ir * (robert ? op::robert_grad_lon(phi) : op::grad_lon(phi));
        CField B_ = v0 + ir * (robert ? op::robert_grad_lat(phi) : op::grad_lat(phi));
        CField rhsa = a * A_ - T * op::mu(B_);
        CField rhsb = T * op::mu(A_) + a * B_;
        u = vel_solver.solve(rhsa);
        v = vel_solver.solve(rhsb);
    } else {
        CField rhs = P * div0 + a * CField(i_phi0);
        phi = rhs.spec_solve_helmholtz(a * a, -P, r);
        u = (1.0 / a) * (u0 + ir * (robert ? op::robert_grad_lon(phi) : op::grad_lon(phi)));
        v = (1.0 / a) * (v0 + ir * (robert ? op::robert_grad_lat(phi) : op::grad_lat(phi)));
    }
    phi *= beta;
    u *= beta;
    v *= beta;
    phi.spat_RealToSPHData(o_phi);
    u.spat_RealToSPHData(o_u);
    v.spat_RealToSPHData(o_v);
}

// ============================================================ SWE tendency + RK4
void swe_tendency(const SWEParams& p, const Field& fdata, const Field& i_h, const Field& i_u, const Field& i_v,
                  Field& o_h_t, Field& o_u_t, Field& o_v_t) {
    using op = Ops;
    auto f = [&](const Field& x) { return fdata * x * 2.0 * p.omega; };
    if (!p.nonlinear) {
        if (!p.robert) {
            o_h_t = -(op::div_lon(i_u) + op::div_lat(i_v)) * (p.h0 / p.a);
            o_u_t = -op::grad_lon(i_h) * (p.g / p.a);
            o_v_t = -op::grad_lat(i_h) * (p.g / p.a);
        } else {
            o_h_t = -(op::robert_div_lon(i_u) + op::robert_div_lat(i_v)) * (p.h0 / p.a);
            o_u_t = -op::robert_grad_lon(i_h) * (p.g / p.a);
            o_v_t = -op::robert_grad_lat(i_h) * (p.g / p.a);
        }
        if (p.omega != 0) {
            o_u_t += f(i_v);
            o_v_t -= f(i_u);
        }
    } else {
        o_h_t = -(op::div_lon(i_h * i_u) + op::div_lat(i_h * i_v)) * (1.0 / p.a);
        o_u_t = -op::grad_lon(i_h) * (p.g / p.a);
        o_v_t = -op::grad_lat(i_h) * (p.g / p.a);
        if (p.omega != 0) {
            o_u_t += f(i_v);
            o_v_t -= f(i_u);
        }
        o_u_t -= (i_u * op::grad_lon(i_u) + i_v * op::grad_lat(i_u)) * (1.0 / p.a);
        o_v_t -= (i_u * op::grad_lon(i_v) + i_v * op::grad_lat(i_v)) * (1.0 / p.a);
    }
    if (p.visc != 0) {
        const double s = p.visc / (p.a * p.a);
        o_h_t += op::laplace(i_h) * s;
        o_u_t += op::laplace(i_u) * s;
        o_v_t += op::laplace(i_v) * s;
    }
}

void swe_rk4_step(const SWEParams& p, const Field& fdata, Field& h, Field& u, Field& v, double dt) {
    const Grid* g = h.g;
    Field h1(g), u1(g), v1(g), h2(g), u2(g), v2(g), h3(g), u3(g), v3(g), h4(g), u4(g), v4(g);
    const double b[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    swe_tendency(p, fdata, h, u, v, h1, u1, v1);
    swe_tendency(p, fdata, h + dt * (0.5 * h1), u + dt * (0.5 * u1), v + dt * (0.5 * v1), h2, u2, v2);
    swe_tendency(p, fdata, h + dt * (0.5 * h2), u + dt * (0.5 * u2), v + dt * (0.5 * v2), h3, u3, v3);
    swe_tendency(p, fdata, h + dt * (1.0 * h3), u + dt * (1.0 * u3), v + dt * (1.0 * v3), h4, u4, v4);
    h += dt * ((b[0] * h1) + (b[1] * h2) + (b[2] * h3) + (b[3] * h4));
    u += dt * ((b[0] * u1) + (b[1] * u2) + (b[2] * u3) + (b[3] * u4));
    v += dt * ((b[0] * v1) + (b[1] * v2) + (b[2] * v3) + (b[3] * v4));
}

}  // namespace orc
