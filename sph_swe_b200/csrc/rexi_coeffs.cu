// REXI coefficients (host code): the rational approximation
//   e^{i x} ~ sum_n beta_n / (i x + alpha_n)
// built from the L = 11 Gaussian approximation of a shifted Gaussian (weights
// a_l, mean mu) and the exponential sum e^{ix} = sum_m b_m G(x - m h),
// b_m = e^{h^2} e^{-i m h}.  With N = M + 11 and n = -N..N:
//   alpha_n = h (mu + i n),   beta_n = h sum_{l+m=n} b_m a_l
// where the real and the imaginary part of b_m give two weight sets (beta_re
// for the real part of e^{ix}, beta_im for the imaginary part).  The half-pole
// set keeps n = -N..0 and doubles the weights of n < 0.
// Follows REXI::setup (rexi/REXI.hpp:52-131), GaussianApproximation
// (rexi/GaussianApproximation.hpp:38-81) and ExponentialApproximation
// (rexi/ExponentialApproximation.hpp:49-124).
#include <complex>
#include <vector>

#include "common.cuh"

namespace {

// Gaussian-approximation weights a_l, l = -11..11, and mean mu: the published
// table of T. Haut, T. Babb, P. Martinsson, B. Wingate, IMA J. Numer. Anal. 36
// (2016), as tabulated in rexi/GaussianApproximation.hpp:51-81.
const double kGaMu = -4.315321510875024;
const double kGaA[23][2] = {
    {-1.0845749544592896e-7, 2.77075431662228e-8},      {1.858753344202957e-8, -9.105375434750162e-7},
    {3.6743713227243024e-6, 7.073284346322969e-7},      {-2.7990058083347696e-6, 0.0000112564827639346},
    {0.000014918577548849352, -0.0000316278486761932},  {-0.0010751767283285608, -0.00047282220513073084},
    {0.003816465653840016, 0.017839810396560574},       {0.12124105653274578, -0.12327042473830248},
    {-0.9774980792734348, -0.1877130220537587},         {1.3432866123333178, 3.2034715228495942},
    {4.072408546157305, -6.123755543580666},            {-9.442699917778205, 0.},
    {4.072408620272648, 6.123755841848161},             {1.3432860877712938, -3.2034712658530275},
    {-0.9774985292598916, 0.18771238018072134},         {0.1212417070363373, 0.12326987628935386},
    {0.0038169724770333343, -0.017839242222443888},     {-0.0010756025812659208, 0.0004731874917343858},
    {0.000014713754789095218, 0.000031358475831136815}, {-2.659323898804944e-6, -0.000011341571201752273},
    {3.6970377676364553e-6, -6.517457477594937e-7},     {3.883933649142257e-9, 9.128496023863376e-7},
    {-1.0816457995911385e-7, -2.954309729192276e-8}};
constexpr int kGaL = 11;

}  // namespace

extern "C" int sph_rexi_coefficients(double h, int M, int half, int cap, double* alpha, double* beta_re,
                                     double* beta_im, int* npoles) {
    using cplx = std::complex<double>;
    if (!(h > 0.0) || M < 1 || !npoles) {
        sphgpu::set_error("sph_rexi_coefficients: need h > 0, M >= 1 and an npoles pointer");
        return SPH_ERR_ARG;
    }
    const int N = M + kGaL;
    const int n_all = 2 * N + 1;
    const int n_out = half ? N + 1 : n_all;
    *npoles = n_out;
    if (cap == 0 && !alpha && !beta_re && !beta_im) return SPH_OK;  // size query
    if (cap < n_out || !alpha || !beta_re || !beta_im) {
        sphgpu::set_error("sph_rexi_coefficients: output capacity below the number of poles");
        return SPH_ERR_ARG;
    }
    std::vector<cplx> a(n_all), br(n_all, cplx(0.0)), bi(n_all, cplx(0.0));
    for (int n = -N; n <= N; n++) a[n + N] = h * cplx(kGaMu, (double)n);
    for (int m = -M; m <= M; m++) {
        const cplx b = std::exp(h * h) * std::exp(cplx(0.0, -(double)m * h));
        for (int l = -kGaL; l <= kGaL; l++) {
            const cplx w = h * cplx(kGaA[l + kGaL][0], kGaA[l + kGaL][1]);
            br[l + m + N] += b.real() * w;
            bi[l + m + N] += b.imag() * w;
        }
    }
    for (int i = 0; i < n_out; i++) {
        const double f = (half && i < N) ? 2.0 : 1.0;
        alpha[2 * i] = a[i].real();
        alpha[2 * i + 1] = a[i].imag();
        beta_re[2 * i] = f * br[i].real();
        beta_re[2 * i + 1] = f * br[i].imag();
        beta_im[2 * i] = f * bi[i].real();
        beta_im[2 * i + 1] = f * bi[i].imag();
    }
    return SPH_OK;
}
