// Recurrence coefficients of the mu-multiplication and (1-mu^2) d/dmu
// identities for orthonormal associated Legendre functions,
//   mu P_n^m = R(n-1,m) P_{n-1}^m... expressed exactly as the reference's
// SPHIdentities (SPHIdentities.hpp:17-103): same arguments (doubles), same
// zero conventions outside |m| <= n, so that spectral operators and band
// matrices match it coefficient for coefficient.
#pragma once

#include <cmath>

#ifndef __CUDACC__
#define __host__
#define __device__
using std::sqrt;
#endif

namespace sphgpu {

__host__ __device__ inline double idR(double k, double m) {
    const double n = k + 1;
    const double am = m < 0 ? -m : m;
    if (n < 0 || n < am || n * n - m * m < 0) return 0.0;
    return sqrt((n * n - m * m) / (4.0 * n * n - 1.0));
}
__host__ __device__ inline double idS(double k, double m) {
    const double n = k - 1;
    const double am = m < 0 ? -m : m;
    if (n < 0 || n < am || n * n - m * m < 0) return 0.0;
    return sqrt(((n + 1.0) * (n + 1.0) - m * m) / ((2.0 * n + 1.0) * (2.0 * n + 3.0)));
}
__host__ __device__ inline double idA(double k, double m) {
    const double n = k + 2.0;
    return idR(n - 1, m) * idR(n - 2, m);
}
__host__ __device__ inline double idB(double n, double m) { return idR(n - 1, m) * idS(n, m) + idS(n + 1, m) * idR(n, m); }
__host__ __device__ inline double idC(double k, double m) {
    const double n = k - 2.0;
    return idS(n + 1, m) * idS(n + 2, m);
}
__host__ __device__ inline double idD(double k, double m) {
    const double n = k + 1;
    return (2.0 * n + 1.0) * sqrt((n * n - m * m) / (4.0 * n * n - 1.0));
}
__host__ __device__ inline double idE(double n, double) { return -n; }
__host__ __device__ inline double idG(double n, double m) {
    n = n + 1;
    return idD(n - 1, m) + idE(n, m) * idR(n - 1, m);
}
__host__ __device__ inline double idH(double n, double m) {
    n = n - 1;
    return idE(n, m) * idS(n + 1, m);
}

}  // namespace sphgpu
