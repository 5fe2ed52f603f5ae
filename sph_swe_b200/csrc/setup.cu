// Grid set-up on the device in FP64: Gauss-Legendre nodes/weights and the
// orthonormal associated Legendre table (SHTNS shtns_set_grid equivalent,
// called from SPHConfig::setup / setupAutoPhysicalSpace, SPHConfig.hpp:324-399).
#include "common.cuh"

#include <vector>

#include <cmath>
#include <cstring>

namespace sphgpu {

// One thread per northern node k: Newton iteration on P_n from the Tricomi
// start cos(pi (k + 3/4) / (n + 1/2)); mirrored to the southern half.  Once a
// step is below 1e-14 the iteration is converged to within rounding after one
// more (quadratically convergent) step.
__global__ void k_gauss_nodes(int n, double* __restrict__ x, double* __restrict__ w) {
    const int nh = (n + 1) / 2;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nh) return;
    double z = cos(kPi * (k + 0.75) / (n + 0.5));
    bool last = false;
    for (int it = 0; it < 100; it++) {
        double p0 = 1.0, p1 = z;
        for (int i = 2; i <= n; i++) {
            double p2 = ((2.0 * i - 1.0) * z * p1 - (i - 1.0) * p0) / i;
            p0 = p1;
            p1 = p2;
        }
        double dp = n * (z * p1 - p0) / (z * z - 1.0);
        double dz = p1 / dp;
        z -= dz;
        if (last) break;
        if (fabs(dz) < 1e-14) last = true;
    }
    double p0 = 1.0, p1 = z;
    for (int i = 2; i <= n; i++) {
        double p2 = ((2.0 * i - 1.0) * z * p1 - (i - 1.0) * p0) / i;
        p0 = p1;
        p1 = p2;
    }
    double dp = n * (z * p1 - p0) / (z * z - 1.0);
    double wk = 2.0 / ((1.0 - z * z) * dp * dp);
    x[k] = z;
    x[n - 1 - k] = -z;
    w[k] = wk;
    w[n - 1 - k] = wk;
}

__global__ void k_lat_tables(int n, const double* __restrict__ x, double* __restrict__ cosphi, double* __restrict__ lat) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double z = x[j];
    cosphi[j] = sqrt((1.0 - z) * (1.0 + z));
    lat[j] = 0.5 * kPi - acos(z);
}

// One thread per (latitude j, order m): P_m^m by the sin(theta) product with a
// carried power-of-two exponent (no underflow at high m), then the three-term
// recurrence in l up to lmax.  Coalesced: consecutive threads = consecutive j.
__global__ void k_plm(int nh, int mmax, int lmax, const double* __restrict__ x, const long long* __restrict__ poff,
                      double* __restrict__ plm) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (j >= nh || m > mmax) return;
    const double z = x[j];
    const double s = sqrt((1.0 - z) * (1.0 + z));
    const double BIG = 0x1p600, SMALL = 0x1p-600;
    double pmm = sqrt(1.0 / (4.0 * kPi));
    int e = 0;
    for (int k = 1; k <= m; k++) {
        pmm *= -sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
        if (fabs(pmm) < SMALL && pmm != 0.0) {
            pmm *= BIG;
            e -= 600;
        }
    }
    double* col = plm + poff[m] + j;
    double p0 = pmm;
    int el = e;
    col[0] = ldexp(p0, el);
    if (m + 1 > lmax) return;
    double p1 = z * sqrt(2.0 * m + 3.0) * p0;
    col[(size_t)nh] = ldexp(p1, el);
    for (int l = m + 2; l <= lmax; l++) {
        const double ll = l, mm = m;
        const double a = sqrt((4.0 * ll * ll - 1.0) / (ll * ll - mm * mm));
        const double b = sqrt(((ll - 1.0) * (ll - 1.0) - mm * mm) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0));
        const double p2 = a * (z * p1 - b * p0);
        p0 = p1;
        p1 = p2;
        if (el < 0 && fabs(p1) > BIG) {
            p0 *= SMALL;
            p1 *= SMALL;
            el += 600;
        }
        col[(size_t)(l - m) * nh] = ldexp(p1, el);
    }
}

int setup_tables(Handle* h) {
    const int n = h->nlat;
    SPH_CUDA_TRY(cudaMalloc(&h->mu, sizeof(double) * n));
    SPH_CUDA_TRY(cudaMalloc(&h->w, sizeof(double) * n));
    SPH_CUDA_TRY(cudaMalloc(&h->cosphi, sizeof(double) * n));
    SPH_CUDA_TRY(cudaMalloc(&h->lat, sizeof(double) * n));
    k_gauss_nodes<<<(h->nh + 127) / 128, 128>>>(n, h->mu, h->w);
    k_lat_tables<<<(n + 127) / 128, 128>>>(n, h->mu, h->cosphi, h->lat);
    SPH_CUDA_TRY(cudaGetLastError());

    const int mmax = h->L + 1, lmax = h->L + 1;
    h->poff_h.assign(mmax + 2, 0);
    long long off = 0;
    for (int m = 0; m <= mmax; m++) {
        h->poff_h[m] = off;
        off += (long long)(lmax - m + 1) * h->nh;
    }
    h->poff_h[mmax + 1] = off;
    SPH_CUDA_TRY(cudaMalloc(&h->poff, sizeof(long long) * (mmax + 2)));
    SPH_CUDA_TRY(cudaMemcpy(h->poff, h->poff_h.data(), sizeof(long long) * (mmax + 2), cudaMemcpyHostToDevice));
    SPH_CUDA_TRY(cudaMalloc(&h->plm, sizeof(double) * off));
    dim3 grid((h->nh + 127) / 128, mmax + 1);
    k_plm<<<grid, 128>>>(h->nh, mmax, lmax, h->mu, h->poff, h->plm);
    SPH_CUDA_TRY(cudaGetLastError());
    SPH_CUDA_TRY(cudaDeviceSynchronize());

    h->mu_h.resize(n);
    h->w_h.resize(n);
    h->cosphi_h.resize(n);
    h->lat_h.resize(n);
    SPH_CUDA_TRY(cudaMemcpy(h->mu_h.data(), h->mu, sizeof(double) * n, cudaMemcpyDeviceToHost));
    SPH_CUDA_TRY(cudaMemcpy(h->w_h.data(), h->w, sizeof(double) * n, cudaMemcpyDeviceToHost));
    SPH_CUDA_TRY(cudaMemcpy(h->cosphi_h.data(), h->cosphi, sizeof(double) * n, cudaMemcpyDeviceToHost));
    SPH_CUDA_TRY(cudaMemcpy(h->lat_h.data(), h->lat, sizeof(double) * n, cudaMemcpyDeviceToHost));
    // Gauss weights over cos(phi): the weights of analyses whose input carries
    // a factor cos(phi) that the integrand does not have (see legendre_analysis_real)
    std::vector<double> wc(n);
    for (int j = 0; j < n; j++) wc[j] = h->w_h[j] / h->cosphi_h[j];
    SPH_CUDA_TRY(cudaMalloc(&h->wc, sizeof(double) * n));
    SPH_CUDA_TRY(cudaMemcpy(h->wc, wc.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    return SPH_OK;
}

// ---------------------------------------------------------------- FFT plan
int fft_plan_init(FFTPlan* p, int n) {
    p->n = n;
    p->nrad = 0;
    int r = n;
    while (r % 4 == 0 && p->nrad < 16) { p->rad[p->nrad++] = 4; r /= 4; }
    while (r % 2 == 0 && p->nrad < 16) { p->rad[p->nrad++] = 2; r /= 2; }
    for (int q = 3; q <= 7 && r > 1; q += 2)
        while (r % q == 0 && p->nrad < 16) { p->rad[p->nrad++] = q; r /= q; }
    if (r != 1) {
        set_error("nphi must factor into radices 2, 3, 4, 5 and 7");
        return SPH_ERR_ARG;
    }
    std::vector<double2> tw(n);
    for (int t = 0; t < n; t++) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
        tw[t] = make_double2((double)cosl(a), (double)sinl(a));
    }
    SPH_CUDA_TRY(cudaMalloc(&p->tw, sizeof(double2) * n));
    SPH_CUDA_TRY(cudaMemcpy(p->tw, tw.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
    return SPH_OK;
}

void fft_plan_free(FFTPlan* p) {
    if (p->tw) cudaFree(p->tw);
    p->tw = nullptr;
}

}  // namespace sphgpu
