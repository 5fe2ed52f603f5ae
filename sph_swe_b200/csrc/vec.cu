// Vector transforms: vorticity/divergence spectra <-> velocity grids on the
// unit sphere, built from the scalar Legendre/FFT stages with the meridional
// derivative kept exact (degree L+1 retained, Legendre range lmax = L+1):
//
//   synthesis  psi = lap^-1 vort, chi = lap^-1 div
//              U = u c = d chi/d lambda - (1-mu^2) d psi/d mu
//              V = v c = d psi/d lambda + (1-mu^2) d chi/d mu
//   analysis   with U' = U/c^2, V' = V/c^2 and a_l(.) the degree-(L+1) analysis
//              (taken as c U' under the weights w / c),
//              vort_l = i m a_l(V') + (l+1) e_l a_{l-1}(U') - l e_{l+1} a_{l+1}(U')
//              div_l  = i m a_l(U') - (l+1) e_l a_{l-1}(V') + l e_{l+1} a_{l+1}(V')
//              (integration by parts of d/dmu; exact by Gauss quadrature)
// with (1-mu^2) dP_l/dmu = (l+1) e_l P_{l-1} - l e_{l+1} P_{l+1},
// e_l = R(l-1, m), e_{l+1} = S(l+1, m) of SPHIdentities.hpp:52-86.
// The reference has no vector transform; its scalar operators grad/div/vort
// (SPHOperators.hpp:100-119, 339-529) are the truncated counterparts.
#include "common.cuh"
#include "identities.cuh"

namespace sphgpu {

// Thread layout of the two coefficient kernels below (packed layout of degree
// K): block row y takes the orders y and K - y (K + 2 coefficients together;
// for even K the middle order alone), so that rows are about equally long; a
// thread takes one (n, m) of every field (fields blockIdx.z, + gridDim.z, ...)
// and forms its recurrence coefficients once.  Returns false past the row.
__device__ __forceinline__ bool vec_nm(int K, int& n, int& m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, len0 = K + 1 - y;
    if (i < len0) {
        m = y;
        n = y + i;
    } else {
        m = K - y;
        if (m == y) return false;
        n = m + (i - len0);
    }
    return n <= K;
}

// vort/div (degree L) -> [U, V] spectra of degree L+1
__global__ void k_vec_prep(const double2* __restrict__ vort, const double2* __restrict__ div, long long ld,
                           double2* __restrict__ X, int L, int nlmp, int batch) {
    const int Lp = L + 1;
    int n, m;
    if (!vec_nm(Lp, n, m)) return;
    const int k = pidx(Lp, n, m);
    // lap^-1 factor of degree nn and the packed index of (nn, m) in degree L (-1: none)
    auto slot = [&](int nn, double& sc) -> int {
        if (m > L || nn < m || nn > L || nn == 0) {
            sc = 0.0;
            return -1;
        }
        sc = -1.0 / ((double)nn * (nn + 1.0));
        return pidx(L, nn, m);
    };
    double s0, sl, sh;
    const int k0 = slot(n, s0), kl = slot(n - 1, sl), kh = slot(n + 1, sh);
    const double dn = n, dm = m;
    const double cl = m > L ? 0.0 : (-dn + 1.0) * idR(dn - 1, dm), ch = m > L ? 0.0 : (dn + 2.0) * idS(dn + 1, dm);
    auto ld2 = [](const double2* x, int q, double sc) -> double2 {
        if (q < 0) return make_double2(0, 0);
        const double2 v = x[q];
        return make_double2(v.x * sc, v.y * sc);
    };
    for (int b = blockIdx.z; b < batch; b += gridDim.z) {
        double2* U = X + (size_t)b * 2 * nlmp;
        double2* V = U + nlmp;
        const double2* z = vort + (size_t)b * ld;
        const double2* d = div + (size_t)b * ld;
        const double2 psi = ld2(z, k0, s0), chi = ld2(d, k0, s0);
        const double2 psl = ld2(z, kl, sl), psh = ld2(z, kh, sh), chl = ld2(d, kl, sl), chh = ld2(d, kh, sh);
        // U = i m chi - Dex psi ; V = i m psi + Dex chi (zero at m = L + 1)
        U[k] = make_double2(-dm * chi.y - (cl * psl.x + ch * psh.x), dm * chi.x - (cl * psl.y + ch * psh.y));
        V[k] = make_double2(-dm * psi.y + (cl * chl.x + ch * chh.x), dm * psi.x + (cl * chl.y + ch * chh.y));
    }
}

// F[f][m][j] *= c_j^(-p)
__global__ void k_fourier_scale(double2* __restrict__ F, long long ldF, int mF, int nlat,
                                const double* __restrict__ cosphi, int p) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long fou = (long long)mF * nlat;
    if (idx >= fou) return;
    const int j = (int)(idx % nlat);
    const double c = cosphi[j];
    const double s = p == 1 ? 1.0 / c : 1.0 / (c * c);
    double2* f = F + (long long)blockIdx.y * ldF + idx;
    const double2 v = *f;
    *f = make_double2(v.x * s, v.y * s);
}

// a(U'), a(V') of degree L+1 -> vort, div of degree L
__global__ void k_vec_post(const double2* __restrict__ A, int nlmp, double2* __restrict__ vort, double2* __restrict__ div,
                           long long ld, int L, int batch) {
    int n, m;
    if (!vec_nm(L, n, m)) return;
    const int Lp = L + 1;
    auto slot = [&](int nn) -> int { return (nn < m || nn > Lp) ? -1 : pidx(Lp, nn, m); };
    const int q0 = slot(n), ql = slot(n - 1), qh = slot(n + 1);
    const double dn = n, dm = m;
    const double el = (dn + 1.0) * idR(dn - 1, dm), eh = dn * idS(dn + 1, dm);
    const int k = pidx(L, n, m);
    auto at = [](const double2* x, int q) -> double2 { return q < 0 ? make_double2(0, 0) : x[q]; };
    for (int b = blockIdx.z; b < batch; b += gridDim.z) {
        const double2* aU = A + (size_t)b * 2 * nlmp;
        const double2* aV = aU + nlmp;
        const double2 u0 = at(aU, q0), ul = at(aU, ql), uh = at(aU, qh);
        const double2 v0 = at(aV, q0), vl = at(aV, ql), vh = at(aV, qh);
        vort[(size_t)b * ld + k] = make_double2(-dm * v0.y + el * ul.x - eh * uh.x, dm * v0.x + el * ul.y - eh * uh.y);
        div[(size_t)b * ld + k] = make_double2(-dm * u0.y - el * vl.x + eh * vh.x, dm * u0.x - el * vl.y + eh * vh.y);
    }
}

}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

int sph_vec_SH_to_spat(sph_handle* hh, const double* vort, const double* div, double* u, double* v, int batch,
                       int robert, void* stream) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || batch < 0 || (batch > 0 && (!vort || !div || !u || !v))) {
        set_error("sph_vec_SH_to_spat: bad arguments");
        return SPH_ERR_ARG;
    }
    if (batch == 0) return SPH_OK;
    if (batch > 32767) { set_error("sph_vec_SH_to_spat: batch too large"); return SPH_ERR_ARG; }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int L = h->L, Lp = L + 1, mF = L + 1;
    const int nlmp = (Lp + 1) * (Lp + 2) / 2;
    const long long ldF = (long long)mF * h->nlat;
    const size_t xbytes = sizeof(double2) * 2 * (size_t)nlmp * batch;
    const size_t fbytes = sizeof(double2) * 2 * (size_t)ldF * batch;
    if (int rc = ensure_workspace(h, xbytes + fbytes)) return rc;
    double2* X = static_cast<double2*>(h->ws);
    double2* F = reinterpret_cast<double2*>(static_cast<char*>(h->ws) + xbytes);
    k_vec_prep<<<dim3((Lp + 2 + 63) / 64, (Lp + 2) / 2, std::min(batch, 16)), 64, 0, s>>>(
        reinterpret_cast<const double2*>(vort), reinterpret_cast<const double2*>(div), h->nlm, X, L, nlmp, batch);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = legendre_synthesis_real(h, X, nlmp, Lp, F, ldF, 2 * batch, s, 1)) return rc;
    // outputs: member b -> u (field 2b) and v (field 2b+1) written to separate
    // arrays; velocities u = U / cos phi: the ring synthesis divides its
    // output rings (Robert form: U, V as they are)
    for (int c = 0; c < 2; c++) {
        const int srcs[1] = {c};
        if (int rc = ring_synthesis_real(h, F, ldF, mF, c == 0 ? u : v, h->nspat, batch, srcs, nullptr, 1, 2, s,
                                         robert ? nullptr : h->cosphi))
            return rc;
    }
    return SPH_OK;
}

int sph_vec_spat_to_SH(sph_handle* hh, const double* u, const double* v, double* vort, double* div, int batch,
                       int robert, void* stream) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || batch < 0 || (batch > 0 && (!vort || !div || !u || !v))) {
        set_error("sph_vec_spat_to_SH: bad arguments");
        return SPH_ERR_ARG;
    }
    if (batch == 0) return SPH_OK;
    if (batch > 32767) { set_error("sph_vec_spat_to_SH: batch too large"); return SPH_ERR_ARG; }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int L = h->L, Lp = L + 1, mF = L + 1;
    const int nlmp = (Lp + 1) * (Lp + 2) / 2;
    const long long ldF = (long long)mF * h->nlat;
    const size_t xbytes = sizeof(double2) * 2 * (size_t)nlmp * batch;
    const size_t fbytes = sizeof(double2) * 2 * (size_t)ldF * batch;
    if (int rc = ensure_workspace(h, xbytes + fbytes)) return rc;
    double2* A = static_cast<double2*>(h->ws);
    double2* F = reinterpret_cast<double2*>(static_cast<char*>(h->ws) + xbytes);
    // Fourier of u into fields 2b, of v into 2b+1
    if (int rc = ring_analysis_real(h, u, h->nspat, F, 2 * ldF, mF, batch, s)) return rc;
    if (int rc = ring_analysis_real(h, v, h->nspat, F + ldF, 2 * ldF, mF, batch, s)) return rc;
    // the integrands U' = U / c^2 are analysed with the weights w / c from
    // c U' = U / c: u itself for velocities, U / c for the Robert form.  Both
    // stay bounded at the polar rings, which keeps the per-column scales of the
    // mixed form at the field's magnitude rather than at 1 / c there
    if (robert) {
        k_fourier_scale<<<dim3((unsigned)((ldF + 255) / 256), 2 * batch), 256, 0, s>>>(F, ldF, mF, h->nlat, h->cosphi, 1);
        SPH_CUDA_TRY(cudaGetLastError());
    }
    if (int rc = legendre_analysis_real(h, F, ldF, A, nlmp, Lp, 2 * batch, s, 1)) return rc;
    k_vec_post<<<dim3((L + 2 + 63) / 64, (L + 2) / 2, std::min(batch, 16)), 64, 0, s>>>(
        A, nlmp, reinterpret_cast<double2*>(vort), reinterpret_cast<double2*>(div), h->nlm, L, batch);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

}  // extern "C"
