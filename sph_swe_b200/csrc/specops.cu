// Spectral-space operators on the packed (l, m) layouts: the coefficient
// loops of SPHOperators / SPHOperatorsComplex / SPHData (reference
// SPHOperators.hpp:30-54, 234-333, 482-498; SPHData.hpp:231-497).
// One thread per coefficient, consecutive threads along n for a fixed m
// (contiguous in the real layout), recurrence neighbours n-2..n+2 read from
// L1/L2 (each is another thread's own coefficient).  Memory bound.
#include "common.cuh"
#include "identities.cuh"

namespace sphgpu {

// Real layout: block row y pairs the orders y and L - y (L + 2 coefficients
// together; for even L the middle order L / 2 alone), so that every row of
// blocks is about as long and few threads idle (one row per order left half
// of them idle at T255).  Complex layout: block row y is the order y - L.
// A thread takes one (n, m) of every field (fields blockIdx.z, + gridDim.z,
// ...): the recurrence coefficients of (n, m) and the Helmholtz reciprocal
// are formed once and reused across the fields.
__global__ void k_spec_op(int op, const double2* __restrict__ in, long long ld_in, double2* __restrict__ out,
                          long long ld_out, double2 a, double2 b, int L, int cplx, int batch) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int m, n;
    if (cplx) {
        m = (int)blockIdx.y - L;
        n = (m < 0 ? -m : m) + i;
    } else {
        const int y = blockIdx.y, len0 = L + 1 - y;
        if (i < len0) {
            m = y;
            n = y + i;
        } else {
            m = L - y;
            if (m == y) return;
            n = m + (i - len0);
        }
    }
    if (n > L) return;
    const int am = m < 0 ? -m : m;
    const long long k = cplx ? cidx(n, m) : pidx(L, n, m);
    const double dn = n, dm = m;
    // index of coefficient (n + d, m), or -1 outside the truncation
    auto nb = [&](int d) -> long long {
        const int nn = n + d;
        if (nn < am || nn > L) return -1;
        return cplx ? (long long)cidx(nn, m) : k + d;
    };
    auto at = [&](const double2* x, long long q) -> double2 { return q < 0 ? make_double2(0, 0) : x[q]; };
    // the coefficients of this (n, m): y = c0 x(n - d) + c1 x(n) + c2 x(n + d), or as noted
    double c0 = 0, c1 = 0, c2 = 0;
    long long klo = -1, khi = -1;
    double2 z = make_double2(0, 0);
    switch (op) {
        case SPH_OP_DIFF_LON: break;  // i m x
        case SPH_OP_D1MU2:
            klo = nb(-1), khi = nb(1);
            c0 = (-dn + 1.0) * idR(dn - 1, dm);
            c2 = (dn + 2.0) * idS(dn + 1, dm);
            break;
        case SPH_OP_MU:
            klo = nb(-1), khi = nb(1);
            c0 = idR(dn - 1, dm);
            c2 = idS(dn + 1, dm);
            break;
        case SPH_OP_MU2:
            klo = nb(-2), khi = nb(2);
            c0 = idA(dn - 2, dm);
            c1 = idB(dn, dm);
            c2 = idC(dn + 2, dm);
            break;
        case SPH_OP_LAPLACE: c1 = -dn * (dn + 1.0); break;
        case SPH_OP_HELMHOLTZ: {  // x / (a - b n (n + 1))
            const double2 d = make_double2(a.x - b.x * dn * (dn + 1.0), a.y - b.y * dn * (dn + 1.0));
            const double den = d.x * d.x + d.y * d.y;
            z = make_double2(d.x / den, -d.y / den);
            break;
        }
        case SPH_OP_SCALE:
        case SPH_OP_AXPY: z = a; break;
        default: return;
    }
    for (int f = blockIdx.z; f < batch; f += gridDim.z) {
        const double2* x = in + (long long)f * ld_in;
        double2* y = out + (long long)f * ld_out;
        double2 r;
        switch (op) {
            case SPH_OP_DIFF_LON: {
                const double2 v = x[k];
                r = make_double2(-dm * v.y, dm * v.x);
                break;
            }
            case SPH_OP_D1MU2:
            case SPH_OP_MU: {
                const double2 lo = at(x, klo), hi = at(x, khi);
                r = make_double2(c0 * lo.x + c2 * hi.x, c0 * lo.y + c2 * hi.y);
                break;
            }
            case SPH_OP_MU2: {
                const double2 lo = at(x, klo), mid = x[k], hi = at(x, khi);
                r = make_double2(c0 * lo.x + c1 * mid.x + c2 * hi.x, c0 * lo.y + c1 * mid.y + c2 * hi.y);
                break;
            }
            case SPH_OP_LAPLACE: {
                const double2 v = x[k];
                r = make_double2(v.x * c1, v.y * c1);
                break;
            }
            case SPH_OP_AXPY: {
                const double2 v = x[k], o = y[k];
                r = make_double2(o.x + z.x * v.x - z.y * v.y, o.y + z.x * v.y + z.y * v.x);
                break;
            }
            default: {  // HELMHOLTZ, SCALE: z x
                const double2 v = x[k];
                r = make_double2(z.x * v.x - z.y * v.y, z.x * v.y + z.y * v.x);
                break;
            }
        }
        y[k] = r;
    }
}

int spec_op(const Handle* h, int op, const double2* in, long long ld_in, double2* out, long long ld_out, double2 a,
            double2 b, int batch, int cplx, cudaStream_t s) {
    if (op < 0 || op > SPH_OP_AXPY) {
        set_error("sph_spec_op: unknown operator");
        return SPH_ERR_ARG;
    }
    if (batch <= 0) return SPH_OK;
    if (batch > 65535) {
        set_error("sph_spec_op: batch too large");
        return SPH_ERR_ARG;
    }
    const int L = h->L;
    // up to 16 field slices; each thread then loops over batch / 16 fields
    const dim3 grid(cplx ? (L + 1 + 63) / 64 : (L + 2 + 63) / 64, cplx ? 2 * L + 1 : (L + 2) / 2, std::min(batch, 16));
    k_spec_op<<<grid, 64, 0, s>>>(op, in, ld_in, out, ld_out, a, b, L, cplx, batch);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// Real packed spectra of truncation Ls -> truncation Ld, field by field
// (SPHData::spec_copyToDifferentModes, SPHData.hpp:108-187): coefficients
// with n <= min(Ls, Ld) are copied, the others of the output are zero.  Grid
// (m of the output, field); threads along n.
__global__ void k_spec_copy_modes(const double2* __restrict__ src, int Ls, long long lds, double2* __restrict__ dst,
                                  int Ld, long long ldd) {
    const int m = blockIdx.x;
    const double2* x = src + (long long)blockIdx.y * lds;
    double2* y = dst + (long long)blockIdx.y * ldd;
    for (int n = m + threadIdx.x; n <= Ld; n += blockDim.x)
        y[pidx(Ld, n, m)] = (n <= Ls) ? x[pidx(Ls, n, m)] : make_double2(0, 0);
}

int spec_copy_modes(const Handle* hs, const double2* src, long long lds, const Handle* hd, double2* dst,
                    long long ldd, int batch, cudaStream_t s) {
    if (batch <= 0) return SPH_OK;
    if (batch > 65535) {
        set_error("sph_spec_copy_modes: batch too large");
        return SPH_ERR_ARG;
    }
    k_spec_copy_modes<<<dim3(hd->L + 1, batch), 128, 0, s>>>(src, hs->L, lds, dst, hd->L, ldd);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

}  // namespace sphgpu
