// Spectral-space operators on the packed (l, m) layouts: the coefficient
// loops of SPHOperators / SPHOperatorsComplex / SPHData (reference
// SPHOperators.hpp:30-54, 234-333, 482-498; SPHData.hpp:231-497).
// One thread per coefficient, consecutive threads along n for a fixed m
// (contiguous in the real layout), recurrence neighbours n-2..n+2 read from
// L1/L2.  Memory bound.
#include "common.cuh"
#include "identities.cuh"

namespace sphgpu {

__device__ __forceinline__ double2 spec_at(const double2* __restrict__ x, int cplx, int L, int n, int m) {
    const int am = m < 0 ? -m : m;
    if (n < 0 || n > L || am > n) return make_double2(0, 0);
    return x[cplx ? cidx(n, m) : pidx(L, n, m)];
}

__global__ void k_spec_op(int op, const double2* __restrict__ in, long long ld_in, double2* __restrict__ out,
                          long long ld_out, double2 a, double2 b, int L, int cplx) {
    const int m = cplx ? (int)blockIdx.y - L : (int)blockIdx.y;
    const int am = m < 0 ? -m : m;
    const int n = am + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const int f = blockIdx.z;
    const double2* x = in + (long long)f * ld_in;
    double2* y = out + (long long)f * ld_out;
    const long long k = cplx ? cidx(n, m) : pidx(L, n, m);
    const double dn = n, dm = m;
    double2 r;
    switch (op) {
        case SPH_OP_DIFF_LON: {
            const double2 v = x[k];
            r = make_double2(-dm * v.y, dm * v.x);
            break;
        }
        case SPH_OP_D1MU2: {
            const double2 lo = spec_at(x, cplx, L, n - 1, m), hi = spec_at(x, cplx, L, n + 1, m);
            const double cl = (-dn + 1.0) * idR(dn - 1, dm), ch = (dn + 2.0) * idS(dn + 1, dm);
            r = make_double2(cl * lo.x + ch * hi.x, cl * lo.y + ch * hi.y);
            break;
        }
        case SPH_OP_MU: {
            const double2 lo = spec_at(x, cplx, L, n - 1, m), hi = spec_at(x, cplx, L, n + 1, m);
            const double cl = idR(dn - 1, dm), ch = idS(dn + 1, dm);
            r = make_double2(cl * lo.x + ch * hi.x, cl * lo.y + ch * hi.y);
            break;
        }
        case SPH_OP_MU2: {
            const double2 lo = spec_at(x, cplx, L, n - 2, m), mid = x[k], hi = spec_at(x, cplx, L, n + 2, m);
            const double ca = idA(dn - 2, dm), cb = idB(dn, dm), cc = idC(dn + 2, dm);
            r = make_double2(ca * lo.x + cb * mid.x + cc * hi.x, ca * lo.y + cb * mid.y + cc * hi.y);
            break;
        }
        case SPH_OP_LAPLACE: {
            const double2 v = x[k];
            const double s = -dn * (dn + 1.0);
            r = make_double2(v.x * s, v.y * s);
            break;
        }
        case SPH_OP_HELMHOLTZ: {
            const double2 v = x[k];
            const double2 d = make_double2(a.x - b.x * dn * (dn + 1.0), a.y - b.y * dn * (dn + 1.0));
            const double den = d.x * d.x + d.y * d.y;
            r = make_double2((v.x * d.x + v.y * d.y) / den, (v.y * d.x - v.x * d.y) / den);
            break;
        }
        case SPH_OP_SCALE: {
            const double2 v = x[k];
            r = make_double2(a.x * v.x - a.y * v.y, a.x * v.y + a.y * v.x);
            break;
        }
        case SPH_OP_AXPY: {
            const double2 v = x[k], o = y[k];
            r = make_double2(o.x + a.x * v.x - a.y * v.y, o.y + a.x * v.y + a.y * v.x);
            break;
        }
        default:
            return;
    }
    y[k] = r;
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
    dim3 grid((L + 1 + 127) / 128, cplx ? 2 * L + 1 : L + 1, batch);
    k_spec_op<<<grid, 128, 0, s>>>(op, in, ld_in, out, ld_out, a, b, L, cplx);
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
