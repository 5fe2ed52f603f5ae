// Elementwise operations on grid (physical-space) arrays, the device side of
// the SPHData / SPHDataComplex grid operators:
//   operator*(const SPHData&)            SPHData.hpp:334-353 (product of two grids)
//   operator+/-/* with scalars on grids, spat_set_value / spat_set_zero
//                                         SPHData.hpp:768-798
//   operator*(const SPHDataComplex&)     SPHDataComplex.hpp:321-340 (full-grid
//                                         product; the reference's loop bound
//                                         stops at (L+1)^2, see the defect note)
#include "common.cuh"

#include <algorithm>

namespace sphgpu {

// one thread per element (vectorised over a grid-stride loop)
__global__ void k_spat_op(int op, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ out,
                          double alpha, double beta, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        switch (op) {
            case SPH_SPAT_MUL:
                out[i] = alpha * x[i] * y[i];
                break;
            case SPH_SPAT_AXPBY:
                out[i] = alpha * x[i] + (y ? beta * y[i] : 0.0);
                break;
            case SPH_SPAT_FILL:
                out[i] = alpha;
                break;
            case SPH_SPAT_ADD_CONST:
                out[i] = x[i] + alpha;
                break;
            default: {  // SPH_SPAT_CMUL: complex elements, n counts complex numbers
                const double2 a = reinterpret_cast<const double2*>(x)[i], b = reinterpret_cast<const double2*>(y)[i];
                reinterpret_cast<double2*>(out)[i] =
                    make_double2(alpha * (a.x * b.x - a.y * b.y), alpha * (a.x * b.y + a.y * b.x));
            }
        }
    }
}

}  // namespace sphgpu

extern "C" int sph_spat_op(sph_handle* h, int op, const double* x, const double* y, double* out, double alpha,
                           double beta, long long n, void* stream) {
    using namespace sphgpu;
    if (!h) {
        set_error("sph_spat_op: NULL handle");
        return SPH_ERR_ARG;
    }
    if (op < SPH_SPAT_MUL || op > SPH_SPAT_CMUL || n < 0 || !out ||
        ((op == SPH_SPAT_MUL || op == SPH_SPAT_CMUL) && (!x || !y)) ||
        ((op == SPH_SPAT_AXPBY || op == SPH_SPAT_ADD_CONST) && !x)) {
        set_error("sph_spat_op: bad arguments");
        return SPH_ERR_ARG;
    }
    if (n == 0) return SPH_OK;
    const int threads = 256;
    const long long blocks = std::min<long long>((n + threads - 1) / threads, 148LL * 16);
    k_spat_op<<<(int)blocks, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(op, x, y, out, alpha, beta, n);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}
