// REXI time integrator for the linear shallow-water equations, Robert
// formulation (SWERexiSPHRobert.hpp): FP64 direct, or (mixed form) complex
// FP32 banded factorisation and solves with two steps of FP64 iterative
// refinement (residuals of the FP64 system, corrections from the FP32 factors).
//
// Reference per step (AppSWE.hpp:414-566): for every pole (alpha_k, beta_k)
// SWERexiSPHRobert::solve (SWERexiSPHRobert.hpp:139-258) promotes phi0 = g h,
// u0, v0 to complex fields, builds a right-hand side from mu / mu^2 / (1-mu^2)d/dmu
// recurrences, solves one banded system per zonal wavenumber m for phi
// (9 diagonals, SPHSolverComplex + zgbsv), recovers u, v with two 5-diagonal
// solves, scales by beta and accumulates Re(.) of the result.
//
// Here every part that does not depend on the pole is computed once per step
// (the complex promotions, the divergence through one real synthesis /
// analysis pair, eta0, and the mu / mu^2 images), so that the right-hand side
// of a pole is a linear combination of 10 pole-independent vectors with
// alpha-dependent weights, and the Phi matrix is
//      A(alpha) = alpha^4 I + alpha^2 C2 + alpha C1 + alpha^-1 Cm1 + C0
// with pole-independent band matrices C (the reference's z1..z8 components,
// SPHSolverComplex.hpp:88-420, grouped by power of alpha).  All offsets are
// even, so each m-block splits into two l-parities: pentadiagonal (Phi) and
// tridiagonal (velocity) systems.  One warp handles one m-block for 32 poles
// (one pole per lane): assembly, LU with partial pivoting (LAPACK zgbtf2 pivot
// rule, |re|+|im|), back substitution, velocity recovery, beta scaling and a
// warp reduction over its poles.  A final kernel sums the pole groups and takes
// Re(.) spectrally: Q_lm = (A_lm + (-1)^m conj(A_l,-m)) / 2.
// The complex grid product of the Coriolis term is applied as the full-grid
// product (the reference multiplies only the first (L+1)^2 grid points,
// SPHDataComplex.hpp:333): Proj[(1-mu^2) G] = G - mu2(G).
#include "common.cuh"
#include "identities.cuh"
#include "rexi_tables.h"
#include "rexi_lane.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>

struct sph_rexi;

namespace sphgpu {

struct RexiPlan {
    Handle* h = nullptr;
    sph_rexi_params p{};
    int npoles = 0, ngroups = 0;
    double2* alpha = nullptr;   // alpha_k / tau
    double2* beta = nullptr;    // beta_k / tau
    double2* Cphi = nullptr;    // [4][ncplx][5]  (C2, C1, Cm1, C0), block (N-compact) rows
    double2* Cvel = nullptr;    // [ncplx][3]
    double* coef = nullptr;     // [ncplx][4]: R(n-1,m), S(n+1,m), (1-n)R(n-1,m), (n+2)S(n+1,m)
    double2* V = nullptr;       // [18][ncplx] block layout
    double2* part = nullptr;    // [ngroups][3][ncplx]
    double2* X = nullptr;       // nlm (real layout)
    double2* Xr = nullptr;      // nlm
    double2* F = nullptr;       // (L+1)*nlat
    int* flag = nullptr;        // bit0 non-finite h, bit1 singular pivot
    // factors of the banded systems, computed once at plan creation (FP64 form,
    // Coriolis case): planes of [ngroups][ncplx][32 lanes]
    double2* fphi = nullptr;    // 7 planes
    double2* fvel = nullptr;    // 4 planes
    float2* fphi32 = nullptr;   // mixed form: the same factors in complex FP32, 7 planes
    float2* fvel32 = nullptr;   // 4 planes
    signed char* pphi = nullptr;
    signed char* pvel = nullptr;
    long long plane = 0;
    // Robert form with stored factors: phi of every pole between the Phi and
    // the velocity phase, [pole group][block row][32 lanes]
    double2* PHr = nullptr;
    bool singular = false;      // a zero pivot met while factoring
    // non-Robert form (SWERexiSPH): per-pole phi and the spectra of its
    // grid-valued gradients, their Fourier buffer, real-layout prep buffers
    double2* PH = nullptr;      // [npoles][ncplx] phi (complex layout n*n+n+m)
    double2* XY = nullptr;      // [2][npoles][ncplx]: i m phi and D phi, then F(grad_lon phi), F(grad_lat phi)
    double2* FXY = nullptr;     // [2 npoles][2L+1][nlat]
    double2* Xs = nullptr;      // [8][nlm] real-layout spectra of the prep
    double2* Fs = nullptr;      // [4][L+1][nlat] Fourier buffers of the prep
    double* glp = nullptr;      // [nlat] grad_lat(mu) projected to degree L, on the rings
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double* state = nullptr;
    cudaStream_t stream = nullptr;
};

// factor every (pole, m-block, parity) system once into the stored FP32 planes (mixed form)
__global__ void __launch_bounds__(64) k_rexi_factor_f(RexiDev d) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int nblk = 2 * d.L + 1;
    if (warp >= nblk * d.ngroups) return;
    const int g = warp % d.ngroups, kk = warp / d.ngroups;
    const int m = (kk & 1) ? -((kk + 1) >> 1) : (kk >> 1);
    const int pole = g * 32 + lane;
    const bool valid = pole < d.npoles;
    const double2 a = d.alpha[valid ? pole : 0];
    const long long gl = (long long)g * d.ncplx * 32 + lane;
    if (!rexi_factor_lane_f(d, m, a, gl) && valid) atomicOr(d.flag, 2);
}

// factor every (pole, m-block, parity) system once into the stored planes
__global__ void __launch_bounds__(64) k_rexi_factor(RexiDev d) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int nblk = 2 * d.L + 1;
    if (warp >= nblk * d.ngroups) return;
    const int g = warp % d.ngroups, kk = warp / d.ngroups;
    const int m = (kk & 1) ? -((kk + 1) >> 1) : (kk >> 1);
    const int pole = g * 32 + lane;
    const bool valid = pole < d.npoles;
    const double2 a = d.alpha[valid ? pole : 0];
    const long long gl = (long long)g * d.ncplx * 32 + lane;
    if (!rexi_factor_lane(d, m, a, gl) && valid) atomicOr(d.flag, 2);
}

template <int MAXN, bool MIXED, bool STORED>
__global__ void __launch_bounds__(64) k_rexi_solve(RexiDev d) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int L = d.L;
    const int nblk = 2 * L + 1;
    if (warp >= nblk * d.ngroups) return;
    const int g = warp % d.ngroups, kk = warp / d.ngroups;
    const int m = (kk & 1) ? -((kk + 1) >> 1) : (kk >> 1);  // 0, -1, 1, -2, 2, ...: largest blocks first
    const int N = L + 1 - (m < 0 ? -m : m);
    const int base = block_off(L, m);
    const int nc = d.ncplx;
    const int pole = g * 32 + lane;
    const bool valid = pole < d.npoles;
    const double2 a = d.alpha[valid ? pole : 0];
    const double2 bt = valid ? d.beta[pole] : make_double2(0, 0);
    double2 phi[MAXN], ra[MAXN], rb[MAXN];
    const long long gl = (long long)g * nc * 32 + lane;
    const bool ok = rexi_lane<MAXN, MIXED, STORED>(d, m, a, phi, ra, rb, gl);
    if (!ok && valid) atomicOr(d.flag, 2);
    // beta scaling and reduction over the 32 poles of this warp
    double2* outp = d.part + (size_t)g * 3 * nc;
    for (int i = 0; i < N; i++) {
        double2 v0 = c_mul(bt, phi[i]), v1 = c_mul(bt, ra[i]), v2 = c_mul(bt, rb[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0.x += __shfl_down_sync(0xffffffffu, v0.x, o);
            v0.y += __shfl_down_sync(0xffffffffu, v0.y, o);
            v1.x += __shfl_down_sync(0xffffffffu, v1.x, o);
            v1.y += __shfl_down_sync(0xffffffffu, v1.y, o);
            v2.x += __shfl_down_sync(0xffffffffu, v2.x, o);
            v2.y += __shfl_down_sync(0xffffffffu, v2.y, o);
        }
        if (lane == 0) {
            const int row = base + i;
            outp[row] = v0;
            outp[(size_t)nc + row] = v1;
            outp[(size_t)2 * nc + row] = v2;
        }
    }
}

// ------------------------------------------------------------ Robert form, stored factors
// The substitutions of k_rexi_solve<.., STORED> split into two launches of one
// warp per (pole group, m-block, l-parity), one pole per lane, so that no lane
// keeps the block's phi, u, v in local memory (that traffic, not the factor
// stream, bounded the single kernel): the Phi phase writes phi of its parity's
// rows to PH[group][block row][lane] (one coalesced 512-byte row per warp
// access) and sums beta phi over its poles; the velocity phase forms each
// row's right-hand sides from a window phi[i-2 .. i+2] of both parities read
// back from PH, solves, and sums beta u, beta v.  The arithmetic of every row
// is that of rexi_phi / rexi_lane.
// resident 64-thread blocks per SM asked of the compiler for the substitution
// kernels, which caps their registers: FP64 8 (at most 128 registers), mixed
// 16 (64 registers, some spills).  T127, M = 256, 535 poles: the mixed step
// took 1.58 ms with the compiler's own choice (166 / 96 registers), 1.34 ms
// at 16; the FP64 step is the same at 8 to 16.
template <bool MX>
constexpr int rx_minb() { return MX ? 16 : 8; }

__device__ __forceinline__ void rx_warp_index(const RexiDev& d, int warp, int& g, int& m, int& par) {
    par = warp & 1;
    const int w2 = warp >> 1;
    g = w2 % d.ngroups;
    const int kk = w2 / d.ngroups;
    m = (kk & 1) ? -((kk + 1) >> 1) : (kk >> 1);  // 0, -1, 1, -2, 2, ...: largest blocks first
}

// beta x summed over the 32 poles of the warp into *dst (lane 0 writes)
__device__ __forceinline__ void rx_warp_sum(double2 bt, double2 x, double2* dst, int lane) {
    double2 v = c_mul(bt, x);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    if (lane == 0) *dst = v;
}

template <int MAXN, bool MX>
__global__ void __launch_bounds__(64, rx_minb<MX>()) k_rexi_phi_st(RexiDev d, double2* __restrict__ PH) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int L = d.L;
    if (warp >= 2 * (2 * L + 1) * d.ngroups) return;
    int g, m, par;
    rx_warp_index(d, warp, g, m, par);
    const int N = L + 1 - (m < 0 ? -m : m);
    const int Np = (N - par + 1) >> 1;
    if (Np <= 0) return;
    const int base = block_off(L, m);
    const int nc = d.ncplx;
    const int pole = g * 32 + lane;
    const bool valid = pole < d.npoles;
    const double2 a = d.alpha[valid ? pole : 0];
    const double2 bt = valid ? d.beta[pole] : make_double2(0, 0);
    const double T = d.T, P = d.P, ir = d.ir;
    const double2 a2 = c_mul(a, a), a3 = c_mul(a2, a), a4 = c_mul(a2, a2);
    const double2 ainv = c_div(make_double2(1, 0), a);
    // right-hand side weights of the 10 pole-independent vectors (as rexi_phi)
    double2 sw[10];
    sw[0] = c_scale(a2, P);
    sw[1] = c_scale(a, -P * T);
    sw[2] = a3;
    sw[3] = c_scale(a, 2.0 * T * T);
    sw[4] = make_double2(T * T * P, 0);
    sw[5] = c_scale(ainv, -P * T * T * T);
    sw[6] = c_scale(ainv, T * T * T * T);
    sw[7] = c_scale(a, -P * T * ir);
    sw[8] = c_scale(ainv, P * T * T * T * ir);
    sw[9] = make_double2(2.0 * P * T * T * ir, 0);
    const double2* V = d.V;
    double2* ph = PH + ((long long)g * nc + base) * 32 + lane;
    double2* outp = d.part + (size_t)g * 3 * nc + base;
    auto rhs = [&](int k, int) -> double2 {
        const int row = base + par + 2 * k;
        double2 v = make_double2(0, 0);
#pragma unroll
        for (int q = 0; q < 10; q++) v = c_add(v, c_mul(sw[q], ld(&V[(size_t)q * nc + row])));
        return v;
    };
    auto out = [&](int k, int, double2 x) {
        const int i = par + 2 * k;
        ph[(long long)i * 32] = x;
        rx_warp_sum(bt, x, outp + i, lane);
    };
    const long long gl = (long long)g * nc * 32 + lane;
    if constexpr (MX) {
        auto entry = [&](int k, int dd) -> double2 { return phi_entry(d, base, par, a, a2, ainv, a4, k, dd); };
        band_solve_stored_mixed<2, (MAXN + 1) / 2, 1>(Np, band_ref_f(d.fphi32, d.pphi, d, gl, base, N, par), d.refine,
                                                     entry, rhs, out);
    } else {
        band_solve_stored<2, (MAXN + 1) / 2, 1>(Np, band_ref(d.fphi, d.pphi, d, gl, base, N, par), rhs, out);
    }
}

template <int MAXN, bool MX>
__global__ void __launch_bounds__(64, rx_minb<MX>()) k_rexi_vel_st(RexiDev d, const double2* __restrict__ PH) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int L = d.L;
    if (warp >= 2 * (2 * L + 1) * d.ngroups) return;
    int g, m, par;
    rx_warp_index(d, warp, g, m, par);
    const int N = L + 1 - (m < 0 ? -m : m);
    const int Np = (N - par + 1) >> 1;
    if (Np <= 0) return;
    const int base = block_off(L, m);
    const int nc = d.ncplx;
    const int pole = g * 32 + lane;
    const bool valid = pole < d.npoles;
    const double2 a = d.alpha[valid ? pole : 0];
    const double2 bt = valid ? d.beta[pole] : make_double2(0, 0);
    const double T = d.T, ir = d.ir, dm = m;
    const double2* V = d.V;
    const double2* ph = PH + ((long long)g * nc + base) * 32 + lane;
    double2* outp = d.part + (size_t)g * 3 * nc + base;
    auto P = [&](int i) -> double2 { return (i >= 0 && i < N) ? ph[(long long)i * 32] : make_double2(0, 0); };
    auto cf = [&](int i, int q) -> double { return RX_LDG(d.coef + (size_t)(base + i) * 4 + q); };
    // D phi of row i (truncated (1-mu^2) d/dmu), zero outside the block
    auto Dp = [&](int i) -> double2 {
        if (i < 0 || i >= N) return make_double2(0, 0);
        return c_add(c_scale(P(i - 1), cf(i, 2)), c_scale(P(i + 1), cf(i, 3)));
    };
    // rhsa = a u0 + a ir i m phi - T mu(v0) - T ir mu(D phi)
    // rhsb = T mu(u0) + T ir mu(i m phi) + a v0 + a ir D phi   (as rexi_lane)
    int last = -1;
    double2 xa = make_double2(0, 0), xb = make_double2(0, 0);
    auto rhs2 = [&](int k, int r) -> double2 {
        if (k != last) {
            const int i = par + 2 * k, row = base + i;
            const double Rl = cf(i, 0), Sh = cf(i, 1);
            const double2 dcur = Dp(i), dprev = Dp(i - 1), dnext = Dp(i + 1);
            const double2 pc = P(i), plo = P(i - 1), phi_hi = P(i + 1);
            const double2 mud = c_add(c_scale(dprev, Rl), c_scale(dnext, Sh));
            const double2 mup = c_add(c_scale(plo, Rl), c_scale(phi_hi, Sh));
            const double2 u0 = ld(&V[(size_t)10 * nc + row]), v0 = ld(&V[(size_t)11 * nc + row]);
            const double2 mv = ld(&V[(size_t)12 * nc + row]), mu0 = ld(&V[(size_t)13 * nc + row]);
            xa = c_mul(a, u0);
            xa = c_add(xa, c_mul(a, c_scale(c_im(pc, dm), ir)));
            xa = c_sub(xa, c_scale(mv, T));
            xa = c_sub(xa, c_scale(mud, T * ir));
            xb = c_scale(mu0, T);
            xb = c_add(xb, c_scale(c_im(mup, dm), T * ir));
            xb = c_add(xb, c_mul(a, v0));
            xb = c_add(xb, c_mul(a, c_scale(dcur, ir)));
            last = k;
        }
        return r == 0 ? xa : xb;
    };
    auto out2 = [&](int k, int r, double2 x) {
        const int i = par + 2 * k;
        rx_warp_sum(bt, x, outp + (size_t)(1 + r) * nc + i, lane);
    };
    const long long gl = (long long)g * nc * 32 + lane;
    if constexpr (MX) {
        const double2 a2 = c_mul(a, a);
        auto entry = [&](int k, int dd) -> double2 { return vel_entry(d, base, par, a2, k, dd); };
        band_solve_stored_mixed<1, (MAXN + 1) / 2, 2>(Np, band_ref_f(d.fvel32, d.pvel, d, gl, base, N, par), d.refine,
                                                     entry, rhs2, out2);
    } else {
        band_solve_stored<1, (MAXN + 1) / 2, 2>(Np, band_ref(d.fvel, d.pvel, d, gl, base, N, par), rhs2, out2);
    }
}

// ------------------------------------------------------------ non-Robert form (SWERexiSPH)
// Phase A: phi of every pole and m-block, written in the complex layout with
// i m phi and the truncated (1-mu^2) d phi/dmu, whose syntheses divided by
// cos phi are grad_lon(phi) and grad_lat(phi) (SPHOperatorsComplex.hpp:99-114,
// 223-249).
template <int MAXN, bool MIXED, bool STORED>
__global__ void __launch_bounds__(64) k_rexi_s0_phi(RexiDev d, double2* __restrict__ PH, double2* __restrict__ XY) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int L = d.L;
    if (warp >= (2 * L + 1) * d.ngroups) return;
    const int g = warp % d.ngroups, kk = warp / d.ngroups;
    const int m = (kk & 1) ? -((kk + 1) >> 1) : (kk >> 1);
    const int am = m < 0 ? -m : m;
    const int N = L + 1 - am;
    const int base = block_off(L, m);
    const int nc = d.ncplx;
    const int pole = g * 32 + lane;
    const bool valid = pole < d.npoles;
    const double2 a = d.alpha[valid ? pole : 0];
    double2 phi[MAXN];
    const long long gl = (long long)g * nc * 32 + lane;
    const bool ok = rexi_phi<MAXN, MIXED, STORED>(d, m, a, phi, gl);
    if (!ok && valid) atomicOr(d.flag, 2);
    if (!valid) return;
    double2* ph = PH + (size_t)pole * nc;
    double2* x = XY + (size_t)pole * nc;
    double2* y = XY + ((size_t)d.npoles + pole) * nc;
    for (int i = 0; i < N; i++) {
        const int n = am + i, ci = n * n + n + m;
        const double* cf = d.coef + (size_t)(base + i) * 4;
        const double2 lo = i > 0 ? phi[i - 1] : make_double2(0, 0);
        const double2 hi = i + 1 < N ? phi[i + 1] : make_double2(0, 0);
        ph[ci] = phi[i];
        x[ci] = c_im(phi[i], (double)m);
        y[ci] = c_add(c_scale(lo, __ldg(cf + 2)), c_scale(hi, __ldg(cf + 3)));
    }
}

// Phase B: velocity of every pole and m-block from the gradients' spectra,
// then beta scaling and the reduction over the 32 poles of the warp (as
// k_rexi_solve).
template <int MAXN, bool MIXED, bool STORED>
__global__ void __launch_bounds__(64) k_rexi_s0_vel(RexiDev d, const double2* __restrict__ PH,
                                                   const double2* __restrict__ XY) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int L = d.L;
    if (warp >= (2 * L + 1) * d.ngroups) return;
    const int g = warp % d.ngroups, kk = warp / d.ngroups;
    const int m = (kk & 1) ? -((kk + 1) >> 1) : (kk >> 1);
    const int am = m < 0 ? -m : m;
    const int N = L + 1 - am;
    const int base = block_off(L, m);
    const int nc = d.ncplx;
    const int pole = g * 32 + lane;
    const bool valid = pole < d.npoles;
    const int pc = valid ? pole : 0;
    const double2 a = d.alpha[pc];
    const double2 bt = valid ? d.beta[pole] : make_double2(0, 0);
    double2 ra[MAXN], rb[MAXN];
    const long long gl = (long long)g * nc * 32 + lane;
    const bool ok = rexi_s0_vel<MAXN, MIXED, STORED>(d, m, a, XY + (size_t)pc * nc, XY + ((size_t)d.npoles + pc) * nc,
                                                    ra, rb, gl);
    if (!ok && valid) atomicOr(d.flag, 2);
    const double2* ph = PH + (size_t)pc * nc;
    double2* outp = d.part + (size_t)g * 3 * nc;
    for (int i = 0; i < N; i++) {
        const int n = am + i;
        double2 v0 = c_mul(bt, ph[n * n + n + m]), v1 = c_mul(bt, ra[i]), v2 = c_mul(bt, rb[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0.x += __shfl_down_sync(0xffffffffu, v0.x, o);
            v0.y += __shfl_down_sync(0xffffffffu, v0.y, o);
            v1.x += __shfl_down_sync(0xffffffffu, v1.x, o);
            v1.y += __shfl_down_sync(0xffffffffu, v1.y, o);
            v2.x += __shfl_down_sync(0xffffffffu, v2.x, o);
            v2.y += __shfl_down_sync(0xffffffffu, v2.y, o);
        }
        if (lane == 0) {
            const int row = base + i;
            outp[row] = v0;
            outp[(size_t)nc + row] = v1;
            outp[(size_t)2 * nc + row] = v2;
        }
    }
}

// Fourier-space factors of the non-Robert projections (per latitude j, times
// 2 pi: synthesis -> analysis convention), c = sqrt(1 - mu^2):
//   mode 0: x c      (the cos(phi) factor of div_lat, SPHOperatorsComplex.hpp:300-312)
//   mode 1: x glp_j  (the Coriolis product with grad_lat(mu); see glp below)
//   mode 2: x / c    (grad_lon, grad_lat of the per-pole phi)
__global__ void k_s0_fscale(double2* __restrict__ F, long long n, int nlat, const double* __restrict__ mu,
                            const double* __restrict__ glp, int mode) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const int j = (int)(idx % nlat);
    const double z = mu[j];
    const double c = sqrt((1.0 - z) * (1.0 + z));
    const double f = 2.0 * kPi * (mode == 0 ? c : (mode == 1 ? glp[j] : 1.0 / c));
    F[idx] = make_double2(F[idx].x * f, F[idx].y * f);
}

// grad_lat(mu) as the Coriolis product of SWERexiSPH::solve uses it
// (SWERexiSPH.hpp:183-186): the grid field (1 - mu^2) / sqrt(1 - mu^2) is
// multiplied by the scalar two_omega * ir first, which takes it to spectral
// space (degree L) and back before the grid product, so the product sees its
// degree-L projection, not cos(phi) itself.  The field is zonal: the
// projection is the m = 0 Legendre analysis (Gauss weights, the 2 pi of the
// longitude quadrature) and synthesis with the orthonormal P_l^0, on the host.
static std::vector<double> s0_grad_lat_mu(const Handle* h) {
    const int L = h->L, nlat = h->nlat;
    std::vector<double> g0(nlat), out(nlat, 0.0), q(L + 1, 0.0);
    std::vector<double> P((size_t)(L + 1) * nlat);
    for (int j = 0; j < nlat; j++) {
        const double z = h->mu_h[j];
        g0[j] = (1.0 - z * z) / std::sqrt((1.0 - z) * (1.0 + z));
        double p0 = std::sqrt(1.0 / (4.0 * kPi)), p1 = z * std::sqrt(3.0) * p0;
        P[j] = p0;
        if (L >= 1) P[(size_t)nlat + j] = p1;
        for (int l = 2; l <= L; l++) {
            const double dl = l;
            const double al = std::sqrt((4.0 * dl * dl - 1.0) / (dl * dl));
            const double bl = std::sqrt(((dl - 1.0) * (dl - 1.0)) / (4.0 * (dl - 1.0) * (dl - 1.0) - 1.0));
            const double p2 = al * (z * p1 - bl * p0);
            p0 = p1;
            p1 = p2;
            P[(size_t)l * nlat + j] = p2;
        }
    }
    for (int l = 0; l <= L; l++)
        for (int j = 0; j < nlat; j++) q[l] += h->w_h[j] * 2.0 * kPi * g0[j] * P[(size_t)l * nlat + j];
    for (int l = 0; l <= L; l++)
        for (int j = 0; j < nlat; j++) out[j] += q[l] * P[(size_t)l * nlat + j];
    return out;
}

// div and eta of the non-Robert operators from the Fourier coefficients of
// F0 = I(i m u0), F1 = I(D w) with w = F(I(v0) cos phi), F2 = I(i m v0),
// F3 = I(D u0) (four consecutive fields of stride ldF): in place, field 0
// becomes div = div_lon(u0) + div_lat(v0) = F0/c + F1/(c cos(lat)) and field 1
// eta = grad_lon(v0) - grad_lat(u0) = (F2 - F3)/c (SPHOperatorsComplex.hpp:
// 99-114, 223-249, 283-335, 479-518), both times 2 pi
__global__ void k_s0_fdiveta(double2* __restrict__ F, long long ldF, int nlat, const double* __restrict__ mu,
                             const double* __restrict__ lat) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ldF) return;
    const int j = (int)(idx % nlat);
    const double z = mu[j];
    const double ic = 2.0 * kPi / sqrt((1.0 - z) * (1.0 + z)), icl = 1.0 / cos(lat[j]);
    const double2 f0 = F[idx], f1 = F[ldF + idx], f2 = F[2 * ldF + idx], f3 = F[3 * ldF + idx];
    F[idx] = make_double2((f0.x + f1.x * icl) * ic, (f0.y + f1.y * icl) * ic);
    F[ldF + idx] = make_double2((f2.x - f3.x) * ic, (f2.y - f3.y) * ic);
}

// ------------------------------------------------------------ pole-independent prep
// real packed (degree L) -> complex block layout, times s:
// c(n,m) = s x(n,m) for m >= 0, s (-1)^m conj(x(n,|m|)) for m < 0
__global__ void k_rx_complexify(const double2* __restrict__ x, double s, double2* __restrict__ out, int L) {
    const int m = (int)blockIdx.y - L;
    const int am = m < 0 ? -m : m;
    const int n = am + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    double2 v = x[pidx(L, n, am)];
    if (m < 0) v = make_double2((am & 1) ? -v.x : v.x, (am & 1) ? v.y : -v.y);
    out[brow(L, n, m)] = make_double2(v.x * s, v.y * s);
}

// block-layout operators: 0 mu, 1 mu2, 2 eta = ir (i m V - D U) (in = U, in2 = V),
// 3 lincomb out = x - y (in, in2)
__global__ void k_rx_block_op(int op, const double2* __restrict__ in, const double2* __restrict__ in2,
                              double2* __restrict__ out, int L, double ir) {
    const int m = (int)blockIdx.y - L;
    const int am = m < 0 ? -m : m;
    const int n = am + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const int base = block_off(L, m);
    auto at = [&](const double2* p, int nn) -> double2 {
        if (nn < am || nn > L) return make_double2(0, 0);
        return p[base + nn - am];
    };
    const double dn = n, dm = m;
    double2 r;
    if (op == 0) {
        const double cl = idR(dn - 1, dm), ch = idS(dn + 1, dm);
        const double2 lo = at(in, n - 1), hi = at(in, n + 1);
        r = make_double2(cl * lo.x + ch * hi.x, cl * lo.y + ch * hi.y);
    } else if (op == 1) {
        const double ca = idA(dn - 2, dm), cb = idB(dn, dm), cc = idC(dn + 2, dm);
        const double2 lo = at(in, n - 2), mid = at(in, n), hi = at(in, n + 2);
        r = make_double2(ca * lo.x + cb * mid.x + cc * hi.x, ca * lo.y + cb * mid.y + cc * hi.y);
    } else if (op == 2) {
        const double cl = (-dn + 1.0) * idR(dn - 1, dm), ch = (dn + 2.0) * idS(dn + 1, dm);
        const double2 ul = at(in, n - 1), uh = at(in, n + 1), v = at(in2, n);
        const double2 du = make_double2(cl * ul.x + ch * uh.x, cl * ul.y + ch * uh.y);
        r = make_double2(ir * (-dm * v.y - du.x), ir * (dm * v.x - du.y));
    } else {
        const double2 x = at(in, n), y = at(in2, n);
        r = make_double2(x.x - y.x, x.y - y.y);
    }
    out[base + n - am] = r;
}

// X = i m u + D v (real packed layout) from the state
__global__ void k_rx_divsrc(const double2* __restrict__ u, const double2* __restrict__ v, double2* __restrict__ X, int L) {
    const int m = blockIdx.y;
    const int n = m + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const double dn = n, dm = m;
    const double cl = (-dn + 1.0) * idR(dn - 1, dm), ch = (dn + 2.0) * idS(dn + 1, dm);
    const double2 lo = n - 1 >= m ? v[pidx(L, n - 1, m)] : make_double2(0, 0);
    const double2 hi = n + 1 <= L ? v[pidx(L, n + 1, m)] : make_double2(0, 0);
    const double2 uu = u[pidx(L, n, m)];
    X[pidx(L, n, m)] = make_double2(-dm * uu.y + cl * lo.x + ch * hi.x, dm * uu.x + cl * lo.y + ch * hi.y);
}

// Fourier-space F *= 2 pi / c^2 (synthesis -> analysis convention, / cos^2 phi)
__global__ void k_rx_fscale(double2* __restrict__ F, int nlat, int mF, const double* __restrict__ cosphi) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= mF * nlat) return;
    const double c = cosphi[idx % nlat];
    const double s = 2.0 * kPi / (c * c);
    F[idx] = make_double2(F[idx].x * s, F[idx].y * s);
}

// sum the pole groups, take Re(.) spectrally and write the real state:
// h = Re(phi)/g, u, v; optional implicit viscosity x / (1 + nu tau n(n+1)/r^2)
__global__ void k_rx_finish(const double2* __restrict__ part, int ngroups, int ncplx, double2* __restrict__ state,
                            int L, int nlm, double inv_g, double visc_fac, int* __restrict__ flag) {
    const int m = blockIdx.y;
    const int n = m + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const int rp = brow(L, n, m), rm = brow(L, n, -m);
    const double dn = n;
    const double vf = 1.0 / (1.0 + visc_fac * dn * (dn + 1.0));
    for (int f = 0; f < 3; f++) {
        double2 ap = make_double2(0, 0), amn = make_double2(0, 0);
        for (int g = 0; g < ngroups; g++) {
            const double2* p = part + ((size_t)g * 3 + f) * ncplx;
            ap = c_add(ap, p[rp]);
            amn = c_add(amn, p[rm]);
        }
        // (A(n,m) + (-1)^m conj(A(n,-m))) / 2
        const double sg = (m & 1) ? -1.0 : 1.0;
        double2 q = make_double2(0.5 * (ap.x + sg * amn.x), 0.5 * (ap.y - sg * amn.y));
        if (f == 0) q = make_double2(q.x * inv_g, q.y * inv_g);
        q = make_double2(q.x * vf, q.y * vf);
        if (f == 0 && !(isfinite(q.x) && isfinite(q.y))) atomicOr(flag, 1);
        state[(size_t)f * nlm + pidx(L, n, m)] = q;
    }
}

static RexiDev rexi_dev(const RexiPlan* R) {
    const Handle* h = R->h;
    RexiDev d{};
    d.L = h->L;
    d.npoles = R->npoles;
    d.ngroups = R->ngroups;
    d.ncplx = h->ncplx;
    d.coriolis = (R->p.coriolis && R->p.omega != 0.0) ? 1 : 0;
    // mixed form: complex FP32 factorisation and solves with FP64 refinement:
    // one step after substitutions with stored FP32 factors, two after an FP32
    // factorisation in the step
    d.refine = R->p.precision == SPH_PREC_MIXED ? (R->fphi32 ? 1 : 2) : 0;
    d.r = R->p.radius;
    d.ir = 1.0 / R->p.radius;
    d.T = 2.0 * R->p.omega;
    d.P = R->p.h0 * R->p.gravity;
    d.alpha = R->alpha;
    d.beta = R->beta;
    d.Cphi = R->Cphi;
    d.Cvel = R->Cvel;
    d.coef = R->coef;
    d.V = R->V;
    d.part = R->part;
    d.flag = R->flag;
    d.fphi = R->fphi;
    d.pphi = R->pphi;
    d.fvel = R->fvel;
    d.pvel = R->pvel;
    d.fphi32 = R->fphi32;
    d.fvel32 = R->fvel32;
    d.plane = R->plane;
    d.lanes = 32;
    return d;
}

// MAXN template dispatch of the lane kernels over the truncation
#define RX_DISPATCH(K, d, nb, s, ...)                                                             \
    do {                                                                                          \
        const int L1 = (d).L + 1;                                                                 \
        if ((d).fphi) {                                                                           \
            if (L1 <= 64) K<64, false, true><<<nb, 64, 0, s>>>(d, __VA_ARGS__);                   \
            else if (L1 <= 128) K<128, false, true><<<nb, 64, 0, s>>>(d, __VA_ARGS__);            \
            else K<256, false, true><<<nb, 64, 0, s>>>(d, __VA_ARGS__);                           \
        } else if ((d).refine > 0) {                                                              \
            if (L1 <= 64) K<64, true, false><<<nb, 64, 0, s>>>(d, __VA_ARGS__);                   \
            else if (L1 <= 128) K<128, true, false><<<nb, 64, 0, s>>>(d, __VA_ARGS__);            \
            else K<256, true, false><<<nb, 64, 0, s>>>(d, __VA_ARGS__);                           \
        } else {                                                                                  \
            if (L1 <= 64) K<64, false, false><<<nb, 64, 0, s>>>(d, __VA_ARGS__);                  \
            else if (L1 <= 128) K<128, false, false><<<nb, 64, 0, s>>>(d, __VA_ARGS__);           \
            else K<256, false, false><<<nb, 64, 0, s>>>(d, __VA_ARGS__);                          \
        }                                                                                         \
    } while (0)

// One step of the non-Robert form (SWERexiSPH::solve for every pole,
// SWERexiSPH.hpp:137-244, and the pole sum of AppSWE::run).  The pole-
// independent vectors of rexi_phi come from the non-Robert operators: div0 =
// ir div(u0, v0), eta0 = ir vort(u0, v0) through the grid divisions by cos phi
// (done per wavenumber on the Legendre coefficients: the divisions do not mix
// wavenumbers), and the Coriolis products grad_lat(mu) x for x = u0, mu2 u0,
// mu v0 (full grid, as the Robert form).  Per pole the velocity needs
// grad_lon(phi), grad_lat(phi) as spectra: one batched complex Legendre
// synthesis of i m phi and D phi over all poles, the division by cos phi, one
// batched analysis.
static int rexi_s0_step_launch(RexiPlan* R, double2* state, cudaStream_t s) {
    Handle* h = R->h;
    const int L = h->L, nlm = h->nlm, nc = h->ncplx, nlat = h->nlat, mF = L + 1;
    const long long ldF = (long long)mF * nlat, ldFc = (long long)(2 * L + 1) * nlat;
    const double g = R->p.gravity, ir = 1.0 / R->p.radius;
    const double2* hh = state;
    const double2* uu = state + nlm;
    const double2* vv = state + 2 * (size_t)nlm;
    const dim3 gc((L + 1 + 63) / 64, 2 * L + 1), gr((L + 1 + 63) / 64, L + 1);
    double2* V = R->V;
    auto Vs = [&](int k) { return V + (size_t)k * nc; };
    auto Xs = [&](int k) { return R->Xs + (size_t)k * nlm; };
    const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
    auto blocks = [](long long n) { return (unsigned)((n + 255) / 256); };
    // w = F(I(v0) cos phi)
    if (int rc = legendre_synthesis_real(h, vv, nlm, L, R->Fs, ldF, 1, s)) return rc;
    k_s0_fscale<<<blocks(ldF), 256, 0, s>>>(R->Fs, ldF, nlat, h->mu, R->glp, 0);
    if (int rc = legendre_analysis_real(h, R->Fs, ldF, Xs(0), nlm, L, 1, s)) return rc;
    // i m u0, D w, i m v0, D u0 -> div, eta
    if (int rc = spec_op(h, SPH_OP_DIFF_LON, uu, nlm, Xs(1), nlm, one, zero, 1, 0, s)) return rc;
    if (int rc = spec_op(h, SPH_OP_D1MU2, Xs(0), nlm, Xs(2), nlm, one, zero, 1, 0, s)) return rc;
    if (int rc = spec_op(h, SPH_OP_DIFF_LON, vv, nlm, Xs(3), nlm, one, zero, 1, 0, s)) return rc;
    if (int rc = spec_op(h, SPH_OP_D1MU2, uu, nlm, Xs(4), nlm, one, zero, 1, 0, s)) return rc;
    if (int rc = legendre_synthesis_real(h, Xs(1), nlm, L, R->Fs, ldF, 4, s)) return rc;
    k_s0_fdiveta<<<blocks(ldF), 256, 0, s>>>(R->Fs, ldF, nlat, h->mu, h->lat);
    if (int rc = legendre_analysis_real(h, R->Fs, ldF, Xs(5), nlm, L, 2, s)) return rc;
    // Coriolis products: G(x) = F(glp I(x)) for x = u0, mu2 u0, mu v0
    if (int rc = spec_op(h, SPH_OP_SCALE, uu, nlm, Xs(1), nlm, one, zero, 1, 0, s)) return rc;
    if (int rc = spec_op(h, SPH_OP_MU2, uu, nlm, Xs(2), nlm, one, zero, 1, 0, s)) return rc;
    if (int rc = spec_op(h, SPH_OP_MU, vv, nlm, Xs(3), nlm, one, zero, 1, 0, s)) return rc;
    if (int rc = legendre_synthesis_real(h, Xs(1), nlm, L, R->Fs, ldF, 3, s)) return rc;
    k_s0_fscale<<<blocks(3 * ldF), 256, 0, s>>>(R->Fs, 3 * ldF, nlat, h->mu, R->glp, 1);
    if (int rc = legendre_analysis_real(h, R->Fs, ldF, Xs(1), nlm, L, 3, s)) return rc;
    // complex promotions: 0 div0 = ir div, 14 eta0 = ir vort, 2 phi0 = g h, 10 u0, 11 v0, 7-9 the products
    k_rx_complexify<<<gc, 64, 0, s>>>(Xs(5), ir, Vs(0), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(Xs(6), ir, Vs(14), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(hh, g, Vs(2), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(uu, 1.0, Vs(10), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(vv, 1.0, Vs(11), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(Xs(1), 1.0, Vs(7), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(Xs(2), 1.0, Vs(8), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(Xs(3), 1.0, Vs(9), L);
    // 1 mu(eta0), 3 mu2(phi0), 4 mu2(div0), 5 mu2(mu eta0), 6 mu2 mu2 phi0
    k_rx_block_op<<<gc, 64, 0, s>>>(0, Vs(14), nullptr, Vs(1), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(2), nullptr, Vs(3), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(0), nullptr, Vs(4), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(1), nullptr, Vs(5), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(3), nullptr, Vs(6), L, ir);
    SPH_CUDA_TRY(cudaGetLastError());
    // phase A: phi of all poles
    const RexiDev d = rexi_dev(R);
    const long long nthreads = (long long)(2 * L + 1) * R->ngroups * 32;
    const unsigned nb = (unsigned)((nthreads + 63) / 64);
    RX_DISPATCH(k_rexi_s0_phi, d, nb, s, R->PH, R->XY);
    SPH_CUDA_TRY(cudaGetLastError());
    // grad_lon(phi), grad_lat(phi) of every pole as spectra
    const int nf = 2 * R->npoles;
    if (int rc = legendre_synthesis_cplx(h, R->XY, nc, R->FXY, ldFc, nf, s)) return rc;
    k_s0_fscale<<<blocks((long long)nf * ldFc), 256, 0, s>>>(R->FXY, (long long)nf * ldFc, nlat, h->mu, R->glp, 2);
    if (int rc = legendre_analysis_cplx(h, R->FXY, ldFc, R->XY, nc, nf, s)) return rc;
    // phase B: velocities, beta scaling, pole reduction
    RX_DISPATCH(k_rexi_s0_vel, d, nb, s, R->PH, R->XY);
    SPH_CUDA_TRY(cudaGetLastError());
    const double visc_fac = R->p.viscosity * R->p.tau / (R->p.radius * R->p.radius);
    k_rx_finish<<<gr, 64, 0, s>>>(R->part, R->ngroups, nc, state, L, nlm, 1.0 / g, visc_fac, R->flag);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

static int rexi_step_launch(RexiPlan* R, double2* state, cudaStream_t s) {
    if (!R->p.robert) return rexi_s0_step_launch(R, state, s);
    Handle* h = R->h;
    const int L = h->L, nlm = h->nlm, nc = h->ncplx, nlat = h->nlat, mF = L + 1;
    const double g = R->p.gravity, ir = 1.0 / R->p.radius;
    const double2* hh = state;
    const double2* uu = state + nlm;
    const double2* vv = state + 2 * (size_t)nlm;
    const dim3 gc((L + 1 + 63) / 64, 2 * L + 1), gr((L + 1 + 63) / 64, L + 1);
    double2* V = R->V;
    auto Vs = [&](int k) { return V + (size_t)k * nc; };
    // divergence of the Robert velocities: F(I(i m u + D v)/c^2), real transforms
    k_rx_divsrc<<<gr, 64, 0, s>>>(uu, vv, R->X, L);
    if (int rc = legendre_synthesis_real(h, R->X, nlm, L, R->F, (long long)mF * nlat, 1, s)) return rc;
    k_rx_fscale<<<(mF * nlat + 255) / 256, 256, 0, s>>>(R->F, nlat, mF, h->cosphi);
    if (int rc = legendre_analysis_real(h, R->F, (long long)mF * nlat, R->Xr, nlm, L, 1, s)) return rc;
    // complex promotions: 0 div0 = ir div, 2 phi0 = g h, 10 u0, 11 v0
    k_rx_complexify<<<gc, 64, 0, s>>>(R->Xr, ir, Vs(0), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(hh, g, Vs(2), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(uu, 1.0, Vs(10), L);
    k_rx_complexify<<<gc, 64, 0, s>>>(vv, 1.0, Vs(11), L);
    // 14 eta0, 1 mu(eta0), 3 mu2(phi0), 4 mu2(div0), 5 mu2(mu eta0), 6 mu2 mu2 phi0
    k_rx_block_op<<<gc, 64, 0, s>>>(2, Vs(10), Vs(11), Vs(14), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(0, Vs(14), nullptr, Vs(1), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(2), nullptr, Vs(3), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(0), nullptr, Vs(4), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(1), nullptr, Vs(5), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(3), nullptr, Vs(6), L, ir);
    // 15 mu2 u0, 16 mu2 mu2 u0, 12 mu v0, 17 mu2 mu v0, 13 mu u0
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(10), nullptr, Vs(15), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(15), nullptr, Vs(16), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(0, Vs(11), nullptr, Vs(12), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(1, Vs(12), nullptr, Vs(17), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(0, Vs(10), nullptr, Vs(13), L, ir);
    // 7 W1 = u0 - mu2 u0, 8 W2 = mu2 u0 - mu2 mu2 u0, 9 W3 = mu v0 - mu2 mu v0
    k_rx_block_op<<<gc, 64, 0, s>>>(3, Vs(10), Vs(15), Vs(7), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(3, Vs(15), Vs(16), Vs(8), L, ir);
    k_rx_block_op<<<gc, 64, 0, s>>>(3, Vs(12), Vs(17), Vs(9), L, ir);
    SPH_CUDA_TRY(cudaGetLastError());
    // all poles x all m x both parities
    const RexiDev d = rexi_dev(R);
    const long long nthreads = (long long)(2 * L + 1) * R->ngroups * 32;
    const unsigned nb = (unsigned)((nthreads + 63) / 64);
    if ((d.fphi || d.fphi32) && R->PHr) {
        // factors stored at plan creation (FP64, or FP32 with one FP64
        // refinement step in the mixed form): substitutions only, a Phi phase and
        // a velocity phase of one warp per (pole group, m-block, parity)
        const unsigned nb2 = 2 * nb;
#define RX_ST(MAXN, MX)                                          \
    do {                                                         \
        k_rexi_phi_st<MAXN, MX><<<nb2, 64, 0, s>>>(d, R->PHr);   \
        k_rexi_vel_st<MAXN, MX><<<nb2, 64, 0, s>>>(d, R->PHr);   \
    } while (0)
        const bool mx = d.fphi32 != nullptr;
        if (L + 1 <= 64) {
            if (mx) RX_ST(64, true);
            else RX_ST(64, false);
        } else if (L + 1 <= 128) {
            if (mx) RX_ST(128, true);
            else RX_ST(128, false);
        } else {
            if (mx) RX_ST(256, true);
            else RX_ST(256, false);
        }
#undef RX_ST
    } else if (d.fphi) {
        if (L + 1 <= 64) k_rexi_solve<64, false, true><<<nb, 64, 0, s>>>(d);
        else if (L + 1 <= 128) k_rexi_solve<128, false, true><<<nb, 64, 0, s>>>(d);
        else k_rexi_solve<256, false, true><<<nb, 64, 0, s>>>(d);
    } else if (d.refine > 0) {
        if (L + 1 <= 64) k_rexi_solve<64, true, false><<<nb, 64, 0, s>>>(d);
        else if (L + 1 <= 128) k_rexi_solve<128, true, false><<<nb, 64, 0, s>>>(d);
        else k_rexi_solve<256, true, false><<<nb, 64, 0, s>>>(d);
    } else {
        if (L + 1 <= 64) k_rexi_solve<64, false, false><<<nb, 64, 0, s>>>(d);
        else if (L + 1 <= 128) k_rexi_solve<128, false, false><<<nb, 64, 0, s>>>(d);
        else k_rexi_solve<256, false, false><<<nb, 64, 0, s>>>(d);
    }
    SPH_CUDA_TRY(cudaGetLastError());
    const double visc_fac = R->p.viscosity * R->p.tau / (R->p.radius * R->p.radius);
    k_rx_finish<<<gr, 64, 0, s>>>(R->part, R->ngroups, nc, state, L, nlm, 1.0 / g, visc_fac, R->flag);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

static void rexi_free(RexiPlan* R) {
    if (!R) return;
    if (R->exec) cudaGraphExecDestroy(R->exec);
    if (R->graph) cudaGraphDestroy(R->graph);
    void* bufs[] = {R->alpha, R->beta, R->Cphi, R->Cvel, R->coef, R->V,  R->part, R->X,  R->Xr, R->F,
                    R->flag,  R->fphi, R->fvel, R->pphi, R->pvel, R->PH, R->XY,   R->FXY, R->Xs, R->Fs, R->glp,
                    R->PHr,   R->fphi32, R->fvel32};
    for (void* p : bufs)
        if (p) cudaFree(p);
    delete R;
}

}  // namespace sphgpu

using namespace sphgpu;

struct sph_rexi : public RexiPlan {};

extern "C" {

int sph_rexi_create(sph_handle* hh, const double* alpha, const double* beta, int npoles, const sph_rexi_params* p,
                    sph_rexi** out) {
    if (out) *out = nullptr;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !alpha || !beta || npoles <= 0 || !p || !out || p->tau == 0.0 || p->radius <= 0.0) {
        set_error("sph_rexi_create: bad arguments");
        return SPH_ERR_ARG;
    }
    if (p->precision != SPH_PREC_FP64 && p->precision != SPH_PREC_MIXED) {
        set_error("sph_rexi_create: precision must be SPH_PREC_FP64 or SPH_PREC_MIXED");
        return SPH_ERR_ARG;
    }
    if (h->L > 255) {
        set_error("sph_rexi_create: truncations above T255 are not supported by the REXI solver");
        return SPH_ERR_ARG;
    }
    sph_rexi* R = new sph_rexi();
    R->h = h;
    R->p = *p;
    R->npoles = npoles;
    R->ngroups = (npoles + 31) / 32;
    const int L = h->L, nc = h->ncplx;
    // pole scalars alpha/tau, beta/tau (SWERexiSPHRobert.hpp:84-85)
    std::vector<double2> al(npoles), be(npoles);
    for (int k = 0; k < npoles; k++) {
        al[k] = make_double2(alpha[2 * k] / p->tau, alpha[2 * k + 1] / p->tau);
        be[k] = make_double2(beta[2 * k] / p->tau, beta[2 * k + 1] / p->tau);
    }
    // pole-independent band matrices, grouped by power of alpha
    const double r = p->radius, T = 2.0 * p->omega, P = p->h0 * p->gravity;
    BandTable C2(L), C1(L), Cm1(L), C0(L), Cv(L);
    const bool cor = p->coriolis && p->omega != 0.0;
    comp_z7(C2, cd(-P), r);
    if (cor) {
        comp_z2(C2, cd(2.0 * T * T));
        comp_z3(C0, cd(T * T * T * T));
        if (p->robert) {  // SWERexiSPHRobert::setup (SWERexiSPHRobert.hpp:109-131)
            comp_z4robert(C1, cd(-P * T), r);
            comp_z5robert(Cm1, cd(P * T * T * T), r, p->fix_z5robert != 0);
            comp_z6robert(C0, cd(P * 2.0 * T * T), r);
        } else {          // SWERexiSPH::setup (SWERexiSPH.hpp:107-129)
            comp_z4(C1, cd(-P * T), r);
            comp_z5(Cm1, cd(P * T * T * T), r);
            comp_z6(C0, cd(P * 2.0 * T * T), r);
        }
        comp_z8(C0, cd(-P * T * T), r);
        comp_z2(Cv, cd(T * T));
    }
    std::vector<double2> cphi((size_t)4 * nc * 5), cvel((size_t)nc * 3);
    const BandTable* tabs[4] = {&C2, &C1, &Cm1, &C0};
    for (int q = 0; q < 4; q++)
        for (size_t i = 0; i < (size_t)nc * 5; i++)
            cphi[(size_t)q * nc * 5 + i] = make_double2(tabs[q]->a[i].real(), tabs[q]->a[i].imag());
    for (int row = 0; row < nc; row++)
        for (int dd = 0; dd < 3; dd++) {
            const cd v = Cv.a[(size_t)row * 5 + dd + 1];
            cvel[(size_t)row * 3 + dd] = make_double2(v.real(), v.imag());
        }
    std::vector<double> coef((size_t)nc * 4);
    for (int m = -L; m <= L; m++)
        for (int n = std::abs(m); n <= L; n++) {
            const int row = brow(L, n, m);
            coef[(size_t)row * 4 + 0] = idR(n - 1, m);
            coef[(size_t)row * 4 + 1] = idS(n + 1, m);
            coef[(size_t)row * 4 + 2] = (-(double)n + 1.0) * idR(n - 1, m);
            coef[(size_t)row * 4 + 3] = ((double)n + 2.0) * idS(n + 1, m);
        }
    auto fail = [&](int rc) {
        rexi_free(R);
        return rc;
    };
#define RX_TRY(x)                                                               \
    do {                                                                        \
        cudaError_t e_ = (x);                                                   \
        if (e_ != cudaSuccess) {                                                \
            set_error(std::string("sph_rexi_create: ") + cudaGetErrorString(e_)); \
            return fail(SPH_ERR_CUDA);                                          \
        }                                                                       \
    } while (0)
    RX_TRY(cudaMalloc(&R->alpha, sizeof(double2) * npoles));
    RX_TRY(cudaMalloc(&R->beta, sizeof(double2) * npoles));
    RX_TRY(cudaMalloc(&R->Cphi, sizeof(double2) * cphi.size()));
    RX_TRY(cudaMalloc(&R->Cvel, sizeof(double2) * cvel.size()));
    RX_TRY(cudaMalloc(&R->coef, sizeof(double) * coef.size()));
    RX_TRY(cudaMalloc(&R->V, sizeof(double2) * 18 * (size_t)nc));
    RX_TRY(cudaMalloc(&R->part, sizeof(double2) * 3 * (size_t)nc * R->ngroups));
    RX_TRY(cudaMalloc(&R->X, sizeof(double2) * h->nlm));
    RX_TRY(cudaMalloc(&R->Xr, sizeof(double2) * h->nlm));
    RX_TRY(cudaMalloc(&R->F, sizeof(double2) * (size_t)(L + 1) * h->nlat));
    RX_TRY(cudaMalloc(&R->flag, sizeof(int)));
    if (!p->robert) {
        const size_t ldFc = (size_t)(2 * L + 1) * h->nlat;
        RX_TRY(cudaMalloc(&R->PH, sizeof(double2) * (size_t)npoles * nc));
        RX_TRY(cudaMalloc(&R->XY, sizeof(double2) * 2 * (size_t)npoles * nc));
        RX_TRY(cudaMalloc(&R->FXY, sizeof(double2) * 2 * (size_t)npoles * ldFc));
        RX_TRY(cudaMalloc(&R->Xs, sizeof(double2) * 8 * (size_t)h->nlm));
        RX_TRY(cudaMalloc(&R->Fs, sizeof(double2) * 4 * (size_t)(L + 1) * h->nlat));
        RX_TRY(cudaMemset(R->PH, 0, sizeof(double2) * (size_t)npoles * nc));
        RX_TRY(cudaMemset(R->XY, 0, sizeof(double2) * 2 * (size_t)npoles * nc));
        const std::vector<double> glp = s0_grad_lat_mu(h);
        RX_TRY(cudaMalloc(&R->glp, sizeof(double) * h->nlat));
        RX_TRY(cudaMemcpy(R->glp, glp.data(), sizeof(double) * h->nlat, cudaMemcpyHostToDevice));
    }
    RX_TRY(cudaMemcpy(R->alpha, al.data(), sizeof(double2) * npoles, cudaMemcpyHostToDevice));
    RX_TRY(cudaMemcpy(R->beta, be.data(), sizeof(double2) * npoles, cudaMemcpyHostToDevice));
    RX_TRY(cudaMemcpy(R->Cphi, cphi.data(), sizeof(double2) * cphi.size(), cudaMemcpyHostToDevice));
    RX_TRY(cudaMemcpy(R->Cvel, cvel.data(), sizeof(double2) * cvel.size(), cudaMemcpyHostToDevice));
    RX_TRY(cudaMemcpy(R->coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice));
    RX_TRY(cudaMemset(R->V, 0, sizeof(double2) * 18 * (size_t)nc));
    RX_TRY(cudaMemset(R->flag, 0, sizeof(int)));
    // FP64 form with Coriolis: factor every banded system once (the matrices
    // depend on the pole and m only), if the factors fit in half the free
    // device memory; every step then runs the substitutions alone
    const char* store_env = std::getenv("SPH_REXI_STORE");  // "0": factor on the fly every step
    if (cor && p->precision == SPH_PREC_FP64 && !p->factor_each_step && !(store_env && store_env[0] == '0')) {
        const long long plane = (long long)R->ngroups * nc * 32;
        const size_t bytes = (size_t)plane * (11 * sizeof(double2) + 2);
        size_t free_b = 0, total_b = 0;
        RX_TRY(cudaMemGetInfo(&free_b, &total_b));
        if (bytes <= free_b / 2) {
            RX_TRY(cudaMalloc(&R->fphi, sizeof(double2) * 7 * (size_t)plane));
            RX_TRY(cudaMalloc(&R->fvel, sizeof(double2) * 4 * (size_t)plane));
            RX_TRY(cudaMalloc(&R->pphi, (size_t)plane));
            RX_TRY(cudaMalloc(&R->pvel, (size_t)plane));
            if (p->robert) RX_TRY(cudaMalloc(&R->PHr, sizeof(double2) * (size_t)plane));
            R->plane = plane;
            const long long nthreads = (long long)(2 * L + 1) * R->ngroups * 32;
            k_rexi_factor<<<(unsigned)((nthreads + 63) / 64), 64>>>(rexi_dev(R));
            RX_TRY(cudaGetLastError());
            int flag = 0;
            RX_TRY(cudaMemcpy(&flag, R->flag, sizeof(int), cudaMemcpyDeviceToHost));
            R->singular = (flag & 2) != 0;
            RX_TRY(cudaMemset(R->flag, 0, sizeof(int)));
        }
    }
    // mixed form, Robert form with Coriolis: the same once-per-plan factoring in
    // complex FP32 (half the bytes); each step substitutes in FP32 and refines
    // once with FP64 residuals
    if (cor && p->precision == SPH_PREC_MIXED && p->robert && !p->factor_each_step &&
        !(store_env && store_env[0] == '0')) {
        const long long plane = (long long)R->ngroups * nc * 32;
        const size_t bytes = (size_t)plane * (11 * sizeof(float2) + 2 + sizeof(double2));
        size_t free_b = 0, total_b = 0;
        RX_TRY(cudaMemGetInfo(&free_b, &total_b));
        if (bytes <= free_b / 2) {
            RX_TRY(cudaMalloc(&R->fphi32, sizeof(float2) * 7 * (size_t)plane));
            RX_TRY(cudaMalloc(&R->fvel32, sizeof(float2) * 4 * (size_t)plane));
            RX_TRY(cudaMalloc(&R->pphi, (size_t)plane));
            RX_TRY(cudaMalloc(&R->pvel, (size_t)plane));
            RX_TRY(cudaMalloc(&R->PHr, sizeof(double2) * (size_t)plane));
            R->plane = plane;
            const long long nthreads = (long long)(2 * L + 1) * R->ngroups * 32;
            k_rexi_factor_f<<<(unsigned)((nthreads + 63) / 64), 64>>>(rexi_dev(R));
            RX_TRY(cudaGetLastError());
            int flag = 0;
            RX_TRY(cudaMemcpy(&flag, R->flag, sizeof(int), cudaMemcpyDeviceToHost));
            R->singular = (flag & 2) != 0;
            RX_TRY(cudaMemset(R->flag, 0, sizeof(int)));
        }
    }
#undef RX_TRY
    *out = R;
    return SPH_OK;
}

int sph_rexi_destroy(sph_rexi* r) {
    if (!r) return SPH_OK;
    cudaDeviceSynchronize();
    rexi_free(r);
    return SPH_OK;
}

int sph_rexi_step(sph_rexi* R, double* state, int nsteps, void* stream) {
    if (!R || !state || nsteps < 0) {
        set_error("sph_rexi_step: bad arguments");
        return SPH_ERR_ARG;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!R->exec || R->state != state || R->stream != s) {
        if (R->exec) { cudaGraphExecDestroy(R->exec); R->exec = nullptr; }
        if (R->graph) { cudaGraphDestroy(R->graph); R->graph = nullptr; }
        // operand workspace of the mixed transforms of the step (at most 4 fields
        // per call): a capture cannot allocate
        if (int rc = tc_reserve(R->h, 4)) return rc;
        cudaStream_t cap;
        SPH_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        SPH_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int rc = rexi_step_launch(R, reinterpret_cast<double2*>(state), cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) { set_error(std::string("sph_rexi_step: capture: ") + cudaGetErrorString(e)); return SPH_ERR_CUDA; }
        R->graph = g;
        SPH_CUDA_TRY(cudaGraphInstantiate(&R->exec, g, 0));
        R->state = state;
        R->stream = s;
    }
    SPH_CUDA_TRY(cudaMemsetAsync(R->flag, 0, sizeof(int), s));
    for (int i = 0; i < nsteps; i++) SPH_CUDA_TRY(cudaGraphLaunch(R->exec, s));
    int flag = 0;
    SPH_CUDA_TRY(cudaMemcpyAsync(&flag, R->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPH_CUDA_TRY(cudaStreamSynchronize(s));
    if (R->singular && nsteps > 0) flag |= 2;
    if (flag & 2) {
        set_error("sph_rexi_step: zero pivot in a banded solve (zgbsv INFO > 0)");
        return SPH_ERR_SINGULAR;
    }
    if (flag & 1) {
        set_error("sph_rexi_step: instability detected (non-finite value in h)");
        return SPH_ERR_NAN;
    }
    return SPH_OK;
}

}  // extern "C"
