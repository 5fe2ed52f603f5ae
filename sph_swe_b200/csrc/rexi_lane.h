// Per-pole arithmetic of the REXI solver (one thread = one pole x one m-block),
// shared by the CUDA kernel in rexi.cu and its CPU unit test.
#pragma once

#include <cmath>
#include <vector_types.h>
#include <vector_functions.h>

#include "rexi_tables.h"

#ifdef __CUDA_ARCH__
#define RX_LDG(p) __ldg(p)
#else
#define RX_LDG(p) (*(p))
using std::fabs;
#endif

namespace sphgpu {

struct RexiDev {
    int L, npoles, ngroups, ncplx;
    int coriolis;
    int refine;  // 0: FP64 direct; k > 0: complex FP32 factor/solve + k FP64 refinement steps
    double r, ir, T, P;  // radius, 1/radius, 2 Omega, average geopotential
    const double2* alpha;
    const double2* beta;
    const double2* Cphi;
    const double2* Cvel;
    const double* coef;
    const double2* V;
    double2* part;
    int* flag;
    // stored factors of the banded systems (nullptr: factor on the fly), see BandRef
    double2* fphi;       // [7 planes][plane]: 1/U_kk, U_k,k+1..k+4, multipliers 1..2
    signed char* pphi;   // [plane] pivot offsets
    double2* fvel;       // [4 planes][plane]: 1/U_kk, U_k,k+1..k+2, multiplier
    signed char* pvel;   // [plane]
    // the same factors in complex FP32 (mixed form), pivots in pphi / pvel
    float2* fphi32;      // [7 planes][plane]
    float2* fvel32;      // [4 planes][plane]
    long long plane;     // ngroups * ncplx * lanes
    int lanes;           // poles per group (32 on the device, 1 on the host)
};

// Row k of one stored banded system: plane q at f[q * plane + i0 + k * lanes].
// Rows of parity par of the m-block at block row `base` (N rows), pole group
// g, lane `lane`: i0 = ((g * ncplx + base + (par ? (N + 1) / 2 : 0)) * lanes + lane.
struct BandRef {
    double2* f;
    signed char* pv;
    long long plane, i0;
    int lanes;
};
// the same for factors stored in complex FP32
struct BandRefF {
    float2* f;
    signed char* pv;
    long long plane, i0;
    int lanes;
};

__host__ __device__ inline double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline double2 c_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline double2 c_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ inline double2 c_div(double2 a, double2 b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__host__ __device__ inline double c_abs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__host__ __device__ inline double2 c_im(double2 a, double m) { return make_double2(-m * a.y, m * a.x); }  // a * i m
__host__ __device__ inline double2 ld(const double2* p) { return RX_LDG(p); }

// Banded LU with partial pivoting (kl = ku = H on the parity-reduced system of
// Np rows) and solve for NR right-hand sides, one system per thread.
// entry(k, d) gives A[k][k+d] for d = -H..H, rhs(k, r) right-hand side r.
// Solutions are written through out(k, r, x).  Returns false on a zero pivot.
// The pivot rule is LAPACK's (first maximum of |re|+|im| in the column).
// U rows (2H+1 entries) and the eliminated right-hand sides live in the
// thread-local arrays U / y.
template <int H, int MAXR, int NR, class Entry, class Rhs, class Out>
__host__ __device__ bool band_solve(int Np, Entry entry, Rhs rhs, Out out) {
    constexpr int W = 2 * H + 1;
    double2 U[MAXR][W];
    double2 y[MAXR][NR];
    double2 win[H + 1][W];  // rows k..k+H, columns k..k+2H
    double2 wr[H + 1][NR];
#pragma unroll
    for (int i = 0; i <= H; i++) {
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - i;  // row i, column j
            win[i][j] = (i < Np && d >= -H && d <= H && j < Np) ? entry(i, d) : make_double2(0, 0);
        }
#pragma unroll
        for (int r = 0; r < NR; r++) wr[i][r] = i < Np ? rhs(i, r) : make_double2(0, 0);
    }
    bool ok = true;
    for (int k = 0; k < Np; k++) {
        int p = 0;
        double best = c_abs1(win[0][0]);
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const double v = (k + i < Np) ? c_abs1(win[i][0]) : -1.0;
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.0) ok = false;
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < W; j++) {
                const double2 t0 = win[0][j], ti = win[i][j];
                win[0][j] = sw ? ti : t0;
                win[i][j] = sw ? t0 : ti;
            }
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const double2 t0 = wr[0][r], ti = wr[i][r];
                wr[0][r] = sw ? ti : t0;
                wr[i][r] = sw ? t0 : ti;
            }
        }
        const double2 rp = best == 0.0 ? make_double2(0, 0) : c_div(make_double2(1, 0), win[0][0]);
#pragma unroll
        for (int j = 0; j < W; j++) U[k][j] = win[0][j];
#pragma unroll
        for (int r = 0; r < NR; r++) y[k][r] = wr[0][r];
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const double2 l = c_mul(win[i][0], rp);
#pragma unroll
            for (int j = 1; j < W; j++) win[i][j] = c_sub(win[i][j], c_mul(l, win[0][j]));
#pragma unroll
            for (int r = 0; r < NR; r++) wr[i][r] = c_sub(wr[i][r], c_mul(l, wr[0][r]));
        }
        // shift the window one row down / one column right, load row k+1+H
#pragma unroll
        for (int i = 0; i < H; i++) {
#pragma unroll
            for (int j = 0; j < W - 1; j++) win[i][j] = win[i + 1][j + 1];
            win[i][W - 1] = make_double2(0, 0);
#pragma unroll
            for (int r = 0; r < NR; r++) wr[i][r] = wr[i + 1][r];
        }
        const int rn = k + 1 + H;
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - H;  // row rn at window row H, column j <-> matrix column k+1+j
            win[H][j] = (rn < Np && k + 1 + j < Np) ? entry(rn, d) : make_double2(0, 0);
        }
#pragma unroll
        for (int r = 0; r < NR; r++) wr[H][r] = rn < Np ? rhs(rn, r) : make_double2(0, 0);
    }
    // back substitution with a sliding window of the last 2H solution values
    double2 x[W][NR];
#pragma unroll
    for (int j = 0; j < W; j++)
#pragma unroll
        for (int r = 0; r < NR; r++) x[j][r] = make_double2(0, 0);
    for (int k = Np - 1; k >= 0; k--) {
        const double2 rd = c_div(make_double2(1, 0), U[k][0]);
#pragma unroll
        for (int r = 0; r < NR; r++) {
            double2 s = y[k][r];
#pragma unroll
            for (int j = 1; j < W; j++) s = c_sub(s, c_mul(U[k][j], x[j - 1][r]));
            const double2 xk = c_mul(s, rd);
#pragma unroll
            for (int j = W - 1; j > 0; j--) x[j][r] = x[j - 1][r];
            x[0][r] = xk;
            out(k, r, xk);
        }
    }
    return ok;
}

// The factorisation of band_solve alone, stored: per row 1/U_kk, the U row's
// 2H off-diagonal entries, the H multipliers and the pivot offset.  The same
// operations in the same order as band_solve, so that band_solve_stored
// reproduces its results.  Returns false on a zero pivot.
template <int H, class Entry>
__host__ __device__ bool band_factor_store(int Np, Entry entry, const BandRef& st) {
    constexpr int W = 2 * H + 1;
    double2 win[H + 1][W];
#pragma unroll
    for (int i = 0; i <= H; i++)
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - i;
            win[i][j] = (i < Np && d >= -H && d <= H && j < Np) ? entry(i, d) : make_double2(0, 0);
        }
    bool ok = true;
    for (int k = 0; k < Np; k++) {
        int p = 0;
        double best = c_abs1(win[0][0]);
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const double v = (k + i < Np) ? c_abs1(win[i][0]) : -1.0;
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.0) ok = false;
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < W; j++) {
                const double2 t0 = win[0][j], ti = win[i][j];
                win[0][j] = sw ? ti : t0;
                win[i][j] = sw ? t0 : ti;
            }
        }
        const double2 rp = best == 0.0 ? make_double2(0, 0) : c_div(make_double2(1, 0), win[0][0]);
        const long long e = st.i0 + (long long)k * st.lanes;
        st.pv[e] = (signed char)p;
        st.f[e] = rp;
#pragma unroll
        for (int j = 1; j < W; j++) st.f[j * st.plane + e] = win[0][j];
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const double2 l = c_mul(win[i][0], rp);
            st.f[(2 * H + i) * st.plane + e] = l;
#pragma unroll
            for (int j = 1; j < W; j++) win[i][j] = c_sub(win[i][j], c_mul(l, win[0][j]));
        }
#pragma unroll
        for (int i = 0; i < H; i++) {
#pragma unroll
            for (int j = 0; j < W - 1; j++) win[i][j] = win[i + 1][j + 1];
            win[i][W - 1] = make_double2(0, 0);
        }
        const int rn = k + 1 + H;
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - H;
            win[H][j] = (rn < Np && k + 1 + j < Np) ? entry(rn, d) : make_double2(0, 0);
        }
    }
    return ok;
}

// Forward elimination and back substitution of band_solve with the factors
// that band_factor_store wrote.  The factors of PF rows are loaded together
// before those rows are processed (they do not depend on the right-hand
// sides), so that a lane keeps several rows' loads in flight; the arithmetic
// is that of band_solve, row by row in the same order.
template <int H, int MAXR, int NR, class Rhs, class Out>
__host__ __device__ void band_solve_stored(int Np, const BandRef& st, Rhs rhs, Out out) {
    constexpr int W = 2 * H + 1;
    constexpr int PF = 4;                  // rows per prefetch group, forward
    constexpr int PB = H >= 2 ? 2 : 4;     // rows per prefetch group, backward
    double2 y[MAXR][NR];
    double2 wr[H + 1][NR];
#pragma unroll
    for (int i = 0; i <= H; i++)
#pragma unroll
        for (int r = 0; r < NR; r++) wr[i][r] = i < Np ? rhs(i, r) : make_double2(0, 0);
    for (int k0 = 0; k0 < Np; k0 += PF) {
        int pvs[PF];
        double2 lm[PF][H];
#pragma unroll
        for (int u = 0; u < PF; u++) {
            const int k = k0 + u < Np ? k0 + u : Np - 1;
            const long long e = st.i0 + (long long)k * st.lanes;
            pvs[u] = RX_LDG(&st.pv[e]);
#pragma unroll
            for (int i = 1; i <= H; i++) lm[u][i - 1] = ld(&st.f[(2 * H + i) * st.plane + e]);
        }
#pragma unroll
        for (int u = 0; u < PF; u++) {
            const int k = k0 + u;
            if (k >= Np) break;
            const int p = pvs[u];
#pragma unroll
            for (int i = 1; i <= H; i++) {
                const bool sw = (p == i);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const double2 t0 = wr[0][r], ti = wr[i][r];
                    wr[0][r] = sw ? ti : t0;
                    wr[i][r] = sw ? t0 : ti;
                }
            }
#pragma unroll
            for (int r = 0; r < NR; r++) y[k][r] = wr[0][r];
#pragma unroll
            for (int i = 1; i <= H; i++) {
                const double2 l = lm[u][i - 1];
#pragma unroll
                for (int r = 0; r < NR; r++) wr[i][r] = c_sub(wr[i][r], c_mul(l, wr[0][r]));
            }
#pragma unroll
            for (int i = 0; i < H; i++)
#pragma unroll
                for (int r = 0; r < NR; r++) wr[i][r] = wr[i + 1][r];
            const int rn = k + 1 + H;
#pragma unroll
            for (int r = 0; r < NR; r++) wr[H][r] = rn < Np ? rhs(rn, r) : make_double2(0, 0);
        }
    }
    double2 x[W][NR];
#pragma unroll
    for (int j = 0; j < W; j++)
#pragma unroll
        for (int r = 0; r < NR; r++) x[j][r] = make_double2(0, 0);
    for (int k1 = Np - 1; k1 >= 0; k1 -= PB) {
        double2 rds[PB], us[PB][W];
#pragma unroll
        for (int u = 0; u < PB; u++) {
            const int k = k1 - u >= 0 ? k1 - u : 0;
            const long long e = st.i0 + (long long)k * st.lanes;
            rds[u] = ld(&st.f[e]);
#pragma unroll
            for (int j = 1; j < W; j++) us[u][j] = ld(&st.f[j * st.plane + e]);
        }
#pragma unroll
        for (int u = 0; u < PB; u++) {
            const int k = k1 - u;
            if (k < 0) break;
#pragma unroll
            for (int r = 0; r < NR; r++) {
                double2 s = y[k][r];
#pragma unroll
                for (int j = 1; j < W; j++) s = c_sub(s, c_mul(us[u][j], x[j - 1][r]));
                const double2 xk = c_mul(s, rds[u]);
#pragma unroll
                for (int j = W - 1; j > 0; j--) x[j][r] = x[j - 1][r];
                x[0][r] = xk;
                out(k, r, xk);
            }
        }
    }
}

__host__ __device__ inline float2 f_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline float2 f_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline float2 f_div(float2 a, float2 b) {
    const float d = b.x * b.x + b.y * b.y;
    return make_float2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__host__ __device__ inline float f_abs1(float2 a) { return fabsf(a.x) + fabsf(a.y); }
__host__ __device__ inline float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
__host__ __device__ inline double2 to_d(float2 a) { return make_double2((double)a.x, (double)a.y); }

// The same banded system as band_solve, factored once in complex FP32 (LAPACK
// pivot rule on |re|+|im| of the FP32 entries; U rows, multipliers and pivot
// offsets kept per thread) and solved in FP32; then `refine` steps of FP64
// iterative refinement: r = b - A x with A and b in FP64 (entry / rhs), the
// correction solved with the FP32 factors, x += correction in FP64.
template <int H, int MAXR, int NR, class Entry, class Rhs, class Out>
__host__ __device__ bool band_solve_mixed(int Np, int refine, Entry entry, Rhs rhs, Out out) {
    constexpr int W = 2 * H + 1;
    float2 U[MAXR][W];
    float2 Lm[MAXR][H];
    signed char pv[MAXR];
    double2 x[MAXR][NR];
    float2 win[H + 1][W];
#pragma unroll
    for (int i = 0; i <= H; i++)
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - i;
            win[i][j] = (i < Np && d >= -H && d <= H && j < Np) ? to_f(entry(i, d)) : make_float2(0.f, 0.f);
        }
    bool ok = true;
    for (int k = 0; k < Np; k++) {
        int p = 0;
        float best = f_abs1(win[0][0]);
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const float v = (k + i < Np) ? f_abs1(win[i][0]) : -1.f;
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.f) ok = false;
        pv[k] = (signed char)p;
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < W; j++) {
                const float2 t0 = win[0][j], ti = win[i][j];
                win[0][j] = sw ? ti : t0;
                win[i][j] = sw ? t0 : ti;
            }
        }
        const float2 rp = best == 0.f ? make_float2(0.f, 0.f) : f_div(make_float2(1.f, 0.f), win[0][0]);
#pragma unroll
        for (int j = 0; j < W; j++) U[k][j] = win[0][j];
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const float2 l = f_mul(win[i][0], rp);
            Lm[k][i - 1] = l;
#pragma unroll
            for (int j = 1; j < W; j++) win[i][j] = f_sub(win[i][j], f_mul(l, win[0][j]));
        }
#pragma unroll
        for (int i = 0; i < H; i++) {
#pragma unroll
            for (int j = 0; j < W - 1; j++) win[i][j] = win[i + 1][j + 1];
            win[i][W - 1] = make_float2(0.f, 0.f);
        }
        const int rn = k + 1 + H;
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - H;
            win[H][j] = (rn < Np && k + 1 + j < Np) ? to_f(entry(rn, d)) : make_float2(0.f, 0.f);
        }
    }
    // solve with the FP32 factors; b(k, r) gives the right-hand side, the
    // solution is added to x (first pass: stored)
    auto lu_solve = [&](auto b, bool add) {
        float2 wr[H + 1][NR];
#pragma unroll
        for (int i = 0; i <= H; i++)
#pragma unroll
            for (int r = 0; r < NR; r++) wr[i][r] = i < Np ? to_f(b(i, r)) : make_float2(0.f, 0.f);
        float2 y[MAXR][NR];
        for (int k = 0; k < Np; k++) {
            const int p = pv[k];
#pragma unroll
            for (int i = 1; i <= H; i++) {
                const bool sw = (p == i);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const float2 t0 = wr[0][r], ti = wr[i][r];
                    wr[0][r] = sw ? ti : t0;
                    wr[i][r] = sw ? t0 : ti;
                }
            }
#pragma unroll
            for (int r = 0; r < NR; r++) y[k][r] = wr[0][r];
#pragma unroll
            for (int i = 1; i <= H; i++)
#pragma unroll
                for (int r = 0; r < NR; r++) wr[i][r] = f_sub(wr[i][r], f_mul(Lm[k][i - 1], wr[0][r]));
#pragma unroll
            for (int i = 0; i < H; i++)
#pragma unroll
                for (int r = 0; r < NR; r++) wr[i][r] = wr[i + 1][r];
            const int rn = k + 1 + H;
#pragma unroll
            for (int r = 0; r < NR; r++) wr[H][r] = rn < Np ? to_f(b(rn, r)) : make_float2(0.f, 0.f);
        }
        float2 xs[W][NR];
#pragma unroll
        for (int j = 0; j < W; j++)
#pragma unroll
            for (int r = 0; r < NR; r++) xs[j][r] = make_float2(0.f, 0.f);
        for (int k = Np - 1; k >= 0; k--) {
            const float2 rd = f_div(make_float2(1.f, 0.f), U[k][0]);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                float2 sm = y[k][r];
#pragma unroll
                for (int j = 1; j < W; j++) sm = f_sub(sm, f_mul(U[k][j], xs[j - 1][r]));
                const float2 xk = f_mul(sm, rd);
#pragma unroll
                for (int j = W - 1; j > 0; j--) xs[j][r] = xs[j - 1][r];
                xs[0][r] = xk;
                x[k][r] = add ? c_add(x[k][r], to_d(xk)) : to_d(xk);
            }
        }
    };
    lu_solve([&](int k, int r) { return rhs(k, r); }, false);
    for (int it = 0; it < refine; it++) {
        // residual r = b - A x in FP64 (entry(k, d) = A[k][k+d])
        lu_solve(
            [&](int k, int r) {
                double2 v = rhs(k, r);
#pragma unroll
                for (int d = -H; d <= H; d++)
                    if (k + d >= 0 && k + d < Np) v = c_sub(v, c_mul(entry(k, d), x[k + d][r]));
                return v;
            },
            true);
    }
    for (int k = 0; k < Np; k++)
#pragma unroll
        for (int r = 0; r < NR; r++) out(k, r, x[k][r]);
    return ok;
}

// The FP32 factorisation of band_solve_mixed alone, stored (complex FP32
// planes: 1/U_kk, the U row's 2H off-diagonal entries, the H multipliers; the
// pivot offset): the operations of band_solve_mixed in the same order.
// Returns false on a zero pivot.
template <int H, class Entry>
__host__ __device__ bool band_factor_store_f(int Np, Entry entry, const BandRefF& st) {
    constexpr int W = 2 * H + 1;
    float2 win[H + 1][W];
#pragma unroll
    for (int i = 0; i <= H; i++)
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - i;
            win[i][j] = (i < Np && d >= -H && d <= H && j < Np) ? to_f(entry(i, d)) : make_float2(0.f, 0.f);
        }
    bool ok = true;
    for (int k = 0; k < Np; k++) {
        int p = 0;
        float best = f_abs1(win[0][0]);
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const float v = (k + i < Np) ? f_abs1(win[i][0]) : -1.f;
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.f) ok = false;
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < W; j++) {
                const float2 t0 = win[0][j], ti = win[i][j];
                win[0][j] = sw ? ti : t0;
                win[i][j] = sw ? t0 : ti;
            }
        }
        const float2 rp = best == 0.f ? make_float2(0.f, 0.f) : f_div(make_float2(1.f, 0.f), win[0][0]);
        const long long e = st.i0 + (long long)k * st.lanes;
        st.pv[e] = (signed char)p;
        st.f[e] = rp;
#pragma unroll
        for (int j = 1; j < W; j++) st.f[j * st.plane + e] = win[0][j];
#pragma unroll
        for (int i = 1; i <= H; i++) {
            const float2 l = f_mul(win[i][0], rp);
            st.f[(2 * H + i) * st.plane + e] = l;
#pragma unroll
            for (int j = 1; j < W; j++) win[i][j] = f_sub(win[i][j], f_mul(l, win[0][j]));
        }
#pragma unroll
        for (int i = 0; i < H; i++) {
#pragma unroll
            for (int j = 0; j < W - 1; j++) win[i][j] = win[i + 1][j + 1];
            win[i][W - 1] = make_float2(0.f, 0.f);
        }
        const int rn = k + 1 + H;
#pragma unroll
        for (int j = 0; j < W; j++) {
            const int d = j - H;
            win[H][j] = (rn < Np && k + 1 + j < Np) ? to_f(entry(rn, d)) : make_float2(0.f, 0.f);
        }
    }
    return ok;
}

// Mixed solve with stored FP32 factors: x = U^-1 L^-1 P b in FP32 from the
// FP64 right-hand side, then `refine` steps of FP64 iterative refinement
// (r = b - A x with A = entry(k, d) and b = rhs(k, r) in FP64, correction
// solved with the FP32 factors, x += correction in FP64), as band_solve_mixed
// with the factorisation read instead of recomputed.  The factors of several
// rows are loaded together as in band_solve_stored.
template <int H, int MAXR, int NR, class Entry, class Rhs, class Out>
__host__ __device__ void band_solve_stored_mixed(int Np, const BandRefF& st, int refine, Entry entry, Rhs rhs,
                                                 Out out) {
    constexpr int W = 2 * H + 1;
    constexpr int PF = 4;
    double2 x[MAXR][NR];
    auto lu_solve = [&](auto b, bool add) {
        float2 y[MAXR][NR];
        float2 wr[H + 1][NR];
#pragma unroll
        for (int i = 0; i <= H; i++)
#pragma unroll
            for (int r = 0; r < NR; r++) wr[i][r] = i < Np ? to_f(b(i, r)) : make_float2(0.f, 0.f);
        for (int k0 = 0; k0 < Np; k0 += PF) {
            int pvs[PF];
            float2 lm[PF][H];
#pragma unroll
            for (int u = 0; u < PF; u++) {
                const int k = k0 + u < Np ? k0 + u : Np - 1;
                const long long e = st.i0 + (long long)k * st.lanes;
                pvs[u] = RX_LDG(&st.pv[e]);
#pragma unroll
                for (int i = 1; i <= H; i++) lm[u][i - 1] = RX_LDG(&st.f[(2 * H + i) * st.plane + e]);
            }
#pragma unroll
            for (int u = 0; u < PF; u++) {
                const int k = k0 + u;
                if (k >= Np) break;
                const int p = pvs[u];
#pragma unroll
                for (int i = 1; i <= H; i++) {
                    const bool sw = (p == i);
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        const float2 t0 = wr[0][r], ti = wr[i][r];
                        wr[0][r] = sw ? ti : t0;
                        wr[i][r] = sw ? t0 : ti;
                    }
                }
#pragma unroll
                for (int r = 0; r < NR; r++) y[k][r] = wr[0][r];
#pragma unroll
                for (int i = 1; i <= H; i++)
#pragma unroll
                    for (int r = 0; r < NR; r++) wr[i][r] = f_sub(wr[i][r], f_mul(lm[u][i - 1], wr[0][r]));
#pragma unroll
                for (int i = 0; i < H; i++)
#pragma unroll
                    for (int r = 0; r < NR; r++) wr[i][r] = wr[i + 1][r];
                const int rn = k + 1 + H;
#pragma unroll
                for (int r = 0; r < NR; r++) wr[H][r] = rn < Np ? to_f(b(rn, r)) : make_float2(0.f, 0.f);
            }
        }
        float2 xs[W][NR];
#pragma unroll
        for (int j = 0; j < W; j++)
#pragma unroll
            for (int r = 0; r < NR; r++) xs[j][r] = make_float2(0.f, 0.f);
        for (int k = Np - 1; k >= 0; k--) {
            const long long e = st.i0 + (long long)k * st.lanes;
            const float2 rd = RX_LDG(&st.f[e]);
            float2 uu[W];
#pragma unroll
            for (int j = 1; j < W; j++) uu[j] = RX_LDG(&st.f[j * st.plane + e]);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                float2 sm = y[k][r];
#pragma unroll
                for (int j = 1; j < W; j++) sm = f_sub(sm, f_mul(uu[j], xs[j - 1][r]));
                const float2 xk = f_mul(sm, rd);
#pragma unroll
                for (int j = W - 1; j > 0; j--) xs[j][r] = xs[j - 1][r];
                xs[0][r] = xk;
                x[k][r] = add ? c_add(x[k][r], to_d(xk)) : to_d(xk);
            }
        }
    };
    lu_solve([&](int k, int r) { return rhs(k, r); }, false);
    for (int it = 0; it < refine; it++) {
        lu_solve(
            [&](int k, int r) {
                double2 v = rhs(k, r);
#pragma unroll
                for (int d = -H; d <= H; d++)
                    if (k + d >= 0 && k + d < Np) v = c_sub(v, c_mul(entry(k, d), x[k + d][r]));
                return v;
            },
            true);
    }
    for (int k = 0; k < Np; k++)
#pragma unroll
        for (int r = 0; r < NR; r++) out(k, r, x[k][r]);
}

// Entry (k, dd) of the parity-`par` Phi system of the m-block at block row
// base: alpha^4 I + alpha^2 C2 + alpha C1 + alpha^-1 Cm1 + C0 (rows par + 2k).
__host__ __device__ inline double2 phi_entry(const RexiDev& d, int base, int par, double2 a, double2 a2, double2 ainv,
                                             double2 a4, int k, int dd) {
    const size_t nc5 = (size_t)d.ncplx * 5;
    const int row = base + par + 2 * k;
    const double2* c = d.Cphi + (size_t)row * 5 + (dd + 2);
    double2 v = c_mul(a2, ld(c));
    v = c_add(v, c_mul(a, ld(c + nc5)));
    v = c_add(v, c_mul(ainv, ld(c + 2 * nc5)));
    v = c_add(v, ld(c + 3 * nc5));
    if (dd == 0) v = c_add(v, a4);
    return v;
}
// Entry (k, dd) of the parity-`par` velocity system: alpha^2 I + Cvel.
__host__ __device__ inline double2 vel_entry(const RexiDev& d, int base, int par, double2 a2, int k, int dd) {
    const int row = base + par + 2 * k;
    double2 v = ld(&d.Cvel[(size_t)row * 3 + dd + 1]);
    if (dd == 0) v = c_add(v, a2);
    return v;
}
__host__ __device__ inline BandRef band_ref(double2* f, signed char* pv, const RexiDev& d, long long gl, int base,
                                            int N, int par) {
    return BandRef{f, pv, d.plane, gl + (long long)(base + (par ? (N + 1) / 2 : 0)) * d.lanes, d.lanes};
}
__host__ __device__ inline BandRefF band_ref_f(float2* f, signed char* pv, const RexiDev& d, long long gl, int base,
                                               int N, int par) {
    return BandRefF{f, pv, d.plane, gl + (long long)(base + (par ? (N + 1) / 2 : 0)) * d.lanes, d.lanes};
}

// Factor the Phi and velocity systems of one pole and one m-block (both
// parities) into the stored planes of d; gl = g * ncplx * lanes + lane.
// Returns false on a zero pivot.  Only the Coriolis case has banded systems.
__host__ __device__ inline bool rexi_factor_lane(const RexiDev& d, int m, double2 a, long long gl) {
    const int am = m < 0 ? -m : m;
    const int N = d.L + 1 - am;
    const int base = block_off(d.L, m);
    const double2 a2 = c_mul(a, a), a4 = c_mul(a2, a2);
    const double2 ainv = c_div(make_double2(1, 0), a);
    bool ok = true;
    for (int par = 0; par < 2; par++) {
        const int Np = (N - par + 1) >> 1;
        if (Np <= 0) continue;
        ok = band_factor_store<2>(
                 Np, [&](int k, int dd) { return phi_entry(d, base, par, a, a2, ainv, a4, k, dd); },
                 band_ref(d.fphi, d.pphi, d, gl, base, N, par)) && ok;
        ok = band_factor_store<1>(
                 Np, [&](int k, int dd) { return vel_entry(d, base, par, a2, k, dd); },
                 band_ref(d.fvel, d.pvel, d, gl, base, N, par)) && ok;
    }
    return ok;
}

// The FP32 factors of the Phi and velocity systems of one pole and one m-block
// (both parities), for the mixed form's stored-factor solves.
__host__ __device__ inline bool rexi_factor_lane_f(const RexiDev& d, int m, double2 a, long long gl) {
    const int am = m < 0 ? -m : m;
    const int N = d.L + 1 - am;
    const int base = block_off(d.L, m);
    const double2 a2 = c_mul(a, a), a4 = c_mul(a2, a2);
    const double2 ainv = c_div(make_double2(1, 0), a);
    bool ok = true;
    for (int par = 0; par < 2; par++) {
        const int Np = (N - par + 1) >> 1;
        if (Np <= 0) continue;
        ok = band_factor_store_f<2>(
                 Np, [&](int k, int dd) { return phi_entry(d, base, par, a, a2, ainv, a4, k, dd); },
                 band_ref_f(d.fphi32, d.pphi, d, gl, base, N, par)) && ok;
        ok = band_factor_store_f<1>(
                 Np, [&](int k, int dd) { return vel_entry(d, base, par, a2, k, dd); },
                 band_ref_f(d.fvel32, d.pvel, d, gl, base, N, par)) && ok;
    }
    return ok;
}

// Phi of one pole and one m-block (both l-parities): the banded Phi systems
// with Coriolis, the spectral Helmholtz solve without; writes the unscaled phi
// of the block's N = L+1-|m| rows; returns false on a zero pivot.  Shared by
// the Robert form and the non-Robert form (whose tables and pole-independent
// vectors differ, not the arithmetic).
template <int MAXN, bool MIXED = false, bool STORED = false>
__host__ __device__ bool rexi_phi(const RexiDev& d, int m, double2 a, double2* phi, long long gl = 0) {
    const int L = d.L;
    const int am = m < 0 ? -m : m;
    const int N = L + 1 - am;
    const int base = block_off(L, m);
    const double T = d.T, P = d.P, ir = d.ir;
    const int nc = d.ncplx;
    const double2* V = d.V;
    const double2 a2 = c_mul(a, a), a3 = c_mul(a2, a), a4 = c_mul(a2, a2);
    const double2 ainv = c_div(make_double2(1, 0), a);
    bool ok = true;
    if (d.coriolis) {
        // right-hand side weights of the 10 pole-independent vectors (the
        // non-Robert form has the same weights; its vectors 0, 1, 4, 5 come from
        // the non-Robert div0 and eta0 and 7, 8, 9 are the grid products
        // grad_lat(mu) u0, grad_lat(mu) mu2 u0, grad_lat(mu) mu v0)
        double2 s[10];
        s[0] = c_scale(a2, P);                       // div0
        s[1] = c_scale(a, -P * T);                    // mu(eta0)
        s[2] = a3;                                    // phi0
        s[3] = c_scale(a, 2.0 * T * T);               // mu2(phi0)
        s[4] = make_double2(T * T * P, 0);            // mu2(div0)
        s[5] = c_scale(ainv, -P * T * T * T);         // mu2(mu(eta0))
        s[6] = c_scale(ainv, T * T * T * T);          // mu2(mu2(phi0))
        s[7] = c_scale(a, -P * T * ir);               // W1 = u0 - mu2 u0
        s[8] = c_scale(ainv, P * T * T * T * ir);     // W2 = mu2 u0 - mu2 mu2 u0
        s[9] = make_double2(2.0 * P * T * T * ir, 0); // W3 = mu v0 - mu2 mu v0
        for (int par = 0; par < 2; par++) {
            const int Np = (N - par + 1) >> 1;
            if (Np <= 0) continue;
            auto entry = [&](int k, int dd) -> double2 { return phi_entry(d, base, par, a, a2, ainv, a4, k, dd); };
            auto rhs = [&](int k, int) -> double2 {
                const int row = base + par + 2 * k;
                double2 v = make_double2(0, 0);
#pragma unroll
                for (int q = 0; q < 10; q++) v = c_add(v, c_mul(s[q], ld(&V[(size_t)q * nc + row])));
                return v;
            };
            auto out = [&](int k, int, double2 x) { phi[par + 2 * k] = x; };
            if constexpr (STORED)
                band_solve_stored<2, (MAXN + 1) / 2, 1>(Np, band_ref(d.fphi, d.pphi, d, gl, base, N, par), rhs, out);
            else if constexpr (MIXED)
                ok = band_solve_mixed<2, (MAXN + 1) / 2, 1>(Np, d.refine, entry, rhs, out) && ok;
            else
                ok = band_solve<2, (MAXN + 1) / 2, 1>(Np, entry, rhs, out) && ok;
        }
    } else {
        // phi = (P div0 + a phi0) / (a^2 + (P/r^2) n(n+1)) (spec_solve_helmholtz)
        for (int i = 0; i < N; i++) {
            const int row = base + i;
            const double n = am + i;
            const double2 rhs = c_add(c_scale(ld(&V[row]), P), c_mul(a, ld(&V[(size_t)2 * nc + row])));
            const double2 den = c_add(a2, make_double2(P / (d.r * d.r) * n * (n + 1.0), 0));
            phi[i] = c_div(rhs, den);
        }
    }
    return ok;
}

// One pole, one m-block: Phi solve (both l-parities), velocity right-hand
// sides and the two velocity solves.  Writes the unscaled phi, u, v of the
// block's N = L+1-|m| rows to phi / ra / rb; returns false on a zero pivot.
// STORED: substitutions only, with the factors rexi_factor_lane stored
// (gl as there).
template <int MAXN, bool MIXED = false, bool STORED = false>
__host__ __device__ bool rexi_lane(const RexiDev& d, int m, double2 a, double2* phi, double2* ra, double2* rb,
                                   long long gl = 0) {
    const int L = d.L;
    const int am = m < 0 ? -m : m;
    const int N = L + 1 - am;
    const int base = block_off(L, m);
    const double T = d.T, ir = d.ir;
    const int nc = d.ncplx;
    const double2* V = d.V;
    const double2 a2 = c_mul(a, a);
    const double2 ainv = c_div(make_double2(1, 0), a);
    const double dm = m;

    bool ok = rexi_phi<MAXN, MIXED, STORED>(d, m, a, phi, gl);
    if (d.coriolis) {
        // rhsa = a u0 + a ir i m phi - T mu(v0) - T ir mu(D phi)
        // rhsb = T mu(u0) + T ir mu(i m phi) + a v0 + a ir D phi
        // D phi of every row, parked in ra until the right-hand sides are formed
        for (int i = 0; i < N; i++) {
            const double* cf = d.coef + (size_t)(base + i) * 4;
            const double2 lo = i > 0 ? phi[i - 1] : make_double2(0, 0);
            const double2 hi = i + 1 < N ? phi[i + 1] : make_double2(0, 0);
            ra[i] = c_add(c_scale(lo, RX_LDG(cf + 2)), c_scale(hi, RX_LDG(cf + 3)));
        }
        double2 dprev = make_double2(0, 0);  // D phi of row i-1 (ra[i-1] is overwritten by then)
        for (int i = 0; i < N; i++) {
            const int row = base + i;
            const double* cf = d.coef + (size_t)row * 4;
            const double Rl = RX_LDG(cf), Sh = RX_LDG(cf + 1);
            const double2 dcur = ra[i];
            const double2 dnext = i + 1 < N ? ra[i + 1] : make_double2(0, 0);
            const double2 plo = i > 0 ? phi[i - 1] : make_double2(0, 0);
            const double2 phi_hi = i + 1 < N ? phi[i + 1] : make_double2(0, 0);
            const double2 mud = c_add(c_scale(dprev, Rl), c_scale(dnext, Sh));  // mu(D phi)_i
            const double2 mup = c_add(c_scale(plo, Rl), c_scale(phi_hi, Sh));   // mu(phi)_i
            const double2 u0 = ld(&V[(size_t)10 * nc + row]), v0 = ld(&V[(size_t)11 * nc + row]);
            const double2 mv = ld(&V[(size_t)12 * nc + row]), mu0 = ld(&V[(size_t)13 * nc + row]);
            double2 xa = c_mul(a, u0);
            xa = c_add(xa, c_mul(a, c_scale(c_im(phi[i], dm), ir)));
            xa = c_sub(xa, c_scale(mv, T));
            xa = c_sub(xa, c_scale(mud, T * ir));
            double2 xb = c_scale(mu0, T);
            xb = c_add(xb, c_scale(c_im(mup, dm), T * ir));
            xb = c_add(xb, c_mul(a, v0));
            xb = c_add(xb, c_mul(a, c_scale(dcur, ir)));
            ra[i] = xa;
            rb[i] = xb;
            dprev = dcur;
        }
        for (int par = 0; par < 2; par++) {
            const int Np = (N - par + 1) >> 1;
            if (Np <= 0) continue;
            auto entry = [&](int k, int dd) -> double2 { return vel_entry(d, base, par, a2, k, dd); };
            // u and v share the matrix: one factorisation, two right-hand sides
            auto rhs2 = [&](int k, int r) -> double2 { return r == 0 ? ra[par + 2 * k] : rb[par + 2 * k]; };
            auto out2 = [&](int k, int r, double2 x) {
                if (r == 0) ra[par + 2 * k] = x;
                else rb[par + 2 * k] = x;
            };
            if constexpr (STORED)
                band_solve_stored<1, (MAXN + 1) / 2, 2>(Np, band_ref(d.fvel, d.pvel, d, gl, base, N, par), rhs2, out2);
            else if constexpr (MIXED)
                ok = band_solve_mixed<1, (MAXN + 1) / 2, 2>(Np, d.refine, entry, rhs2, out2) && ok;
            else
                ok = band_solve<1, (MAXN + 1) / 2, 2>(Np, entry, rhs2, out2) && ok;
        }
    } else {
        // u = (u0 + ir i m phi)/a; v = (v0 + ir D phi)/a
        for (int i = 0; i < N; i++) {
            const int row = base + i;
            const double* cf = d.coef + (size_t)row * 4;
            const double2 lo = i > 0 ? phi[i - 1] : make_double2(0, 0);
            const double2 hi = i + 1 < N ? phi[i + 1] : make_double2(0, 0);
            const double2 dp = c_add(c_scale(lo, RX_LDG(cf + 2)), c_scale(hi, RX_LDG(cf + 3)));
            ra[i] = c_mul(ainv, c_add(ld(&V[(size_t)10 * nc + row]), c_scale(c_im(phi[i], dm), ir)));
            rb[i] = c_mul(ainv, c_add(ld(&V[(size_t)11 * nc + row]), c_scale(dp, ir)));
        }
    }
    return ok;
}

// Non-Robert form (SWERexiSPH.hpp:137-244), velocity phase of one pole and one
// m-block, once the pole's grid-valued gradients of phi have come back as
// spectra (complex layout n*n+n+m): cx = F(grad_lon phi) = F(I(i m phi)/cos phi),
// cy = F(grad_lat phi) = F(I((1-mu^2) d phi/dmu)/cos phi).  With
// a_ = u0 + ir cx and b_ = v0 + ir cy:
//   Coriolis:  rhsa = a a_ - T mu(b_), rhsb = T mu(a_) + a b_, then the two
//              velocity solves (same matrix as the Robert form);
//   otherwise: u = a_ / a, v = b_ / a.
// Writes the unscaled u, v of the block's rows to ra / rb.
template <int MAXN, bool MIXED = false, bool STORED = false>
__host__ __device__ bool rexi_s0_vel(const RexiDev& d, int m, double2 a, const double2* cx, const double2* cy,
                                     double2* ra, double2* rb, long long gl = 0) {
    const int L = d.L;
    const int am = m < 0 ? -m : m;
    const int N = L + 1 - am;
    const int base = block_off(L, m);
    const double T = d.T, ir = d.ir;
    const int nc = d.ncplx;
    const double2* V = d.V;
    const double2 a2 = c_mul(a, a);
    const double2 ainv = c_div(make_double2(1, 0), a);
    for (int i = 0; i < N; i++) {
        const int row = base + i, n = am + i, ci = n * n + n + m;
        ra[i] = c_add(ld(&V[(size_t)10 * nc + row]), c_scale(ld(&cx[ci]), ir));
        rb[i] = c_add(ld(&V[(size_t)11 * nc + row]), c_scale(ld(&cy[ci]), ir));
    }
    bool ok = true;
    if (d.coriolis) {
        double2 aprev = make_double2(0, 0), bprev = make_double2(0, 0);  // a_, b_ of row i-1
        for (int i = 0; i < N; i++) {
            const double* cf = d.coef + (size_t)(base + i) * 4;
            const double Rl = RX_LDG(cf), Sh = RX_LDG(cf + 1);
            const double2 acur = ra[i], bcur = rb[i];
            const double2 anext = i + 1 < N ? ra[i + 1] : make_double2(0, 0);
            const double2 bnext = i + 1 < N ? rb[i + 1] : make_double2(0, 0);
            const double2 mua = c_add(c_scale(aprev, Rl), c_scale(anext, Sh));  // mu(a_)_i
            const double2 mub = c_add(c_scale(bprev, Rl), c_scale(bnext, Sh));  // mu(b_)_i
            ra[i] = c_sub(c_mul(a, acur), c_scale(mub, T));
            rb[i] = c_add(c_scale(mua, T), c_mul(a, bcur));
            aprev = acur;
            bprev = bcur;
        }
        for (int par = 0; par < 2; par++) {
            const int Np = (N - par + 1) >> 1;
            if (Np <= 0) continue;
            auto entry = [&](int k, int dd) -> double2 { return vel_entry(d, base, par, a2, k, dd); };
            auto rhs2 = [&](int k, int r) -> double2 { return r == 0 ? ra[par + 2 * k] : rb[par + 2 * k]; };
            auto out2 = [&](int k, int r, double2 x) {
                if (r == 0) ra[par + 2 * k] = x;
                else rb[par + 2 * k] = x;
            };
            if constexpr (STORED)
                band_solve_stored<1, (MAXN + 1) / 2, 2>(Np, band_ref(d.fvel, d.pvel, d, gl, base, N, par), rhs2, out2);
            else if constexpr (MIXED)
                ok = band_solve_mixed<1, (MAXN + 1) / 2, 2>(Np, d.refine, entry, rhs2, out2) && ok;
            else
                ok = band_solve<1, (MAXN + 1) / 2, 2>(Np, entry, rhs2, out2) && ok;
        }
    } else {
        for (int i = 0; i < N; i++) {
            ra[i] = c_mul(ainv, ra[i]);
            rb[i] = c_mul(ainv, rb[i]);
        }
    }
    return ok;
}

}  // namespace sphgpu
