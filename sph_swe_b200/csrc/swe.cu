// Fused RK4 shallow-water step on the sphere (FP64 plain method).
//
// Reference: AppSWE::p_run_euler_timestep_update (AppSWE.hpp:574-659) driven
// by TimesteppingRK::run_rk_timestep order 4 (TimesteppingRK.hpp:310-392).
// The reference evaluates every operator through lazily transformed fields;
// the projection points it produces for the nonlinear advective form are
// (H = I(h), U = I(u), V = I(v), c = cos(phi), iM = times i*m,
//  D = truncated (1-mu^2) d/dmu recurrence, F = analysis, I = synthesis):
//
//   h_t = -(1/a) [ F(I(iM F(HU))/c) + F(I(D F(cHV))/c^2) ]
//   u_t = -(g/a) F(I(iM h)/c) + 2 Omega F(mu V) - (1/a)[F(U I(iM u)/c) + F(V I(D u)/c)]
//   v_t = -(g/a) F(I(D h)/c)  - 2 Omega F(mu U) - (1/a)[F(U I(iM v)/c) + F(V I(D v)/c)]
//   (+ nu/a^2 laplace for each field)
//
// This file keeps exactly those projection points and reorganises the work
// into waves (F is linear, so a sum of projections is one projection of the
// sum; I(iM x) is the longitude derivative of I(x), taken in Fourier space; a
// division by a function of latitude commutes with the longitude FFT):
//   W1  spectral: x, D x for x in {h,u,v}; Legendre synthesis of 6 fields;
//       inverse FFTs to 9 grids {H,U,V, H_l,U_l,V_l, H_m,U_m,V_m}
//   W2  pointwise products -> 4 grids {HU, cHV, u-term, v-term}; FFT +
//       Legendre analysis (4 fields)
//   W3  spectral: A = F(HU), B = D F(cHV); Legendre synthesis (2 fields);
//       Fourier-space latitude scaling i m A/c + B/c^2 (no FFT needed)
//   W4  Legendre analysis of the h term; combine into the RK stage.
// The linear forms (AppSWE.hpp:590-621) use the same waves with h0 in place
// of H in the flux products and no advection terms; the Robert linear form
// divides by c^2 and takes the geopotential gradient in spectral space.
// With nonlinear = 1 the reference ignores use_robert_functions
// (AppSWE.hpp:622-650) and so does this file.
//
// nonlinear = 2 selects a form the reference does not have: the full
// nonlinear equations in vorticity-divergence form with the Robert velocity
// U = u c, V = v c on the grid (the NCAR spectral model's formulation; state
// [h | zeta | delta], physical units).  With eta = zeta + 2 Omega mu:
//   zeta_t  = -(1/a) div(eta v),  h_t = -(1/a) div(h v)
//   delta_t =  (1/a) curl(eta v) - (1/a^2) lap(g h + (U^2 + V^2) / (2 c^2))
// One wave each way: the exact vector synthesis of (a zeta, a delta) to U, V
// plus the syntheses of zeta and h (4 fields, degree L+1 kept); pointwise
// A, B = eta (U, V) / c^2, C, D = h (U, V) / c^2, E; 5 analyses of degree L+1;
// div / curl by the integration-by-parts recurrence of the vector analysis.
// No grid value is differentiated, so the truncation error is not divided by
// cos^2 at the polar rings, and div has no l = 0 term: h_00 (mass) and
// zeta_00 change by rounding only.
// The whole step (4 stages + update) is captured once in a CUDA graph.
#include "common.cuh"
#include "identities.cuh"

#include <algorithm>
#include <cstring>

namespace sphgpu {

struct RKState {
    double2* X6 = nullptr;
    double2* F6 = nullptr;
    double* G9 = nullptr;
    double* G4 = nullptr;
    double2* F4 = nullptr;
    double2* T4 = nullptr;
    double2* X2 = nullptr;
    double2* F2 = nullptr;
    double2* Fh = nullptr;
    double2* Th = nullptr;
    double2* K = nullptr;    // [stage][member][3][nlm]
    double* dts = nullptr;   // per-member dt (device)
    int* flag = nullptr;     // non-finite flag (device)
    int nmem = 0;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    double* state = nullptr;
    cudaStream_t stream = nullptr;
    sph_swe_params params{};
    std::vector<double> dts_h;
    int launches = 0;  // kernel launches in one replay of the step graph
};

static void rk_release(RKState* r) {
    if (!r) return;
    if (r->exec) cudaGraphExecDestroy(r->exec);
    if (r->graph) cudaGraphDestroy(r->graph);
    void* bufs[] = {r->X6, r->F6, r->G9, r->G4, r->F4, r->T4, r->X2, r->F2, r->Fh, r->Th, r->K, r->dts, r->flag};
    for (void* p : bufs)
        if (p) cudaFree(p);
    delete r;
}

// stage buffers for nmem members of one truncation
static int rk_buffers(const Handle* h, RKState* r, int nmem) {
    r->nmem = nmem;
    const size_t nlm = h->nlm, fou = (size_t)(h->L + 1) * h->nlat, sp = h->nspat;
    const size_t M = nmem;
    // X6 also holds the 5 degree-(L+1) analyses of the vorticity-divergence form
    const size_t nlmp = (size_t)(h->L + 2) * (h->L + 3) / 2;
    SPH_CUDA_TRY(cudaMalloc(&r->X6, sizeof(double2) * std::max(6 * nlm, 5 * nlmp) * M));
    SPH_CUDA_TRY(cudaMalloc(&r->F6, sizeof(double2) * 6 * fou * M));
    SPH_CUDA_TRY(cudaMalloc(&r->G9, sizeof(double) * 9 * sp * M));
    SPH_CUDA_TRY(cudaMalloc(&r->G4, sizeof(double) * 4 * sp * M));
    SPH_CUDA_TRY(cudaMalloc(&r->F4, sizeof(double2) * 4 * fou * M));
    SPH_CUDA_TRY(cudaMalloc(&r->T4, sizeof(double2) * 4 * nlm * M));
    SPH_CUDA_TRY(cudaMalloc(&r->X2, sizeof(double2) * 2 * nlm * M));
    SPH_CUDA_TRY(cudaMalloc(&r->F2, sizeof(double2) * 2 * fou * M));
    SPH_CUDA_TRY(cudaMalloc(&r->Fh, sizeof(double2) * fou * M));
    SPH_CUDA_TRY(cudaMalloc(&r->Th, sizeof(double2) * nlm * M));
    SPH_CUDA_TRY(cudaMalloc(&r->K, sizeof(double2) * 4 * 3 * nlm * M));
    SPH_CUDA_TRY(cudaMalloc(&r->dts, sizeof(double) * M));
    SPH_CUDA_TRY(cudaMalloc(&r->flag, sizeof(int)));
    SPH_CUDA_TRY(cudaMemset(r->flag, 0, sizeof(int)));
    return SPH_OK;
}

void rk_free(Handle* h) {
    rk_release(static_cast<RKState*>(h->rk));
    h->rk = nullptr;
}

void rk_invalidate(Handle* h) {
    if (RKState* r = static_cast<RKState*>(h->rk)) r->state = nullptr;
}

static int rk_alloc(Handle* h, int nmem) {
    RKState* r = static_cast<RKState*>(h->rk);
    if (r && r->nmem >= nmem) return SPH_OK;
    cudaDeviceSynchronize();
    rk_free(h);
    r = new RKState();
    h->rk = r;
    return rk_buffers(h, r, nmem);
}

// ------------------------------------------------------------------ kernels
// index helpers for the real packed layout: block y = m, threads over n
struct SweConst {
    double a, g, omega, h0, visc;
    int mode;  // 0 nonlinear, 1 linear, 2 linear Robert
};

__device__ __forceinline__ double2 ld2(const double2* p, int L, int n, int m) {
    if (n < m || n > L) return make_double2(0, 0);
    return p[pidx(L, n, m)];
}

// stage input x = S + (coef*dt_member) K_prev; writes X6 = [x_h, x_u, x_v, D x_h, D x_u, D x_v]
__global__ void k_rk_prep(const double2* __restrict__ S, const double2* __restrict__ Kp, double coef,
                          const double* __restrict__ dts, double2* __restrict__ X6, int L, int nlm) {
    const int m = blockIdx.y;
    const int n = m + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const int mem = blockIdx.z / 3, q = blockIdx.z - mem * 3;
    const double c = Kp ? coef * dts[mem] : 0.0;
    const double2* s = S + ((size_t)mem * 3 + q) * nlm;
    const double2* kp = Kp ? Kp + ((size_t)mem * 3 + q) * nlm : nullptr;
    auto x_at = [&](int nn) -> double2 {
        if (nn < m || nn > L) return make_double2(0, 0);
        const int k = pidx(L, nn, m);
        double2 v = s[k];
        if (kp) {
            const double2 t = kp[k];
            v.x += c * t.x;
            v.y += c * t.y;
        }
        return v;
    };
    const double2 x = x_at(n), lo = x_at(n - 1), hi = x_at(n + 1);
    const double dn = n, dm = m;
    const double cl = (-dn + 1.0) * idR(dn - 1, dm), ch = (dn + 2.0) * idS(dn + 1, dm);
    const int k = pidx(L, n, m);
    double2* out = X6 + (size_t)mem * 6 * nlm;
    out[(size_t)q * nlm + k] = x;
    out[(size_t)(3 + q) * nlm + k] = make_double2(cl * lo.x + ch * hi.x, cl * lo.y + ch * hi.y);
}

// G9 per member: [H, U, V, H_l, U_l, V_l, H_m, U_m, V_m] -> G4 [A, B, u-term, v-term]
__global__ void k_swe_pointwise(const double* __restrict__ G9, double* __restrict__ G4, const double* __restrict__ mu,
                                const double* __restrict__ cosphi, int nlat, int nspat, SweConst k) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nspat) return;
    const int mem = blockIdx.y;
    const int j = idx % nlat;
    const double* g = G9 + (size_t)mem * 9 * nspat + idx;
    double* o = G4 + (size_t)mem * 4 * nspat + idx;
    const double H = g[0], U = g[(size_t)nspat], V = g[2 * (size_t)nspat];
    const double Hl = g[3 * (size_t)nspat], Ul = g[4 * (size_t)nspat], Vl = g[5 * (size_t)nspat];
    const double Hm = g[6 * (size_t)nspat], Um = g[7 * (size_t)nspat], Vm = g[8 * (size_t)nspat];
    const double c = cosphi[j], m_ = mu[j];
    const double ga = k.g / k.a, ia = 1.0 / k.a, to = 2.0 * k.omega;
    double A, B, ut, vt;
    if (k.mode == 0) {
        A = H * U;
        B = c * (H * V);
        ut = -ga * (Hl / c) + to * (m_ * V) - ia * (U * (Ul / c) + V * (Um / c));
        vt = -ga * (Hm / c) - to * (m_ * U) - ia * (U * (Vl / c) + V * (Vm / c));
    } else if (k.mode == 1) {
        A = k.h0 * U;
        B = k.h0 * (c * V);
        ut = -ga * (Hl / c) + to * (m_ * V);
        vt = -ga * (Hm / c) - to * (m_ * U);
    } else {
        A = k.h0 * U;
        B = k.h0 * V;
        ut = to * (m_ * V);
        vt = -to * (m_ * U);
    }
    o[0] = A;
    o[(size_t)nspat] = B;
    o[2 * (size_t)nspat] = ut;
    o[3 * (size_t)nspat] = vt;
}

// X2 = [A, D B] from T4 = [A, B, ., .]
__global__ void k_rk_mid(const double2* __restrict__ T4, double2* __restrict__ X2, int L, int nlm) {
    const int m = blockIdx.y;
    const int n = m + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const int mem = blockIdx.z;
    const double2* A = T4 + (size_t)mem * 4 * nlm;
    const double2* B = A + nlm;
    double2* o = X2 + (size_t)mem * 2 * nlm;
    const int k = pidx(L, n, m);
    o[k] = A[k];
    const double dn = n, dm = m;
    const double cl = (-dn + 1.0) * idR(dn - 1, dm), ch = (dn + 2.0) * idS(dn + 1, dm);
    const double2 lo = ld2(B, L, n - 1, m), hi = ld2(B, L, n + 1, m);
    o[nlm + k] = make_double2(cl * lo.x + ch * hi.x, cl * lo.y + ch * hi.y);
}

// Fh[m][j] = c (i m A_m(j) / c^pa + B_m(j) / c^2)   (pa = 1, or 2 for Robert):
// the integrand times c, bounded at the polar rings, for the analysis with the
// weights w / c
__global__ void k_fourier_h(const double2* __restrict__ F2, double2* __restrict__ Fh, const double* __restrict__ cosphi,
                            int nlat, int mF, int pa) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t fou = (size_t)mF * nlat;
    if (idx >= fou) return;
    const int mem = blockIdx.y;
    const int m = idx / nlat, j = idx - m * nlat;
    const double2 a = F2[(size_t)mem * 2 * fou + idx], b = F2[(size_t)mem * 2 * fou + fou + idx];
    const double c = cosphi[j];
    const double ca = pa == 1 ? 1.0 : c;
    // the synthesis Fourier coefficients lack the 2 pi longitude quadrature
    // weight that the ring analysis applies
    const double tp = 2.0 * kPi;
    Fh[(size_t)mem * fou + idx] = make_double2(tp * (-m * a.y / ca + b.x / c), tp * (m * a.x / ca + b.y / c));
}

// K_s = [-(1/a) Th, T4[2], T4[3]] (+ Robert spectral gradient terms) + viscosity
__global__ void k_rk_stage_out(const double2* __restrict__ S, const double2* __restrict__ Kp, double coef,
                               const double* __restrict__ dts, const double2* __restrict__ T4, const double2* __restrict__ Th,
                               double2* __restrict__ Ks, int L, int nlm, SweConst kc) {
    const int m = blockIdx.y;
    const int n = m + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const int mem = blockIdx.z;
    const int k = pidx(L, n, m);
    const double c = Kp ? coef * dts[mem] : 0.0;
    const double2* s = S + (size_t)mem * 3 * nlm;
    const double2* kp = Kp ? Kp + (size_t)mem * 3 * nlm : nullptr;
    auto x_at = [&](int q, int nn) -> double2 {
        if (nn < m || nn > L) return make_double2(0, 0);
        const int kk = pidx(L, nn, m);
        double2 v = s[(size_t)q * nlm + kk];
        if (kp) {
            const double2 t = kp[(size_t)q * nlm + kk];
            v.x += c * t.x;
            v.y += c * t.y;
        }
        return v;
    };
    const double2* t4 = T4 + (size_t)mem * 4 * nlm;
    const double ia = 1.0 / kc.a;
    const double2 th = Th[(size_t)mem * nlm + k];
    double2 ht = make_double2(-ia * th.x, -ia * th.y);
    double2 ut = t4[2 * (size_t)nlm + k];
    double2 vt = t4[3 * (size_t)nlm + k];
    const double dn = n, dm = m;
    if (kc.mode == 2) {
        // -(g/a) iM h  and  -(g/a) D h in spectral space
        const double ga = kc.g / kc.a;
        const double2 xh = x_at(0, n), lo = x_at(0, n - 1), hi = x_at(0, n + 1);
        ut.x += -ga * (-dm * xh.y);
        ut.y += -ga * (dm * xh.x);
        const double cl = (-dn + 1.0) * idR(dn - 1, dm), ch = (dn + 2.0) * idS(dn + 1, dm);
        vt.x += -ga * (cl * lo.x + ch * hi.x);
        vt.y += -ga * (cl * lo.y + ch * hi.y);
    }
    if (kc.visc != 0.0) {
        const double sc = kc.visc / (kc.a * kc.a) * (-dn * (dn + 1.0));
        const double2 xh = x_at(0, n), xu = x_at(1, n), xv = x_at(2, n);
        ht.x += xh.x * sc; ht.y += xh.y * sc;
        ut.x += xu.x * sc; ut.y += xu.y * sc;
        vt.x += xv.x * sc; vt.y += xv.y * sc;
    }
    double2* o = Ks + (size_t)mem * 3 * nlm;
    o[k] = ht;
    o[(size_t)nlm + k] = ut;
    o[2 * (size_t)nlm + k] = vt;
}

// S += dt (K0/6 + K1/3 + K2/3 + K3/6); flags non-finite h
__global__ void k_rk_final(double2* __restrict__ S, const double2* __restrict__ K, const double* __restrict__ dts, int nmem,
                           int nlm, int* __restrict__ flag) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t per = (size_t)3 * nlm;
    const size_t tot = per * nmem;
    if (idx >= tot) return;
    const int mem = (int)(idx / per);
    const size_t st = (size_t)nmem * per;
    const double dt = dts[mem];
    const double2 k0 = K[idx], k1 = K[st + idx], k2 = K[2 * st + idx], k3 = K[3 * st + idx];
    const double b0 = 1.0 / 6.0, b1 = 1.0 / 3.0, b2 = 1.0 / 3.0, b3 = 1.0 / 6.0;
    double2 s = S[idx];
    s.x += dt * ((b0 * k0.x) + (b1 * k1.x) + (b2 * k2.x) + (b3 * k3.x));
    s.y += dt * ((b0 * k0.y) + (b1 * k1.y) + (b2 * k2.y) + (b3 * k3.y));
    S[idx] = s;
    if ((idx - (size_t)mem * per) < (size_t)nlm && !(isfinite(s.x) && isfinite(s.y))) atomicOr(flag, 1);
}

// ------------------------------------------------------------------ vorticity-divergence form
// stage input x = S + (coef dt) K_prev of [h, zeta, delta]; writes, in the
// packed layout of degree L+1, X = [U_s, V_s, zeta, h]: the Robert velocity
// spectra of (a zeta, a delta) (inverse Laplacian, then U = i m chi - D psi,
// V = i m psi + D chi with D the untruncated (1-mu^2) d/dmu) and the two
// scalar fields padded with zeros at degree L+1
__global__ void k_vd_prep(const double2* __restrict__ S, const double2* __restrict__ Kp, double coef,
                          const double* __restrict__ dts, double2* __restrict__ X, int L, int nlm, int nlmp, double a) {
    const int m = blockIdx.y;  // 0..L+1
    const int n = m + blockIdx.x * blockDim.x + threadIdx.x;
    const int Lp = L + 1;
    if (n > Lp) return;
    const int mem = blockIdx.z;
    const double c = Kp ? coef * dts[mem] : 0.0;
    const double2* s = S + (size_t)mem * 3 * nlm;
    const double2* kp = Kp ? Kp + (size_t)mem * 3 * nlm : nullptr;
    auto x_at = [&](int q, int nn) -> double2 {
        if (nn < m || nn > L || m > L) return make_double2(0, 0);
        const int kk = pidx(L, nn, m);
        double2 v = s[(size_t)q * nlm + kk];
        if (kp) {
            const double2 t = kp[(size_t)q * nlm + kk];
            v.x += c * t.x;
            v.y += c * t.y;
        }
        return v;
    };
    auto inv = [&](int q, int nn) -> double2 {  // a x / (-nn (nn + 1))
        if (nn <= 0) return make_double2(0, 0);
        const double2 v = x_at(q, nn);
        const double f = -a / ((double)nn * (nn + 1.0));
        return make_double2(v.x * f, v.y * f);
    };
    const int k = pidx(Lp, n, m);
    double2* o = X + (size_t)mem * 4 * nlmp;
    if (m > L) {
        o[k] = o[nlmp + k] = o[2 * (size_t)nlmp + k] = o[3 * (size_t)nlmp + k] = make_double2(0, 0);
        return;
    }
    const double dn = n, dm = m;
    const double cl = (-dn + 1.0) * idR(dn - 1, dm), ch = (dn + 2.0) * idS(dn + 1, dm);
    const double2 psi = inv(1, n), chi = inv(2, n);
    const double2 psl = inv(1, n - 1), psh = inv(1, n + 1), chl = inv(2, n - 1), chh = inv(2, n + 1);
    o[k] = make_double2(-dm * chi.y - (cl * psl.x + ch * psh.x), dm * chi.x - (cl * psl.y + ch * psh.y));
    o[nlmp + k] = make_double2(-dm * psi.y + (cl * chl.x + ch * chh.x), dm * psi.x + (cl * chl.y + ch * chh.y));
    o[2 * (size_t)nlmp + k] = x_at(1, n);
    o[3 * (size_t)nlmp + k] = x_at(0, n);
}

// G4 per member [U, V, zeta, h] -> G5 = c [eta U / c^2, eta V / c^2, h U / c^2, h V / c^2, g h + (U^2 + V^2) / (2 c^2)],
// the five integrands times c for the analysis with the weights w / c (bounded at the polar rings)
__global__ void k_vd_pointwise(const double* __restrict__ G4, double* __restrict__ G5, const double* __restrict__ mu,
                               const double* __restrict__ cosphi, int nlat, int nspat, double grav, double omega) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nspat) return;
    const int mem = blockIdx.y;
    const int j = idx % nlat;
    const double* g = G4 + (size_t)mem * 4 * nspat + idx;
    double* o = G5 + (size_t)mem * 5 * nspat + idx;
    const double U = g[0], V = g[(size_t)nspat], Z = g[2 * (size_t)nspat], H = g[3 * (size_t)nspat];
    const double c = cosphi[j];
    const double ic = 1.0 / c;
    const double eta = Z + 2.0 * omega * mu[j];
    o[0] = eta * U * ic;
    o[(size_t)nspat] = eta * V * ic;
    o[2 * (size_t)nspat] = H * U * ic;
    o[3 * (size_t)nspat] = H * V * ic;
    o[4 * (size_t)nspat] = grav * H * c + 0.5 * (U * U + V * V) * ic;
}

// K_s = [h_t, zeta_t, delta_t] from the degree-(L+1) analyses A5 = [a(A), a(B), a(C), a(D), a(E)]
__global__ void k_vd_stage_out(const double2* __restrict__ S, const double2* __restrict__ Kp, double coef,
                               const double* __restrict__ dts, const double2* __restrict__ A5,
                               double2* __restrict__ Ks, int L, int nlm, int nlmp, double a, double visc) {
    const int m = blockIdx.y;
    const int n = m + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > L) return;
    const int mem = blockIdx.z;
    const int Lp = L + 1;
    const double2* aA = A5 + (size_t)mem * 5 * nlmp;
    auto at = [&](int q, int nn) -> double2 {
        if (nn < m || nn > Lp) return make_double2(0, 0);
        return aA[(size_t)q * nlmp + pidx(Lp, nn, m)];
    };
    const double dn = n, dm = m;
    const double el = (dn + 1.0) * idR(dn - 1, dm), eh = dn * idS(dn + 1, dm);
    const double2 A0 = at(0, n), Al = at(0, n - 1), Ah = at(0, n + 1);
    const double2 B0 = at(1, n), Bl = at(1, n - 1), Bh = at(1, n + 1);
    const double2 C0 = at(2, n), Dl = at(3, n - 1), Dh = at(3, n + 1);
    const double2 E0 = at(4, n);
    // curl and div of (A, B), div of (C, D) on the unit sphere
    const double2 crf = make_double2(-dm * B0.y + el * Al.x - eh * Ah.x, dm * B0.x + el * Al.y - eh * Ah.y);
    const double2 dvf = make_double2(-dm * A0.y - el * Bl.x + eh * Bh.x, dm * A0.x - el * Bl.y + eh * Bh.y);
    const double2 dvh = make_double2(-dm * C0.y - el * Dl.x + eh * Dh.x, dm * C0.x - el * Dl.y + eh * Dh.y);
    const double ia = 1.0 / a, ll = dn * (dn + 1.0);
    double2 ht = make_double2(-ia * dvh.x, -ia * dvh.y);
    double2 zt = make_double2(-ia * dvf.x, -ia * dvf.y);
    double2 dt = make_double2(ia * crf.x + ll * ia * ia * E0.x, ia * crf.y + ll * ia * ia * E0.y);
    const int k = pidx(L, n, m);
    if (visc != 0.0) {
        const double c = Kp ? coef * dts[mem] : 0.0;
        const double sc = -visc * ia * ia * ll;
        double2 x[3];
        for (int q = 0; q < 3; q++) {
            x[q] = S[((size_t)mem * 3 + q) * nlm + k];
            if (Kp) {
                const double2 t = Kp[((size_t)mem * 3 + q) * nlm + k];
                x[q].x += c * t.x;
                x[q].y += c * t.y;
            }
        }
        ht.x += sc * x[0].x; ht.y += sc * x[0].y;
        zt.x += sc * x[1].x; zt.y += sc * x[1].y;
        dt.x += sc * x[2].x; dt.y += sc * x[2].y;
    }
    double2* o = Ks + (size_t)mem * 3 * nlm;
    o[k] = ht;
    o[(size_t)nlm + k] = zt;
    o[2 * (size_t)nlm + k] = dt;
}

// ------------------------------------------------------------------ host pipeline
static SweConst make_const(const sph_swe_params* p) {
    SweConst k;
    k.a = p->radius;
    k.g = p->gravity;
    k.omega = p->omega;
    k.h0 = p->h0;
    k.visc = p->viscosity;
    k.mode = p->nonlinear ? 0 : (p->robert ? 2 : 1);
    return k;
}

// one tendency evaluation of the stage input x = S + coef*dt*Kp into Ks
static int swe_stage(Handle* h, RKState* r, const sph_swe_params* p, const double2* S, const double2* Kp, double coef,
                     double2* Ks, int nmem, cudaStream_t s) {
    const int L = h->L, nlm = h->nlm, nlat = h->nlat, mF = L + 1;
    const long long fou = (long long)mF * nlat;
    const SweConst kc = make_const(p);
    const dim3 gs((L + 1 + 63) / 64, L + 1, 3 * nmem);
    k_rk_prep<<<gs, 64, 0, s>>>(S, Kp, coef, r->dts, r->X6, L, nlm);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = legendre_synthesis_real(h, r->X6, nlm, L, r->F6, fou, 6 * nmem, s, 1)) return rc;
    static const int src9[9] = {0, 1, 2, 0, 1, 2, 3, 4, 5};
    static const int mod9[9] = {0, 0, 0, 1, 1, 1, 0, 0, 0};
    if (int rc = ring_synthesis_real(h, r->F6, fou, mF, r->G9, h->nspat, 9 * nmem, src9, mod9, 9, 6, s)) return rc;
    k_swe_pointwise<<<dim3((h->nspat + 255) / 256, nmem), 256, 0, s>>>(r->G9, r->G4, h->mu, h->cosphi, nlat, h->nspat, kc);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = ring_analysis_real(h, r->G4, h->nspat, r->F4, fou, mF, 4 * nmem, s)) return rc;
    if (int rc = legendre_analysis_real(h, r->F4, fou, r->T4, nlm, L, 4 * nmem, s)) return rc;
    k_rk_mid<<<dim3((L + 1 + 63) / 64, L + 1, nmem), 64, 0, s>>>(r->T4, r->X2, L, nlm);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = legendre_synthesis_real(h, r->X2, nlm, L, r->F2, fou, 2 * nmem, s, 1)) return rc;
    k_fourier_h<<<dim3((unsigned)((fou + 255) / 256), nmem), 256, 0, s>>>(r->F2, r->Fh, h->cosphi, nlat, mF,
                                                                          kc.mode == 2 ? 2 : 1);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = legendre_analysis_real(h, r->Fh, fou, r->Th, nlm, L, nmem, s, 1)) return rc;
    k_rk_stage_out<<<dim3((L + 1 + 63) / 64, L + 1, nmem), 64, 0, s>>>(S, Kp, coef, r->dts, r->T4, r->Th, Ks, L, nlm, kc);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// one tendency evaluation of the vorticity-divergence form
static int swe_stage_vd(Handle* h, RKState* r, const sph_swe_params* p, const double2* S, const double2* Kp,
                        double coef, double2* Ks, int nmem, cudaStream_t s) {
    const int L = h->L, Lp = L + 1, nlm = h->nlm, nlat = h->nlat, mF = L + 1;
    const int nlmp = (Lp + 1) * (Lp + 2) / 2;
    const long long fou = (long long)mF * nlat;
    k_vd_prep<<<dim3((Lp + 1 + 63) / 64, Lp + 1, nmem), 64, 0, s>>>(S, Kp, coef, r->dts, r->X6, L, nlm, nlmp,
                                                                     p->radius);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = legendre_synthesis_real(h, r->X6, nlmp, Lp, r->F6, fou, 4 * nmem, s, 1)) return rc;
    if (int rc = ring_synthesis_real(h, r->F6, fou, mF, r->G4, h->nspat, 4 * nmem, nullptr, nullptr, 0, 0, s)) return rc;
    k_vd_pointwise<<<dim3((h->nspat + 255) / 256, nmem), 256, 0, s>>>(r->G4, r->G9, h->mu, h->cosphi, nlat, h->nspat,
                                                                      p->gravity, p->omega);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = ring_analysis_real(h, r->G9, h->nspat, r->F6, fou, mF, 5 * nmem, s)) return rc;
    if (int rc = legendre_analysis_real(h, r->F6, fou, r->X6, nlmp, Lp, 5 * nmem, s, 1)) return rc;
    k_vd_stage_out<<<dim3((L + 1 + 63) / 64, L + 1, nmem), 64, 0, s>>>(S, Kp, coef, r->dts, r->X6, Ks, L, nlm, nlmp,
                                                                       p->radius, p->viscosity);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

static int swe_any_stage(Handle* h, RKState* r, const sph_swe_params* p, const double2* S, const double2* Kp,
                         double coef, double2* Ks, int nmem, cudaStream_t s) {
    if (p->nonlinear == 2) return swe_stage_vd(h, r, p, S, Kp, coef, Ks, nmem, s);
    return swe_stage(h, r, p, S, Kp, coef, Ks, nmem, s);
}

static int swe_step(Handle* h, RKState* r, const sph_swe_params* p, double2* S, int nmem, cudaStream_t s) {
    const size_t st = (size_t)nmem * 3 * h->nlm;
    double2* K0 = r->K;
    double2* K1 = r->K + st;
    double2* K2 = r->K + 2 * st;
    double2* K3 = r->K + 3 * st;
    if (int rc = swe_any_stage(h, r, p, S, nullptr, 0.0, K0, nmem, s)) return rc;
    if (int rc = swe_any_stage(h, r, p, S, K0, 0.5, K1, nmem, s)) return rc;
    if (int rc = swe_any_stage(h, r, p, S, K1, 0.5, K2, nmem, s)) return rc;
    if (int rc = swe_any_stage(h, r, p, S, K2, 1.0, K3, nmem, s)) return rc;
    const size_t tot = st;
    k_rk_final<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(S, r->K, r->dts, nmem, h->nlm, r->flag);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// kernel launches in a captured graph
static int kernel_nodes(cudaGraph_t graph, int* out) {
    size_t nodes = 0;
    SPH_CUDA_TRY(cudaGraphGetNodes(graph, nullptr, &nodes));
    std::vector<cudaGraphNode_t> list(nodes);
    if (nodes) SPH_CUDA_TRY(cudaGraphGetNodes(graph, list.data(), &nodes));
    int k = 0;
    for (cudaGraphNode_t n : list) {
        cudaGraphNodeType t;
        SPH_CUDA_TRY(cudaGraphNodeGetType(n, &t));
        if (t == cudaGraphNodeTypeKernel) k++;
    }
    *out = k;
    return SPH_OK;
}

static bool same_params(const sph_swe_params& a, const sph_swe_params& b) {
    return std::memcmp(&a, &b, sizeof(a)) == 0;
}

static int rk_run(Handle* h, const sph_swe_params* p, const double* dts_h, double* state, int nmem, int nsteps,
                  cudaStream_t s) {
    if (!p || !state || nmem <= 0 || nsteps < 0) {
        set_error("sph_swe_rk4: bad arguments");
        return SPH_ERR_ARG;
    }
    if (nmem > 65535 / 9) {
        set_error("sph_swe_rk4: too many members for one launch");
        return SPH_ERR_ARG;
    }
    if (int rc = rk_alloc(h, nmem)) return rc;
    RKState* r = static_cast<RKState*>(h->rk);
    std::vector<double> d(nmem);
    for (int i = 0; i < nmem; i++) d[i] = dts_h ? dts_h[i] : p->dt;
    const bool rebuild = !r->exec || r->state != state || r->stream != s || !same_params(r->params, *p) ||
                         r->nmem != nmem || r->dts_h != d;
    if (rebuild) {
        if (r->exec) { cudaGraphExecDestroy(r->exec); r->exec = nullptr; }
        if (r->graph) { cudaGraphDestroy(r->graph); r->graph = nullptr; }
        SPH_CUDA_TRY(cudaMemcpyAsync(r->dts, d.data(), sizeof(double) * nmem, cudaMemcpyHostToDevice, s));
        SPH_CUDA_TRY(cudaStreamSynchronize(s));
        // the largest Legendre call of a step has 6 fields per member: workspace
        // of autotuned kernel variants is reserved now (a capture cannot allocate)
        if (int rc = tc_reserve(h, 6 * nmem)) return rc;
        // the legacy default stream cannot be captured: capture on a private stream
        cudaStream_t cap;
        SPH_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        SPH_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int rc = swe_step(h, r, p, reinterpret_cast<double2*>(state), nmem, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) { set_error(std::string("graph capture: ") + cudaGetErrorString(e)); return SPH_ERR_CUDA; }
        r->graph = g;
        if (int krc = kernel_nodes(g, &r->launches)) return krc;
        SPH_CUDA_TRY(cudaGraphInstantiate(&r->exec, g, 0));
        r->state = state;
        r->stream = s;
        r->params = *p;
        r->nmem = nmem;
        r->dts_h = d;
    }
    SPH_CUDA_TRY(cudaMemsetAsync(r->flag, 0, sizeof(int), s));
    for (int i = 0; i < nsteps; i++) SPH_CUDA_TRY(cudaGraphLaunch(r->exec, s));
    int flag = 0;
    SPH_CUDA_TRY(cudaMemcpyAsync(&flag, r->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPH_CUDA_TRY(cudaStreamSynchronize(s));
    if (flag) {
        set_error("sph_swe_rk4: instability detected (non-finite value in h)");
        return SPH_ERR_NAN;
    }
    return tc_check(h);
}

// ------------------------------------------------------------------ ensembles
// Members of several truncations advanced by one CUDA graph.  Group g is the
// batched RK4 step of its handle over nmem[g] members stored contiguously at
// states[g]; each group is captured on its own branch (fork and join events on
// private streams), so one replay advances every member by one step and the
// groups' kernels may overlap where a launch leaves SMs idle (the small
// truncations' launches are latency-bound).  Every group owns its stage
// buffers, so a handle's own sph_swe_rk4 graph is not disturbed.
struct EnsembleGroup {
    Handle* h = nullptr;
    RKState* r = nullptr;
    sph_swe_params p{};
    double* state = nullptr;
    int nmem = 0;
};

struct Ensemble {
    std::vector<EnsembleGroup> g;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
};

static void ensemble_release(Ensemble* e) {
    if (!e) return;
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    for (auto& g : e->g) rk_release(g.r);
    delete e;
}

// streams and events of one capture, released on every return path
struct CaptureStreams {
    cudaStream_t cap = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;  // ev[0]: fork; ev[1 + g]: join of group g
    ~CaptureStreams() {
        for (cudaStream_t x : side)
            if (x) cudaStreamDestroy(x);
        if (cap) cudaStreamDestroy(cap);
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);
    }
};

static int ensemble_capture(Ensemble* e) {
    const int ng = (int)e->g.size();
    CaptureStreams cs;
    cs.side.assign(ng, nullptr);
    cs.ev.assign(ng + 1, nullptr);
    SPH_CUDA_TRY(cudaStreamCreateWithFlags(&cs.cap, cudaStreamNonBlocking));
    for (int i = 0; i < ng; i++) SPH_CUDA_TRY(cudaStreamCreateWithFlags(&cs.side[i], cudaStreamNonBlocking));
    for (cudaEvent_t& x : cs.ev) SPH_CUDA_TRY(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    SPH_CUDA_TRY(cudaStreamBeginCapture(cs.cap, cudaStreamCaptureModeThreadLocal));
    int rc = SPH_OK;
    cudaError_t ce = cudaEventRecord(cs.ev[0], cs.cap);
    for (int i = 0; i < ng && rc == SPH_OK && ce == cudaSuccess; i++) {
        EnsembleGroup& g = e->g[i];
        ce = cudaStreamWaitEvent(cs.side[i], cs.ev[0], 0);
        if (ce != cudaSuccess) break;
        rc = swe_step(g.h, g.r, &g.p, reinterpret_cast<double2*>(g.state), g.nmem, cs.side[i]);
        if (rc != SPH_OK) break;
        ce = cudaEventRecord(cs.ev[1 + i], cs.side[i]);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cs.cap, cs.ev[1 + i], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(cs.cap, &graph);
    if (rc != SPH_OK || ce != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (rc != SPH_OK) return rc;
        set_error(std::string("ensemble graph capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        return SPH_ERR_CUDA;
    }
    e->graph = graph;
    if (int rc = kernel_nodes(graph, &e->launches)) return rc;
    SPH_CUDA_TRY(cudaGraphInstantiate(&e->exec, graph, 0));
    return SPH_OK;
}

static int ensemble_create(int ngroups, sph_handle* const* handles, const sph_swe_params* params,
                           double* const* states, const int* nmem, const double* const* dts, Ensemble** out) {
    if (!out || ngroups <= 0 || !handles || !params || !states || !nmem) {
        set_error("sph_ensemble_create: bad arguments");
        return SPH_ERR_ARG;
    }
    *out = nullptr;
    for (int i = 0; i < ngroups; i++) {
        if (!handles[i] || !states[i] || nmem[i] <= 0 || nmem[i] > 65535 / 9) {
            set_error("sph_ensemble_create: group " + std::to_string(i) +
                      ": needs a handle, a state and 1 .. 7281 members");
            return SPH_ERR_ARG;
        }
        for (int k = 0; k < i; k++)
            if (handles[k] == handles[i]) {
                // the groups run concurrently and a handle's workspace is not shared
                set_error("sph_ensemble_create: groups " + std::to_string(k) + " and " + std::to_string(i) +
                          " use the same handle");
                return SPH_ERR_ARG;
            }
    }
    Ensemble* e = new Ensemble();
    e->g.resize(ngroups);
    for (int i = 0; i < ngroups; i++) {
        EnsembleGroup& g = e->g[i];
        g.h = reinterpret_cast<Handle*>(handles[i]);
        g.p = params[i];
        g.state = states[i];
        g.nmem = nmem[i];
        g.r = new RKState();
        if (int rc = rk_buffers(g.h, g.r, g.nmem)) { ensemble_release(e); return rc; }
        if (int rc = tc_reserve(g.h, 6 * g.nmem)) { ensemble_release(e); return rc; }
        std::vector<double> d(g.nmem);
        for (int k = 0; k < g.nmem; k++) d[k] = (dts && dts[i]) ? dts[i][k] : g.p.dt;
        const cudaError_t ce = cudaMemcpy(g.r->dts, d.data(), sizeof(double) * g.nmem, cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) {
            set_error(std::string("sph_ensemble_create: ") + cudaGetErrorString(ce));
            ensemble_release(e);
            return SPH_ERR_CUDA;
        }
    }
    if (int rc = ensemble_capture(e)) { ensemble_release(e); return rc; }
    *out = e;
    return SPH_OK;
}

static int ensemble_run(Ensemble* e, int nsteps, cudaStream_t s) {
    if (!e || nsteps < 0) { set_error("sph_ensemble_step: bad arguments"); return SPH_ERR_ARG; }
    const int ng = (int)e->g.size();
    for (auto& g : e->g) SPH_CUDA_TRY(cudaMemsetAsync(g.r->flag, 0, sizeof(int), s));
    for (int i = 0; i < nsteps; i++) SPH_CUDA_TRY(cudaGraphLaunch(e->exec, s));
    std::vector<int> flags(ng, 0);
    for (int i = 0; i < ng; i++)
        SPH_CUDA_TRY(cudaMemcpyAsync(&flags[i], e->g[i].r->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPH_CUDA_TRY(cudaStreamSynchronize(s));
    std::string bad;
    for (int i = 0; i < ng; i++)
        if (flags[i]) bad += (bad.empty() ? "" : ", ") + std::to_string(i);
    if (!bad.empty()) {
        set_error("sph_ensemble_step: instability detected (non-finite value in h) in group(s) " + bad);
        return SPH_ERR_NAN;
    }
    for (auto& g : e->g)
        if (int rc = tc_check(g.h)) return rc;
    return SPH_OK;
}

}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

int sph_swe_tendency(sph_handle* hh, const sph_swe_params* p, const double* state, double* tend, void* stream) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !p || !state || !tend) { set_error("sph_swe_tendency: bad arguments"); return SPH_ERR_ARG; }
    if (int rc = rk_alloc(h, 1)) return rc;
    RKState* r = static_cast<RKState*>(h->rk);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    r->state = nullptr;  // dts[0] is overwritten: the cached step graph must be re-captured
    SPH_CUDA_TRY(cudaMemcpyAsync(r->dts, &p->dt, sizeof(double), cudaMemcpyHostToDevice, s));
    if (int rc = swe_any_stage(h, r, p, reinterpret_cast<const double2*>(state), nullptr, 0.0,
                               reinterpret_cast<double2*>(tend), 1, s))
        return rc;
    SPH_CUDA_TRY(cudaStreamSynchronize(s));
    return SPH_OK;
}

int sph_swe_rk4(sph_handle* hh, const sph_swe_params* p, double* state, int nsteps, void* stream) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) { set_error("sph_swe_rk4: NULL handle"); return SPH_ERR_ARG; }
    return rk_run(h, p, nullptr, state, 1, nsteps, reinterpret_cast<cudaStream_t>(stream));
}

int sph_swe_rk4_batched(sph_handle* hh, const sph_swe_params* p, const double* dts, double* state, int nmem,
                        int nsteps, void* stream) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) { set_error("sph_swe_rk4_batched: NULL handle"); return SPH_ERR_ARG; }
    return rk_run(h, p, dts, state, nmem, nsteps, reinterpret_cast<cudaStream_t>(stream));
}

int sph_ensemble_create(int ngroups, sph_handle* const* handles, const sph_swe_params* params, double* const* states,
                        const int* nmem, const double* const* dts, sph_ensemble** out) {
    Ensemble* e = nullptr;
    const int rc = ensemble_create(ngroups, handles, params, states, nmem, dts, &e);
    if (out) *out = reinterpret_cast<sph_ensemble*>(e);
    return rc;
}

int sph_ensemble_step(sph_ensemble* e, int nsteps, void* stream) {
    return ensemble_run(reinterpret_cast<Ensemble*>(e), nsteps, reinterpret_cast<cudaStream_t>(stream));
}

int sph_swe_rk4_launches(const sph_handle* hh) {
    const Handle* h = reinterpret_cast<const Handle*>(hh);
    const RKState* r = h ? static_cast<const RKState*>(h->rk) : nullptr;
    return r && r->exec ? r->launches : 0;
}

int sph_ensemble_launches(const sph_ensemble* e) {
    return e ? reinterpret_cast<const Ensemble*>(e)->launches : 0;
}

int sph_ensemble_destroy(sph_ensemble* e) {
    if (!e) return SPH_OK;
    cudaDeviceSynchronize();
    ensemble_release(reinterpret_cast<Ensemble*>(e));
    return SPH_OK;
}

}  // extern "C"
