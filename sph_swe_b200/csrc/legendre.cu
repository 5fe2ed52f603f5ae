// Legendre stage of the spherical-harmonic transforms in FP64 (the plain
// method): per zonal wavenumber m a dense contraction between the table
// P_l^m(mu_j) (northern rings only, equatorial symmetry) and the batch of
// fields, tiled as a small GEMM on the FP64 pipe.
//
//   synthesis  E_j = sum_{l-m even} Q_l P_l(mu_j),  O_j = sum_{l-m odd} Q_l P_l(mu_j)
//              F(mu_j) = E_j + O_j,  F(-mu_j) = E_j - O_j
//   analysis   Q_l = sum_{j<nh} w_j P_l(mu_j) (F(mu_j) +/- F(-mu_j))   (+ for l-m even)
//
// Real fields use m = 0..min(lmax, L) and the packed layout of degree lmax
// (lmax = L, or L+1 for the vector transforms); complex fields use
// m = -L..L, layout n*n+n+m and P_l^{-m} = (-1)^m P_l^m.
// Columns of the GEMM are (field, re/im) pairs.
#include "common.cuh"

#include <atomic>

namespace sphgpu {

namespace {
constexpr int TJ = 64;   // latitudes per CTA tile (synthesis)
constexpr int TLT = 64;  // degrees per CTA tile (analysis)
constexpr int TC = 32;   // real columns per tile (16 complex fields)
constexpr int TK = 16;   // contraction chunk
constexpr int NT = 256;  // threads
}  // namespace

struct SpecMap {
    int cplx;      // 0 real packed(lmax), 1 complex n*n+n+m
    int lmax;
    int L;
    long long ld;  // per-field stride (double2)
};

__device__ __forceinline__ long long spec_index(const SpecMap& s, int l, int m) {
    return s.cplx ? (long long)cidx(l, m) : (long long)pidx(s.lmax, l, m);
}

// grid: x = j tile, y = column tile, z = m slot (real: m, complex: m + L)
__global__ void __launch_bounds__(NT) k_legendre_synthesis(const double* __restrict__ plm, const long long* __restrict__ poff,
                                                           int nh, int nlat, const double2* __restrict__ spec, SpecMap sm,
                                                           double2* __restrict__ F, long long ldF, int batch) {
    __shared__ double As[TK][TJ];
    __shared__ double Bs[TK][TC + 1];
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int j0 = blockIdx.x * TJ;
    const int f0 = blockIdx.y * (TC / 2);
    const int tid = threadIdx.x;
    const int tx = tid & 15;   // field within tile
    const int ty = tid >> 4;   // 4 latitudes: ty*4 .. ty*4+3
    const double* P = plm + poff[am];

    double eR[4] = {0, 0, 0, 0}, eI[4] = {0, 0, 0, 0}, oR[4] = {0, 0, 0, 0}, oI[4] = {0, 0, 0, 0};

    for (int l0 = am; l0 <= lmax; l0 += TK) {
        // A tile: P rows l0..l0+TK-1, latitudes j0..j0+TJ-1
        for (int idx = tid; idx < TK * TJ; idx += NT) {
            const int kk = idx / TJ, jj = idx - kk * TJ;
            const int l = l0 + kk, j = j0 + jj;
            As[kk][jj] = (l <= lmax && j < nh) ? P[(long long)(l - am) * nh + j] * sg : 0.0;
        }
        // B tile: coefficients of 16 fields, degrees l0..l0+TK-1
        {
            const int kk = tid & 15, ff = tid >> 4;
            const int l = l0 + kk, f = f0 + ff;
            double2 q = make_double2(0, 0);
            if (l <= lmax && f < batch) q = spec[(long long)f * sm.ld + spec_index(sm, l, m)];
            Bs[kk][2 * ff] = q.x;
            Bs[kk][2 * ff + 1] = q.y;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; kk += 2) {
            const double br0 = Bs[kk][2 * tx], bi0 = Bs[kk][2 * tx + 1];
            const double br1 = Bs[kk + 1][2 * tx], bi1 = Bs[kk + 1][2 * tx + 1];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const double a0 = As[kk][ty * 4 + r], a1 = As[kk + 1][ty * 4 + r];
                eR[r] = fma(a0, br0, eR[r]);
                eI[r] = fma(a0, bi0, eI[r]);
                oR[r] = fma(a1, br1, oR[r]);
                oI[r] = fma(a1, bi1, oI[r]);
            }
        }
        __syncthreads();
    }
    const int f = f0 + tx;
    if (f >= batch) return;
    double2* out = F + (long long)f * ldF + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int j = j0 + ty * 4 + r;
        if (j >= nh) continue;
        out[j] = make_double2(eR[r] + oR[r], eI[r] + oI[r]);
        out[nlat - 1 - j] = make_double2(eR[r] - oR[r], eI[r] - oI[r]);
    }
}

// grid: x = degree tile, y = column tile, z = m slot
__global__ void __launch_bounds__(NT) k_legendre_analysis(const double* __restrict__ plm, const long long* __restrict__ poff,
                                                          int nh, int nlat, const double* __restrict__ w,
                                                          const double2* __restrict__ F, long long ldF,
                                                          double2* __restrict__ spec, SpecMap sm, int batch) {
    __shared__ double Ps[TK][TLT + 1];
    __shared__ double Ss[TK][TC + 1];
    __shared__ double Ds[TK][TC + 1];
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int lbase = am + blockIdx.x * TLT;
    if (lbase > lmax) return;
    const int f0 = blockIdx.y * (TC / 2);
    const int tid = threadIdx.x;
    const int tx = tid & 15;
    const int ty = tid >> 4;  // degrees lbase + ty + 16 r, r = 0..3 (same parity)
    const double* P = plm + poff[am];
    const double2* Fm = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
    const bool odd = ((lbase + ty - am) & 1) != 0;

    double aR[4] = {0, 0, 0, 0}, aI[4] = {0, 0, 0, 0};
    for (int j0 = 0; j0 < nh; j0 += TK) {
        for (int idx = tid; idx < TK * TLT; idx += NT) {
            const int ll = idx / TK, kk = idx - ll * TK;
            const int l = lbase + ll, j = j0 + kk;
            Ps[kk][ll] = (l <= lmax && j < nh) ? P[(long long)(l - am) * nh + j] * sg : 0.0;
        }
        {
            const int kk = tid & 15, ff = tid >> 4;
            const int j = j0 + kk, f = f0 + ff;
            double2 s = make_double2(0, 0), d = make_double2(0, 0);
            if (j < nh && f < batch) {
                const double2* Ff = Fm + (long long)f * ldF;
                const double2 n = Ff[j], so = Ff[nlat - 1 - j];
                const double wj = w[j];
                s = make_double2(wj * (n.x + so.x), wj * (n.y + so.y));
                d = make_double2(wj * (n.x - so.x), wj * (n.y - so.y));
            }
            Ss[kk][2 * ff] = s.x;
            Ss[kk][2 * ff + 1] = s.y;
            Ds[kk][2 * ff] = d.x;
            Ds[kk][2 * ff + 1] = d.y;
        }
        __syncthreads();
        const double(*G)[TC + 1] = odd ? Ds : Ss;
#pragma unroll
        for (int kk = 0; kk < TK; kk++) {
            const double gr = G[kk][2 * tx], gi = G[kk][2 * tx + 1];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const double p = Ps[kk][ty + 16 * r];
                aR[r] = fma(p, gr, aR[r]);
                aI[r] = fma(p, gi, aI[r]);
            }
        }
        __syncthreads();
    }
    const int f = f0 + tx;
    if (f >= batch) return;
    double2* out = spec + (long long)f * sm.ld;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int l = lbase + ty + 16 * r;
        if (l <= lmax) out[spec_index(sm, l, m)] = make_double2(aR[r], aI[r]);
    }
}

// Wide-tile variants for larger batches: CTA tile 64 rows x 64 real columns
// (32 fields), 128 threads with 8 rows x 4 columns each (64 / 32 FP64
// accumulators), contraction chunks of 16 double-buffered in shared memory
// with the next chunk's global loads issued before the current chunk's FMAs.
// Per k step a thread loads 4 + 2 (+2) double2 from shared memory for 32 FMAs.
namespace {
constexpr int WR = 64;        // rows per CTA (latitudes, or degrees in the analysis)
constexpr int WC = 64;        // real columns per CTA
constexpr int WK = 16;        // contraction chunk
constexpr int WNT = 128;      // threads
constexpr int WP = WR + 2;    // padded shared-memory row (16-byte aligned, spreads banks)
constexpr int WSMEM_ANA = 3 * 2 * WK * WP * (int)sizeof(double);  // analysis: P, sum, difference tiles
}  // namespace

__global__ void __launch_bounds__(WNT) k_legendre_synthesis_w(const double* __restrict__ plm,
                                                                   const long long* __restrict__ poff, int nh, int nlat,
                                                                   const double2* __restrict__ spec, SpecMap sm,
                                                                   double2* __restrict__ F, long long ldF, int batch) {
    __shared__ __align__(16) double As[2][WK][WP];
    __shared__ __align__(16) double Bs[2][WK][WP];
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int j0 = blockIdx.x * WR;
    const int f0 = blockIdx.y * (WC / 2);
    const int tid = threadIdx.x;
    const int tx = tid & 15;  // columns 4 tx .. 4 tx + 3 (fields f0 + 2 tx, f0 + 2 tx + 1)
    const int ty = tid >> 4;  // rows 8 ty .. 8 ty + 7
    const double* P = plm + poff[am];

    double ra[8];
    double2 rb[4];
    auto fetch = [&](int l0) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int idx = tid + WNT * i, kk = idx / WR, jj = idx % WR;
            const int l = l0 + kk, j = j0 + jj;
            ra[i] = (l <= lmax && j < nh) ? P[(long long)(l - am) * nh + j] * sg : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int idx = tid + WNT * i, kk = idx & 15, ff = idx >> 4;
            const int l = l0 + kk, f = f0 + ff;
            rb[i] = (l <= lmax && f < batch) ? spec[(long long)f * sm.ld + spec_index(sm, l, m)] : make_double2(0, 0);
        }
    };
    auto stash = [&](int b) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int idx = tid + WNT * i;
            As[b][idx / WR][idx % WR] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int idx = tid + WNT * i, kk = idx & 15, ff = idx >> 4;
            *reinterpret_cast<double2*>(&Bs[b][kk][2 * ff]) = rb[i];
        }
    };

    double E[8][4], O[8][4];
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) E[r][c] = O[r][c] = 0.0;

    fetch(am);
    stash(0);
    __syncthreads();
    int cur = 0;
    for (int l0 = am; l0 <= lmax; l0 += WK) {
        const bool more = l0 + WK <= lmax;
        if (more) fetch(l0 + WK);
#pragma unroll
        for (int kk = 0; kk < WK; kk++) {
            double a[8], b[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const double2 v = *reinterpret_cast<const double2*>(&As[cur][kk][8 * ty + 2 * q]);
                a[2 * q] = v.x;
                a[2 * q + 1] = v.y;
            }
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const double2 v = *reinterpret_cast<const double2*>(&Bs[cur][kk][4 * tx + 2 * q]);
                b[2 * q] = v.x;
                b[2 * q + 1] = v.y;
            }
            // degree l0 + kk has the parity of kk (l0 - am is a multiple of 16)
#pragma unroll
            for (int r = 0; r < 8; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    if (kk & 1) O[r][c] = fma(a[r], b[c], O[r][c]);
                    else E[r][c] = fma(a[r], b[c], E[r][c]);
                }
        }
        if (more) stash(cur ^ 1);
        __syncthreads();
        cur ^= 1;
    }
    double2* outm = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int f = f0 + 2 * tx + c;
        if (f >= batch) continue;
        double2* out = outm + (long long)f * ldF;
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int j = j0 + 8 * ty + r;
            if (j >= nh) continue;
            out[j] = make_double2(E[r][2 * c] + O[r][2 * c], E[r][2 * c + 1] + O[r][2 * c + 1]);
            out[nlat - 1 - j] = make_double2(E[r][2 * c] - O[r][2 * c], E[r][2 * c + 1] - O[r][2 * c + 1]);
        }
    }
}

__global__ void __launch_bounds__(WNT) k_legendre_analysis_w(const double* __restrict__ plm,
                                                                  const long long* __restrict__ poff, int nh, int nlat,
                                                                  const double* __restrict__ w,
                                                                  const double2* __restrict__ F, long long ldF,
                                                                  double2* __restrict__ spec, SpecMap sm, int batch) {
    extern __shared__ __align__(16) double wsm[];
    double(*Ps)[WK][WP] = reinterpret_cast<double(*)[WK][WP]>(wsm);
    double(*Ss)[WK][WP] = Ps + 2;
    double(*Ds)[WK][WP] = Ps + 4;
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int lbase = am + blockIdx.x * WR;
    if (lbase > lmax) return;
    const int f0 = blockIdx.y * (WC / 2);
    const int tid = threadIdx.x;
    const int tx = tid & 15;
    const int ty = tid >> 4;
    // the 64 degrees of the tile by parity (lbase - am is a multiple of 64):
    // degree lbase + 2 e + par is shared-memory row par * 32 + e; a thread
    // takes 8 degrees of one parity, e = e0 .. e0 + 7, and so needs only the
    // sum (even) or the difference (odd) columns
    const int par = ty >> 2, e0 = 8 * (ty & 3);
    const double* P = plm + poff[am];
    const double2* Fm = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;

    double rp[8];
    double2 rs[4], rd[4];
    auto fetch = [&](int j0) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int idx = tid + WNT * i, kk = idx & 15, ll = idx >> 4;
            const int l = lbase + ll, j = j0 + kk;
            rp[i] = (l <= lmax && j < nh) ? P[(long long)(l - am) * nh + j] * sg : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int idx = tid + WNT * i, kk = idx & 15, ff = idx >> 4;
            const int j = j0 + kk, f = f0 + ff;
            double2 sv = make_double2(0, 0), dv = make_double2(0, 0);
            if (j < nh && f < batch) {
                const double2* Ff = Fm + (long long)f * ldF;
                const double2 n = Ff[j], so = Ff[nlat - 1 - j];
                const double wj = w[j];
                sv = make_double2(wj * (n.x + so.x), wj * (n.y + so.y));
                dv = make_double2(wj * (n.x - so.x), wj * (n.y - so.y));
            }
            rs[i] = sv;
            rd[i] = dv;
        }
    };
    auto stash = [&](int b) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int idx = tid + WNT * i;
            const int ll = idx >> 4;
            Ps[b][idx & 15][(ll & 1) * 32 + (ll >> 1)] = rp[i];
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int idx = tid + WNT * i, kk = idx & 15, ff = idx >> 4;
            *reinterpret_cast<double2*>(&Ss[b][kk][2 * ff]) = rs[i];
            *reinterpret_cast<double2*>(&Ds[b][kk][2 * ff]) = rd[i];
        }
    };

    double acc[8][4];
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = 0.0;

    fetch(0);
    stash(0);
    __syncthreads();
    int cur = 0;
    for (int j0 = 0; j0 < nh; j0 += WK) {
        const bool more = j0 + WK < nh;
        if (more) fetch(j0 + WK);
        const double(*G)[WK][WP] = par ? Ds : Ss;
#pragma unroll
        for (int kk = 0; kk < WK; kk++) {
            double p[8], g[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const double2 v = *reinterpret_cast<const double2*>(&Ps[cur][kk][par * 32 + e0 + 2 * q]);
                p[2 * q] = v.x;
                p[2 * q + 1] = v.y;
            }
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const double2 u = *reinterpret_cast<const double2*>(&G[cur][kk][4 * tx + 2 * q]);
                g[2 * q] = u.x;
                g[2 * q + 1] = u.y;
            }
#pragma unroll
            for (int r = 0; r < 8; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fma(p[r], g[c], acc[r][c]);
        }
        if (more) stash(cur ^ 1);
        __syncthreads();
        cur ^= 1;
    }
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int f = f0 + 2 * tx + c;
        if (f >= batch) continue;
        double2* out = spec + (long long)f * sm.ld;
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int l = lbase + 2 * (e0 + r) + par;
            if (l <= lmax) out[spec_index(sm, l, m)] = make_double2(acc[r][2 * c], acc[r][2 * c + 1]);
        }
    }
}

// Small-batch variants (batch <= NB <= 8).  With one to a few fields the
// tiled kernels above fill 1/16 .. 1/2 of their column tile and walk the
// degrees in short chunks, each a global-load round trip and two barriers
// long: bound by latency (54-70 us per launch at T255 for 1-8 fields, where
// the 50 MB table streams in ~8 us).  Here the table is streamed with 8 to
// 16 independent loads per thread in flight (the next 8 rows' loads go out
// before the current 8 rows' sums) and the fields' values come from shared
// memory, staged for the whole degree (latitude) range of the m at once where
// it fits in 48 KB:
//   synthesis: a CTA takes 32 latitudes of one m; warp q sums the degrees
//     l = |m| + q (mod 8), so that a thread's terms all have the parity of q;
//     the eight classes meet in shared memory, E = even q, O = odd q.
//   analysis: a CTA takes 32 degrees of one m, 8 lanes per degree, each lane
//     a strided eighth of the latitudes, against the weighted north + south
//     (even degrees) and north - south (odd) values of the fields; the 8
//     lanes of a degree are summed by shuffles at the end.
// Shared arrays are field-major with the degree / latitude innermost, so
// that the lanes of a warp read consecutive 16-byte words.
namespace {
constexpr int SNT = 256;              // threads
constexpr int SJ = 32;                // latitudes per CTA (synthesis)
constexpr int SQ = SNT / SJ;          // degree classes (synthesis)
constexpr int AL = 32;                // degrees per CTA (analysis)
constexpr int ALANES = 8;             // lanes per degree (analysis)
constexpr int NB_SMEM = 48 * 1024;    // shared-memory budget of both kernels
constexpr int NBATCH = 4;             // staging loads in flight per thread
#ifndef SPH_NB_MAX
#define SPH_NB_MAX 8
#endif
constexpr int NB_MAX = SPH_NB_MAX;    // largest batch given to the small-batch kernels
// degrees (synthesis) or latitudes (analysis) staged per chunk: the whole
// range where it fits, else the largest multiple of 64 that does
inline int nb_chunk(int n, int bytes_per) {
    const int cap = (NB_SMEM / bytes_per) / 64 * 64;
    const int want = (n + 63) / 64 * 64;
    return want < cap ? want : cap;
}
}  // namespace

template <int NB>
__global__ void __launch_bounds__(SNT) k_legendre_synthesis_nb(const double* __restrict__ plm,
                                                               const long long* __restrict__ poff, int nh, int nlat,
                                                               const double2* __restrict__ spec, SpecMap sm,
                                                               double2* __restrict__ F, long long ldF, int batch,
                                                               int cq) {
    extern __shared__ double2 sh[];  // Q[NB][cq] during the sums, then R[SQ][NB][SJ]
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int tid = threadIdx.x;
    const int jl = tid % SJ, q = tid / SJ;
    const int j = blockIdx.x * SJ + jl;
    const bool jv = j < nh;
    const double* P = plm + poff[am] + (jv ? j : 0);
    double2 acc[NB];
#pragma unroll
    for (int f = 0; f < NB; f++) acc[f] = make_double2(0, 0);
    for (int lc = am; lc <= lmax; lc += cq) {
        const int nk = min(cq, lmax + 1 - lc);
        // stage the chunk's spectra, NBATCH loads in flight per thread
        for (int base = tid; base < cq * NB; base += NBATCH * SNT) {
            double2 v[NBATCH];
#pragma unroll
            for (int u = 0; u < NBATCH; u++) {
                const int idx = base + u * SNT;
                const int f = idx / cq, kk = idx - f * cq;
                v[u] = (idx < cq * NB && kk < nk && f < batch) ? spec[(long long)f * sm.ld + spec_index(sm, lc + kk, m)]
                                                               : make_double2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < NBATCH; u++) {
                const int idx = base + u * SNT;
                if (idx < cq * NB) sh[idx] = make_double2(v[u].x * sg, v[u].y * sg);
            }
        }
        __syncthreads();
        // degrees kk = q + 8 i of the chunk; the table loads of the next 8 are
        // issued before the sums of the current 8
        const int ni = nk > q ? (nk - q + SQ - 1) / SQ : 0;
        auto ldp = [&](int i) -> double {
            return (jv && i < ni) ? __ldg(P + (long long)(lc + q + SQ * i - am) * nh) : 0.0;
        };
        double pc[8];
#pragma unroll
        for (int u = 0; u < 8; u++) pc[u] = ldp(u);
        for (int i0 = 0; i0 < ni; i0 += 8) {
            double pn[8];
#pragma unroll
            for (int u = 0; u < 8; u++) pn[u] = ldp(i0 + 8 + u);
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int i = i0 + u;
                if (i >= ni) break;
                const int kk = q + SQ * i;
#pragma unroll
                for (int f = 0; f < NB; f++) {
                    const double2 c = sh[f * cq + kk];
                    acc[f].x = fma(pc[u], c.x, acc[f].x);
                    acc[f].y = fma(pc[u], c.y, acc[f].y);
                }
            }
#pragma unroll
            for (int u = 0; u < 8; u++) pc[u] = pn[u];
        }
        __syncthreads();
    }
    double2* R = sh;  // [SQ][NB][SJ]
#pragma unroll
    for (int f = 0; f < NB; f++) R[(q * NB + f) * SJ + jl] = acc[f];
    __syncthreads();
    double2* out = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
    for (int idx = tid; idx < SJ * NB; idx += SNT) {
        const int jj = idx % SJ, f = idx / SJ;
        const int jo = blockIdx.x * SJ + jj;
        if (jo >= nh || f >= batch) continue;
        double er = 0, ei = 0, orr = 0, oi = 0;
#pragma unroll
        for (int c = 0; c < SQ; c += 2) {
            const double2 e = R[(c * NB + f) * SJ + jj], o = R[((c + 1) * NB + f) * SJ + jj];
            er += e.x;
            ei += e.y;
            orr += o.x;
            oi += o.y;
        }
        double2* o = out + (long long)f * ldF;
        o[jo] = make_double2(er + orr, ei + oi);
        o[nlat - 1 - jo] = make_double2(er - orr, ei - oi);
    }
}

template <int NB>
__global__ void __launch_bounds__(SNT) k_legendre_analysis_nb(const double* __restrict__ plm,
                                                              const long long* __restrict__ poff, int nh, int nlat,
                                                              const double* __restrict__ w,
                                                              const double2* __restrict__ F, long long ldF,
                                                              double2* __restrict__ spec, SpecMap sm, int batch,
                                                              int cj) {
    extern __shared__ double2 sh[];  // G[2][NB][cj]: weighted north + south, north - south
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int lbase = am + blockIdx.x * AL;
    if (lbase > lmax) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane / ALANES, t = lane % ALANES;
    const int l = lbase + warp * (32 / ALANES) + g;
    const bool lv = l <= lmax;
    const int par = (l - am) & 1;
    const double* Pl = plm + poff[am] + (long long)((lv ? l : am) - am) * nh;
    const double2* Fm = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
    double2 acc[NB];
#pragma unroll
    for (int f = 0; f < NB; f++) acc[f] = make_double2(0, 0);
    for (int jc = 0; jc < nh; jc += cj) {
        const int nj = min(cj, nh - jc);
        // stage the chunk's weighted sums and differences, NBATCH entries in flight per thread
        for (int base = tid; base < cj * NB; base += NBATCH * SNT) {
            double2 n[NBATCH], so[NBATCH];
            double wj[NBATCH];
#pragma unroll
            for (int u = 0; u < NBATCH; u++) {
                const int idx = base + u * SNT;
                const int f = idx / cj, jj = idx - f * cj;
                const bool v = idx < cj * NB && jj < nj && f < batch;
                const double2* Ff = Fm + (long long)(v ? f : 0) * ldF;
                const int j = jc + (v ? jj : 0);
                n[u] = v ? Ff[j] : make_double2(0, 0);
                so[u] = v ? Ff[nlat - 1 - j] : make_double2(0, 0);
                wj[u] = v ? w[j] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < NBATCH; u++) {
                const int idx = base + u * SNT;
                if (idx >= cj * NB) break;
                sh[idx] = make_double2(wj[u] * (n[u].x + so[u].x), wj[u] * (n[u].y + so[u].y));
                sh[NB * cj + idx] = make_double2(wj[u] * (n[u].x - so[u].x), wj[u] * (n[u].y - so[u].y));
            }
        }
        __syncthreads();
        // latitudes jj = t + 8 i of the chunk; the table loads of the next 8
        // are issued before the sums of the current 8
        const double2* G = sh + par * NB * cj;
        const int ni = nj > t ? (nj - t + ALANES - 1) / ALANES : 0;
        auto ldp = [&](int i) -> double { return (lv && i < ni) ? __ldg(Pl + jc + t + ALANES * i) : 0.0; };
        double pc[8];
#pragma unroll
        for (int u = 0; u < 8; u++) pc[u] = ldp(u);
        for (int i0 = 0; i0 < ni; i0 += 8) {
            double pn[8];
#pragma unroll
            for (int u = 0; u < 8; u++) pn[u] = ldp(i0 + 8 + u);
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int i = i0 + u;
                if (i >= ni) break;
                const int jj = t + ALANES * i;
#pragma unroll
                for (int f = 0; f < NB; f++) {
                    const double2 c = G[f * cj + jj];
                    acc[f].x = fma(pc[u], c.x, acc[f].x);
                    acc[f].y = fma(pc[u], c.y, acc[f].y);
                }
            }
#pragma unroll
            for (int u = 0; u < 8; u++) pc[u] = pn[u];
        }
        __syncthreads();
    }
#pragma unroll
    for (int f = 0; f < NB; f++) {
#pragma unroll
        for (int o = ALANES / 2; o > 0; o >>= 1) {
            acc[f].x += __shfl_xor_sync(0xffffffffu, acc[f].x, o);
            acc[f].y += __shfl_xor_sync(0xffffffffu, acc[f].y, o);
        }
    }
    if (!lv) return;
    // lane t of the degree writes field t
#pragma unroll
    for (int f = 0; f < NB; f++)
        if (f == t && f < batch)
            spec[(long long)f * sm.ld + spec_index(sm, l, m)] = make_double2(acc[f].x * sg, acc[f].y * sg);
}

// FP64 tensor-core variants (mma.sync m8n8k4 f64, the FP64 MMA of sm_100;
// tcgen05 has no FP64 kind).  One instruction is an 8 x 8 x 4 product, 256
// FMAs from one table value and one field value per lane, where the FMA
// kernels above need a shared-memory load per one or two FMAs.  Per m the
// columns (field, re/im) are cut in blocks of CN = 8 RN (4 RN fields); a
// warp owns 16 rows of one l - m parity and all CN columns (2 x RN
// accumulator fragments of 2 doubles per lane).
//   analysis: A = P (8 degrees x 4 latitudes, straight from the table, rows
//     two degrees apart), B = the weighted north + south (even degrees) or
//     north - south (odd) values of the column block, staged column-major in
//     shared memory; a CTA of 8 warps takes 128 degrees (4 warps per parity).
//   synthesis: A = P^T (8 latitudes x 4 degrees of one parity), B = the
//     spectra of the column block staged per parity column-major; a CTA of 8
//     warps takes 64 latitudes, even warps summing the even degrees and odd
//     warps the odd ones, which meet in shared memory for north E + O, south E - O.
// Shared rows are padded to 4 (mod 16) doubles, so that the 32 lanes of a B
// fragment load (8 columns x 4 consecutive entries) take two wavefronts.
// Fragment layout of m8n8k4 f64 (lane = 4 g + t): A row g col t, B row t col
// g, C row g cols 2 t, 2 t + 1.
namespace {
constexpr int MNT = 256;                  // threads (8 warps)
#ifndef SPH_MSMEM
#define SPH_MSMEM 100352
#endif
constexpr int MSMEM = SPH_MSMEM;          // dynamic shared-memory budget per CTA (2 CTAs per SM)
constexpr int MSTAGE = 8;                 // staging loads in flight per thread (synthesis)
constexpr int MSTAGE_A = 4;               // staging entries in flight per thread (analysis: 3 loads each)
constexpr int MCHUNK = 192;               // most entries staged per column and parity
// entries staged per column and parity: the whole range where it fits (up to
// MCHUNK), else the largest multiple of 16 that does; the row stride is that + 4
inline int mma_chunk(int n, int cn) {
    const int cap = std::min(MCHUNK, ((MSMEM / (2 * cn * (int)sizeof(double)) - 4) / 16) * 16);
    const int want = (n + 15) / 16 * 16;
    return want < cap ? want : cap;
}
}  // namespace

#ifdef SPH_MMA_MINB
#define MMA_LB __launch_bounds__(MNT, SPH_MMA_MINB)
#else
#define MMA_LB __launch_bounds__(MNT)
#endif

__device__ __forceinline__ void dmma8844(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <int RN>
__global__ void MMA_LB k_legendre_analysis_mma(const double* __restrict__ plm,
                                                               const long long* __restrict__ poff, int nh, int nlat,
                                                               const double* __restrict__ w,
                                                               const double2* __restrict__ F, long long ldF,
                                                               double2* __restrict__ spec, SpecMap sm, int batch,
                                                               int cj) {
    constexpr int CN = 8 * RN, NFB = CN / 2;
    extern __shared__ double msh[];  // G[parity][CN][cj + 4]
    const int S = cj + 4;
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int lbase = am + blockIdx.x * (MNT / 2);
    if (lbase > lmax) return;
    const int f0 = blockIdx.y * NFB;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int p = warp & 1, hw = warp >> 1;
    const bool busy = lbase + p + 2 * 16 * hw <= lmax;  // some row of this warp is a degree
    // A rows of this lane: degrees lbase + p + 2 (16 hw + 8 rm + g); rows past
    // lmax read row |m| (their sums are not stored)
    const double* prow[2];
#pragma unroll
    for (int rm = 0; rm < 2; rm++) {
        const int l = lbase + p + 2 * (16 * hw + 8 * rm + g);
        prow[rm] = plm + poff[am] + (long long)((l <= lmax ? l : am) - am) * nh + t;
    }
    const double2* Fm = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
    double acc[2][RN][2];
#pragma unroll
    for (int rm = 0; rm < 2; rm++)
#pragma unroll
        for (int nb = 0; nb < RN; nb++) acc[rm][nb][0] = acc[rm][nb][1] = 0.0;

    for (int jc = 0; jc < nh; jc += cj) {
        const int nj = min(cj, nh - jc);
        // stage the column block's weighted sums / differences, latitude-minor:
        // segment `row` = (field, 32 latitudes), warp w takes rows w, w + 8, ...
        const int nseg = (cj + 31) / 32;
#pragma unroll 4
        for (int row = warp; row < NFB * nseg; row += MNT / 32) {
            const int fl = row / nseg, jj = (row - fl * nseg) * 32 + lane;
            if (jj >= cj) continue;
            const bool v = f0 + fl < batch && jj < nj;
            const double2* Ff = Fm + (long long)(v ? f0 + fl : 0) * ldF;
            const int j = jc + (v ? jj : 0);
            const double2 n = v ? Ff[j] : make_double2(0, 0);
            const double2 so = v ? Ff[nlat - 1 - j] : make_double2(0, 0);
            const double wj = v ? w[j] : 0.0;
            double* s0 = msh + (2 * fl) * S + jj;          // parity 0, column re
            double* s1 = msh + (CN + 2 * fl) * S + jj;     // parity 1, column re
            s0[0] = wj * (n.x + so.x);
            s0[S] = wj * (n.y + so.y);
            s1[0] = wj * (n.x - so.x);
            s1[S] = wj * (n.y - so.y);
        }
        __syncthreads();
        const double* G = msh + (p * CN + g) * S + t;  // column 8 nb + g, latitude j0 + t
        // latitudes past nh - 1 read latitude nh - 1 (their staged values are zero)
        const int jlast = nh - 1 - jc - t;
        double a[4][2];
        auto lda = [&](int j0) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int j = min(j0 + 4 * k, jlast);
#pragma unroll
                for (int rm = 0; rm < 2; rm++) a[k][rm] = __ldg(prow[rm] + jc + j);
            }
        };
        if (busy) lda(0);
        for (int j0 = 0; busy && j0 < nj; j0 += 16) {
            double an[4][2];
#pragma unroll
            for (int k = 0; k < 4; k++)
#pragma unroll
                for (int rm = 0; rm < 2; rm++) an[k][rm] = a[k][rm];
            if (j0 + 16 < nj) lda(j0 + 16);  // next step's table values, ahead of this step's MMAs
#pragma unroll
            for (int k = 0; k < 4; k++) {
                double b[RN];
#pragma unroll
                for (int nb = 0; nb < RN; nb++) b[nb] = G[nb * 8 * S + j0 + 4 * k];
#pragma unroll
                for (int rm = 0; rm < 2; rm++)
#pragma unroll
                    for (int nb = 0; nb < RN; nb++) dmma8844(acc[rm][nb][0], acc[rm][nb][1], an[k][rm], b[nb]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int rm = 0; rm < 2; rm++) {
        const int l = lbase + p + 2 * (16 * hw + 8 * rm + g);
        if (l > lmax) continue;
#pragma unroll
        for (int nb = 0; nb < RN; nb++) {
            const int f = f0 + 4 * nb + t;
            if (f < batch)
                spec[(long long)f * sm.ld + spec_index(sm, l, m)] =
                    make_double2(acc[rm][nb][0] * sg, acc[rm][nb][1] * sg);
        }
    }
}

template <int RN>
__global__ void MMA_LB k_legendre_synthesis_mma(const double* __restrict__ plm,
                                                                const long long* __restrict__ poff, int nh, int nlat,
                                                                const double2* __restrict__ spec, SpecMap sm,
                                                                double2* __restrict__ F, long long ldF, int batch,
                                                                int kc) {
    constexpr int CN = 8 * RN, NFB = CN / 2;
    extern __shared__ double msh[];  // Q[parity][CN][kc + 4] (entry i: degree |m| + parity + 2 (i0 + i))
    const int S = kc + 4;
    const int m = sm.cplx ? (int)blockIdx.z - sm.L : (int)blockIdx.z;
    const int am = m < 0 ? -m : m;
    const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
    const int lmax = sm.lmax;
    const int jbase = blockIdx.x * (MNT / 4);
    const int f0 = blockIdx.y * NFB;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int p = warp & 1, hw = warp >> 1;
    const bool busy = jbase + 16 * hw < nh;  // some row of this warp is a latitude
    // A rows of this lane: latitudes jbase + 16 hw + 8 rm + g; rows past nh - 1
    // read latitude nh - 1 (their sums are not stored)
    const int j0r = jbase + 16 * hw + g;
    const double* P = plm + poff[am] + min(j0r, nh - 1);
    const int d1 = min(j0r + 8, nh - 1) - min(j0r, nh - 1);  // second row, relative
    const int npair = (lmax + 2 - am) / 2;  // degree pairs (even + odd) from |m|
    const int last = lmax - am;             // last table row of this m
    double acc[2][RN][2];
#pragma unroll
    for (int rm = 0; rm < 2; rm++)
#pragma unroll
        for (int nb = 0; nb < RN; nb++) acc[rm][nb][0] = acc[rm][nb][1] = 0.0;

    for (int ic = 0; ic < npair; ic += kc) {
        const int ni = min(kc, npair - ic);
        // stage the spectra of the chunk, both parities, column-major: entry r =
        // 2 i + parity is degree l0 + r
        const int l0 = am + 2 * ic;
        const long long b0 = sm.cplx ? 0 : (long long)pidx(lmax, l0, m);  // packed index of l0 (real)
        for (int r = tid; r < 2 * kc; r += MNT) {
            const int l = l0 + r;
            const bool vr = (r >> 1) < ni && l <= lmax;
            const long long si = sm.cplx ? (long long)cidx(vr ? l : am, m) : b0 + (vr ? r : 0);
            double* q = msh + ((r & 1) * CN) * S + (r >> 1);
#pragma unroll 8
            for (int fl = 0; fl < NFB; fl++) {
                const bool v = vr && f0 + fl < batch;
                const double2 x = v ? spec[(long long)(f0 + fl) * sm.ld + si] : make_double2(0, 0);
                q[(2 * fl) * S] = x.x * sg;
                q[(2 * fl + 1) * S] = x.y * sg;
            }
        }
        __syncthreads();
        const double* Q = msh + (p * CN + g) * S + t;  // column 8 nb + g, entry i0 + t
        // table row of entry i: p + 2 (ic + i); rows past lmax read row lmax - |m|
        // (their staged spectra are zero)
        const int r0 = p + 2 * (ic + t);
        double a[4][2];
        auto lda = [&](int i0) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int r = min(r0 + 2 * (i0 + 4 * k), last);
                const double* q = P + (long long)r * nh;
                a[k][0] = __ldg(q);
                a[k][1] = __ldg(q + d1);
            }
        };
        if (busy) lda(0);
        for (int i0 = 0; busy && i0 < ni; i0 += 16) {
            double an[4][2];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                an[k][0] = a[k][0];
                an[k][1] = a[k][1];
            }
            if (i0 + 16 < ni) lda(i0 + 16);  // next step's table values, ahead of this step's MMAs
#pragma unroll
            for (int k = 0; k < 4; k++) {
                double b[RN];
#pragma unroll
                for (int nb = 0; nb < RN; nb++) b[nb] = Q[nb * 8 * S + i0 + 4 * k];
#pragma unroll
                for (int rm = 0; rm < 2; rm++)
#pragma unroll
                    for (int nb = 0; nb < RN; nb++) dmma8844(acc[rm][nb][0], acc[rm][nb][1], an[k][rm], b[nb]);
            }
        }
        __syncthreads();
    }
    // odd sums to shared memory; the even warps combine and store
    double* X = msh + (size_t)hw * (2 * RN * 2 * 32);
    if (p == 1) {
#pragma unroll
        for (int rm = 0; rm < 2; rm++)
#pragma unroll
            for (int nb = 0; nb < RN; nb++) {
                X[((rm * RN + nb) * 2 + 0) * 32 + lane] = acc[rm][nb][0];
                X[((rm * RN + nb) * 2 + 1) * 32 + lane] = acc[rm][nb][1];
            }
    }
    __syncthreads();
    if (p == 1) return;
    double2* outm = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
#pragma unroll
    for (int rm = 0; rm < 2; rm++) {
        const int j = j0r + 8 * rm;
        if (j >= nh) continue;
#pragma unroll
        for (int nb = 0; nb < RN; nb++) {
            const int f = f0 + 4 * nb + t;
            if (f >= batch) continue;
            const double er = acc[rm][nb][0], ei = acc[rm][nb][1];
            const double orr = X[((rm * RN + nb) * 2 + 0) * 32 + lane], oi = X[((rm * RN + nb) * 2 + 1) * 32 + lane];
            double2* out = outm + (long long)f * ldF;
            out[j] = make_double2(er + orr, ei + oi);
            out[nlat - 1 - j] = make_double2(er - orr, ei - oi);
        }
    }
}

// zero the m = L+1 column of a degree-(L+1) packed spectrum (no wavenumber L+1 exists)
__global__ void k_zero_top(double2* spec, long long ld, int lmax, int batch) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < batch) spec[(long long)f * ld + pidx(lmax, lmax, lmax)] = make_double2(0, 0);
}

// The orders m = 0 and 1 alone, FP64 (blockIdx.z = m): a CTA of 8 warps takes
// 32 consecutive northern latitudes (one per lane: coalesced table reads) of
// one field, each warp an eighth of the degrees; the partial even / odd sums
// E = sum over l - m even, O = over l - m odd of P_l^m(mu_j) X_lm meet in shared
// memory; north E + O, south E - O.  A few microseconds for any batch, where
// the general kernel given two orders runs a handful of long CTAs.
__global__ void __launch_bounds__(256) k_legendre_synthesis_m01(const double* __restrict__ plm,
                                                                const long long* __restrict__ poff, int nh, int nlat,
                                                                const double2* __restrict__ spec, long long ld_spec,
                                                                int lmax, double2* __restrict__ F, long long ldF) {
    __shared__ double2 part[8][2][32];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int j = blockIdx.x * 32 + lane;
    const int f = blockIdx.y, m = blockIdx.z;
    const double* P = plm + poff[m];                                      // rows l - m
    const double2* x = spec + (long long)f * ld_spec + pidx(lmax, m, m);  // degrees m..lmax
    const int nk = lmax - m + 1;
    const int per = ((nk + 15) / 16) * 2;  // degrees per warp, even
    const int k0 = wp * per, k1 = min(nk, k0 + per);
    double2 e = make_double2(0, 0), o = make_double2(0, 0);
    if (j < nh) {
#pragma unroll 4
        for (int k = k0; k < k1; k += 2) {
            const double p0 = P[(long long)k * nh + j];
            const double2 x0 = __ldg(&x[k]);
            e.x = fma(p0, x0.x, e.x);
            e.y = fma(p0, x0.y, e.y);
            if (k + 1 < k1) {
                const double p1 = P[(long long)(k + 1) * nh + j];
                const double2 x1 = __ldg(&x[k + 1]);
                o.x = fma(p1, x1.x, o.x);
                o.y = fma(p1, x1.y, o.y);
            }
        }
    }
    part[wp][0][lane] = e;
    part[wp][1][lane] = o;
    __syncthreads();
    if (wp == 0 && j < nh) {
        e = o = make_double2(0, 0);
#pragma unroll
        for (int w = 0; w < 8; w++) {
            e.x += part[w][0][lane].x;
            e.y += part[w][0][lane].y;
            o.x += part[w][1][lane].x;
            o.y += part[w][1][lane].y;
        }
        double2* out = F + (long long)f * ldF + (long long)m * nlat;
        out[j] = make_double2(e.x + o.x, e.y + o.y);
        out[nlat - 1 - j] = make_double2(e.x - o.x, e.y - o.y);
    }
}

// The orders m = 0 and 1 of an analysis alone, FP64: one warp per (degree l,
// order m, field), lanes over the northern latitudes, a_lm = sum_j w_j
// P_l^m(mu_j) (F(j) + (-1)^(l-m) F(nlat-1-j)), reduced by shuffles.
__global__ void __launch_bounds__(128) k_legendre_analysis_m01(const double* __restrict__ plm,
                                                               const long long* __restrict__ poff, int nh, int nlat,
                                                               const double* __restrict__ w,
                                                               const double2* __restrict__ F, long long ldF,
                                                               double2* __restrict__ spec, long long ld_spec, int lmax,
                                                               int batch) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int per = 2 * lmax + 1;  // (l, m) pairs: m = 0: l = 0..lmax, m = 1: l = 1..lmax
    if (warp >= (long long)per * batch) return;
    const int f = (int)(warp / per), q = (int)(warp % per);
    const int m = q <= lmax ? 0 : 1, l = m == 0 ? q : q - lmax;
    const double* P = plm + poff[m] + (long long)(l - m) * nh;
    const double2* src = F + (long long)f * ldF + (long long)m * nlat;
    const double sg = ((l - m) & 1) ? -1.0 : 1.0;
    double2 acc = make_double2(0, 0);
    for (int j = lane; j < nh; j += 32) {
        const double pw = P[j] * w[j];
        const double2 a = src[j], b = src[nlat - 1 - j];
        acc.x = fma(pw, fma(sg, b.x, a.x), acc.x);
        acc.y = fma(pw, fma(sg, b.y, a.y), acc.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane == 0) spec[(long long)f * ld_spec + pidx(lmax, l, m)] = acc;
}

#ifndef SPH_LEG_MMA
#define SPH_LEG_MMA 1
#endif

// column-block width of the tensor-core kernels for a batch: 4, 8 or 16 fields
static int mma_rn(int batch) { return batch <= 4 ? 1 : batch <= 8 ? 2 : 4; }

static int launch_synth(const Handle* h, const double2* spec, SpecMap sm, double2* F, long long ldF, int batch,
                        cudaStream_t s) {
    if (batch <= 0) return SPH_OK;
    const int nm = sm.cplx ? 2 * h->L + 1 : std::min(sm.lmax, h->L) + 1;
    if (SPH_LEG_MMA) {
        const int rn = mma_rn(batch), cn = 8 * rn;
        const int kc = mma_chunk((sm.lmax + 2) / 2, cn);
        // staged spectra, then the odd sums of the 4 warp pairs
        const size_t smem = (size_t)std::max(2 * cn * (kc + 4), 4 * 2 * rn * 2 * 32) * sizeof(double);
        const dim3 grid((h->nh + MNT / 4 - 1) / (MNT / 4), (2 * batch + cn - 1) / cn, nm);
#define SYN_MMA(RN) \
    k_legendre_synthesis_mma<RN><<<grid, MNT, smem, s>>>(h->plm, h->poff, h->nh, h->nlat, spec, sm, F, ldF, batch, kc)
        if (rn == 1) SYN_MMA(1);
        else if (rn == 2) SYN_MMA(2);
        else SYN_MMA(4);
#undef SYN_MMA
        SPH_CUDA_TRY(cudaGetLastError());
        return SPH_OK;
    }
    if (batch > 16) {
        dim3 grid((h->nh + WR - 1) / WR, (batch + WC / 2 - 1) / (WC / 2), nm);
        k_legendre_synthesis_w<<<grid, WNT, 0, s>>>(h->plm, h->poff, h->nh, h->nlat, spec, sm, F, ldF, batch);
        SPH_CUDA_TRY(cudaGetLastError());
        return SPH_OK;
    }
    if (batch <= NB_MAX) {
        const dim3 grid((h->nh + SJ - 1) / SJ, 1, nm);
        const int nb = batch == 1 ? 1 : batch == 2 ? 2 : batch <= 4 ? 4 : 8;
        const int cq = nb_chunk(sm.lmax + 1, nb * (int)sizeof(double2));
        const size_t smem = (size_t)std::max(cq, SQ * SJ) * nb * sizeof(double2);
#define SYN_NB(NB) \
    k_legendre_synthesis_nb<NB><<<grid, SNT, smem, s>>>(h->plm, h->poff, h->nh, h->nlat, spec, sm, F, ldF, batch, cq)
        if (nb == 1) SYN_NB(1);
        else if (nb == 2) SYN_NB(2);
        else if (nb == 4) SYN_NB(4);
        else SYN_NB(8);
#undef SYN_NB
        SPH_CUDA_TRY(cudaGetLastError());
        return SPH_OK;
    }
    dim3 grid((h->nh + TJ - 1) / TJ, (batch + TC / 2 - 1) / (TC / 2), nm);
    k_legendre_synthesis<<<grid, NT, 0, s>>>(h->plm, h->poff, h->nh, h->nlat, spec, sm, F, ldF, batch);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

static int launch_anal(const Handle* h, const double2* F, long long ldF, double2* spec, SpecMap sm, int batch,
                       cudaStream_t s, const double* wts = nullptr) {
    if (!wts) wts = h->w;
    if (batch <= 0) return SPH_OK;
    const int nm = sm.cplx ? 2 * h->L + 1 : std::min(sm.lmax, h->L) + 1;
    if (SPH_LEG_MMA) {
        const int rn = mma_rn(batch), cn = 8 * rn;
        const int cj = mma_chunk(h->nh, cn);
        const size_t smem = (size_t)2 * cn * (cj + 4) * sizeof(double);
        const dim3 grid((sm.lmax + 1 + MNT / 2 - 1) / (MNT / 2), (2 * batch + cn - 1) / cn, nm);
#define ANA_MMA(RN)                                                                                                  \
    k_legendre_analysis_mma<RN><<<grid, MNT, smem, s>>>(h->plm, h->poff, h->nh, h->nlat, wts, F, ldF, spec, sm, batch, \
                                                        cj)
        if (rn == 1) ANA_MMA(1);
        else if (rn == 2) ANA_MMA(2);
        else ANA_MMA(4);
#undef ANA_MMA
    } else if (batch > 16) {
        // the shared-memory opt-in is a per-device attribute: once per device
        static std::atomic<unsigned long long> attr_done{0};
        const unsigned long long bit = h->device >= 0 && h->device < 64 ? 1ull << h->device : 0ull;
        if (!bit || !(attr_done.load() & bit)) {
            SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_w, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              WSMEM_ANA));
            attr_done.fetch_or(bit);
        }
        dim3 grid((sm.lmax + 1 + WR - 1) / WR, (batch + WC / 2 - 1) / (WC / 2), nm);
        k_legendre_analysis_w<<<grid, WNT, WSMEM_ANA, s>>>(h->plm, h->poff, h->nh, h->nlat, wts, F, ldF, spec, sm,
                                                        batch);
    } else if (batch <= NB_MAX) {
        const dim3 grid((sm.lmax + 1 + AL - 1) / AL, 1, nm);
        const int nb = batch == 1 ? 1 : batch == 2 ? 2 : batch <= 4 ? 4 : 8;
        const int cj = nb_chunk(h->nh, 2 * nb * (int)sizeof(double2));
        const size_t smem = (size_t)2 * nb * cj * sizeof(double2);
#define ANA_NB(NB)                                                                                                   \
    k_legendre_analysis_nb<NB><<<grid, SNT, smem, s>>>(h->plm, h->poff, h->nh, h->nlat, wts, F, ldF, spec, sm, batch, \
                                                       cj)
        if (nb == 1) ANA_NB(1);
        else if (nb == 2) ANA_NB(2);
        else if (nb == 4) ANA_NB(4);
        else ANA_NB(8);
#undef ANA_NB
    } else {
        dim3 grid((sm.lmax + 1 + TLT - 1) / TLT, (batch + TC / 2 - 1) / (TC / 2), nm);
        k_legendre_analysis<<<grid, NT, 0, s>>>(h->plm, h->poff, h->nh, h->nlat, wts, F, ldF, spec, sm, batch);
    }
    SPH_CUDA_TRY(cudaGetLastError());
    if (!sm.cplx && sm.lmax > h->L) {
        k_zero_top<<<(batch + 127) / 128, 128, 0, s>>>(spec, sm.ld, sm.lmax, batch);
        SPH_CUDA_TRY(cudaGetLastError());
    }
    return SPH_OK;
}

// Query every FP64 Legendre kernel once.  Under lazy module loading (the
// CUDA default) a kernel's code is loaded onto the device on first use; the
// query loads it at handle creation instead, so that later calls (among them
// the no-allocation synthesis) load nothing.
int legendre_kernels_init() {
    cudaFuncAttributes fa;
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_synthesis));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_synthesis_w));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_analysis));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_analysis_w));
    // the wide analysis needs its shared-memory opt-in on this device before any
    // launch, also before launches inside a stream capture
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_w, cudaFuncAttributeMaxDynamicSharedMemorySize, WSMEM_ANA));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_synthesis_nb<1>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_synthesis_nb<2>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_synthesis_nb<4>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_synthesis_nb<8>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_analysis_nb<1>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_analysis_nb<2>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_analysis_nb<4>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_analysis_nb<8>));
    // the tensor-core kernels take up to MSMEM of dynamic shared memory
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_synthesis_mma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_synthesis_mma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_synthesis_mma<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_mma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_mma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_mma<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_zero_top));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_synthesis_m01));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_legendre_analysis_m01));
    return SPH_OK;
}

int legendre_synthesis_real(const Handle* h, const double2* spec, long long ld_spec, int lmax, double2* F,
                            long long ldF, int batch, cudaStream_t s, int exact_m0, int nobuf) {
    SpecMap sm{0, lmax, h->L, ld_spec};
    // mixed handles: the tensor-core kernels unless the autotuner found the FP64 kernel faster (variant bit 16)
    if ((h->flags & SPH_PREC_MIXED) && !(tune_get(h, TUNE_TC_SYNTHESIS, batch, 0) & 16)) {
        if (int rc = legendre_synthesis_tc(h, spec, ld_spec, lmax, F, ldF, batch, s, nobuf)) return rc;
        if (!exact_m0) return SPH_OK;
        if (batch > 65535) { set_error("legendre synthesis: too many fields for one launch"); return SPH_ERR_ARG; }
        k_legendre_synthesis_m01<<<dim3((h->nh + 31) / 32, batch, 2), 256, 0, s>>>(h->plm, h->poff, h->nh, h->nlat,
                                                                                   spec, ld_spec, lmax, F, ldF);
        SPH_CUDA_TRY(cudaGetLastError());
        return SPH_OK;
    }
    return launch_synth(h, spec, sm, F, ldF, batch, s);
}

int legendre_analysis_real(const Handle* h, const double2* F, long long ldF, double2* spec, long long ld_spec,
                           int lmax, int batch, cudaStream_t s, int wmode) {
    if ((h->flags & SPH_PREC_MIXED) && !(tune_get(h, TUNE_TC_ANALYSIS, batch, 0) & 16)) {
        if (int rc = legendre_analysis_tc(h, F, ldF, spec, ld_spec, lmax, batch, s, wmode)) return rc;
        if (wmode) {
            // integrands of velocity-derived fields: the orders m = 0, 1 in FP64
            const long long warps = (long long)(2 * lmax + 1) * batch;
            k_legendre_analysis_m01<<<(unsigned)((warps + 3) / 4), 128, 0, s>>>(h->plm, h->poff, h->nh, h->nlat, h->wc, F,
                                                                               ldF, spec, ld_spec, lmax, batch);
            SPH_CUDA_TRY(cudaGetLastError());
        }
        if (lmax > h->L) {
            k_zero_top<<<(batch + 127) / 128, 128, 0, s>>>(spec, ld_spec, lmax, batch);
            SPH_CUDA_TRY(cudaGetLastError());
        }
        return SPH_OK;
    }
    SpecMap sm{0, lmax, h->L, ld_spec};
    return launch_anal(h, F, ldF, spec, sm, batch, s, wmode ? h->wc : h->w);
}

int legendre_synthesis_cplx(const Handle* h, const double2* spec, long long ld_spec, double2* F, long long ldF,
                            int batch, cudaStream_t s) {
    SpecMap sm{1, h->L, h->L, ld_spec};
    return launch_synth(h, spec, sm, F, ldF, batch, s);
}

int legendre_analysis_cplx(const Handle* h, const double2* F, long long ldF, double2* spec, long long ld_spec,
                           int batch, cudaStream_t s) {
    SpecMap sm{1, h->L, h->L, ld_spec};
    return launch_anal(h, F, ldF, spec, sm, batch, s);
}

}  // namespace sphgpu
