// Legendre stage of the spherical-harmonic transforms in FP64 (the plain
// method): per zonal wavenumber m a dense contraction between the table
// P_l^m(mu_j) (northern rings only, equatorial symmetry) and the batch of
// fields, run on the FP64 tensor cores.
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

namespace sphgpu {

struct SpecMap {
    int cplx;      // 0 real packed(lmax), 1 complex n*n+n+m
    int lmax;
    int L;
    long long ld;  // per-field stride (double2)
};

__device__ __forceinline__ long long spec_index(const SpecMap& s, int l, int m) {
    return s.cplx ? (long long)cidx(l, m) : (long long)pidx(s.lmax, l, m);
}

// The kernels use mma.sync m8n8k4 f64, the FP64 MMA of sm_100 (tcgen05 has
// no FP64 kind; measured here 37 TFLOP/s against 34 for scalar FMA).  One
// instruction is an 8 x 8 x 4 product, 256 FMAs from one table value and one
// field value per lane, where register-tiled FMA kernels need a shared-memory
// load per one to four FMAs (those measured 158 / 206 us for the 64-field
// synthesis / analysis at T255, 33 / 48 us for 8 fields; these 116 / 117 and
// 19 / 21 us).  Per m the
// columns (field, re/im) are cut in blocks of CN = 8 RN (4 RN fields); a
// warp owns 16 rows of one l - m parity and all CN columns (2 x RN
// accumulator fragments of 2 doubles per lane).
//   analysis: A = P (8 degrees x 4 latitudes, rows two degrees apart), each
//     warp copying its 16 rows x 16 latitudes of a step into its own ring of
//     MRING slots in shared memory with cp.async, two steps ahead of its MMAs
//     (no registers held, no barrier between warps); B = the weighted north +
//     south (even degrees) or north - south (odd) values of the column block,
//     staged column-major in shared memory; a CTA of 8 warps takes 128
//     degrees (4 warps per parity).
//   synthesis: A = P^T (8 latitudes x 4 degrees of one parity), B = the
//     spectra of the column block staged per parity column-major; a CTA of 8
//     warps takes 64 latitudes, even warps summing the even degrees and odd
//     warps the odd ones, which meet in shared memory for north E + O, south E - O.
// Shared rows are padded to 4 (mod 16) doubles, so that the 32 lanes of an A
// or B fragment load (8 rows or columns x 4 consecutive entries) take two
// wavefronts.
// Fragment layout of m8n8k4 f64 (lane = 4 g + t): A row g col t, B row t col
// g, C row g cols 2 t, 2 t + 1.
namespace {
constexpr int MNT = 256;                  // threads (8 warps)
constexpr int MRING = 3;                  // ring slots of table tiles per warp (steps in flight)
constexpr int ASA = 20;                   // analysis tile row: 16 latitudes + 4 (two-wavefront fragment loads)
constexpr int RING_A = 8 * MRING * 16 * ASA;  // doubles of the analysis rings of a CTA
constexpr int MSMEM = 115712;             // dynamic shared memory per CTA at most (2 CTAs per SM)
constexpr int MCHUNK = 192;               // most entries staged per column and parity
// entries staged per column and parity: the whole range where it fits (up to
// MCHUNK) next to the rings of `ring` doubles, else the largest multiple of 16
// that does; the row stride is that + 4
inline int mma_chunk(int n, int cn, int ring) {
    const int bytes = MSMEM - ring * (int)sizeof(double);
    const int cap = std::min(MCHUNK, ((bytes / (2 * cn * (int)sizeof(double)) - 4) / 16) * 16);
    const int want = (n + 15) / 16 * 16;
    return want < cap ? want : cap;
}
}  // namespace

// asynchronous global -> shared copies of 8 or 16 bytes (cp.async, through L1)
__device__ __forceinline__ void acp(double* dst, const double* src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (bytes == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void acp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void acp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// steps of table values the synthesis keeps in flight per warp in registers
// (16 contraction terms each): two with 16-field column blocks (T255 x 64
// fields: 140 -> 117 us), one with the narrow blocks, where more registers
// cost more occupancy than the extra loads gain.  (A shared-memory ring of
// asynchronous copies, as in the analysis, measured slower here: its space
// leaves less for the staged spectra, which then take more chunks.)
constexpr int mma_depth_syn(int rn) { return rn == 4 ? 2 : 1; }


__device__ __forceinline__ void dmma8844(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <int RN>
__global__ void __launch_bounds__(MNT) k_legendre_analysis_mma(const double* __restrict__ plm,
                                               const long long* __restrict__ poff, int nh, int nlat,
                                               const double* __restrict__ w, const double2* __restrict__ F,
                                               long long ldF, double2* __restrict__ spec, SpecMap sm, int batch,
                                               int cj) {
    constexpr int CN = 8 * RN, NFB = CN / 2;
    extern __shared__ __align__(16) double msh[];  // G[parity][CN][cj + 4], then the warps' A rings
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
    // this warp's A rows: degrees lbase + p + 2 (16 hw + r), r = 8 rm + g; table
    // row index of r (rows past lmax read the last row: their sums are not stored)
    const double* P = plm + poff[am];
    const int row0 = lbase - am + p + 32 * hw, last = lmax - am;
    auto trow = [&](int r) -> const double* { return P + (long long)min(row0 + 2 * r, last) * nh; };
    double* ring = msh + 2 * CN * S + (size_t)warp * MRING * 16 * ASA;
    const bool v16 = (nh & 1) == 0;  // table rows 16-byte aligned: 16-byte copies
    const double2* Fm = F + (long long)(sm.cplx ? (m + sm.L) : m) * nlat;
    double acc[2][RN][2];
#pragma unroll
    for (int rm = 0; rm < 2; rm++)
#pragma unroll
        for (int nb = 0; nb < RN; nb++) acc[rm][nb][0] = acc[rm][nb][1] = 0.0;

    for (int jc = 0; jc < nh; jc += cj) {
        const int nj = min(cj, nh - jc);
        // copy the 16 rows x 16 latitudes of step j0 into ring slot st (latitudes
        // past nh - 1 read the row's first entry: their staged values are zero)
        auto issue = [&](int st, int j0) {
            double* dst = ring + st * 16 * ASA;
            if (v16) {
                const int c = (lane & 7) * 2, j = jc + j0 + c;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int r = (lane >> 3) + 4 * i;
                    const double* src = trow(r) + (j < nh ? j : 0);
                    acp(dst + r * ASA + c, src, 16);
                }
            } else {
                const int c = lane & 15, j = jc + j0 + c;
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int r = (lane >> 4) + 2 * i;
                    const double* src = trow(r) + (j < nh ? j : 0);
                    acp(dst + r * ASA + c, src, 8);
                }
            }
        };
        const int nst = (nj + 15) / 16;
        // the first ring slots go out before the fields are staged
        if (busy) {
#pragma unroll
            for (int q = 0; q < MRING - 1; q++) {
                if (q < nst) issue(q, 16 * q);
                acp_commit();
            }
        }
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
        for (int q = 0; busy && q < nst; q++) {
            // slot of step q + MRING - 1 was read at step q - 1 (the warp synced after it)
            if (q + MRING - 1 < nst) issue((q + MRING - 1) % MRING, 16 * (q + MRING - 1));
            acp_commit();
            acp_wait<MRING - 1>();
            __syncwarp();
            const double* A = ring + (q % MRING) * 16 * ASA + g * ASA + t;
            const int j0 = 16 * q;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                double a[2], b[RN];
#pragma unroll
                for (int rm = 0; rm < 2; rm++) a[rm] = A[8 * rm * ASA + 4 * k];
#pragma unroll
                for (int nb = 0; nb < RN; nb++) b[nb] = G[nb * 8 * S + j0 + 4 * k];
#pragma unroll
                for (int rm = 0; rm < 2; rm++)
#pragma unroll
                    for (int nb = 0; nb < RN; nb++) dmma8844(acc[rm][nb][0], acc[rm][nb][1], a[rm], b[nb]);
            }
            __syncwarp();
        }
        acp_wait<0>();
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
__global__ void __launch_bounds__(MNT) k_legendre_synthesis_mma(const double* __restrict__ plm,
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
        constexpr int D = mma_depth_syn(RN);  // register ring of D steps
        double a[D][4][2];
        auto lda = [&](int i0, double(&dst)[4][2]) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int r = min(r0 + 2 * (i0 + 4 * k), last);
                const double* q = P + (long long)r * nh;
                dst[k][0] = __ldg(q);
                dst[k][1] = __ldg(q + d1);
            }
        };
        if (busy) {
#pragma unroll
            for (int d = 0; d < D; d++)
                if (16 * d < ni) lda(16 * d, a[d]);
        }
        for (int i0 = 0; busy && i0 < ni; i0 += 16 * D) {
#pragma unroll
            for (int d = 0; d < D; d++) {
                const int is = i0 + 16 * d;
                if (is >= ni) break;
                double an[4][2];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    an[k][0] = a[d][k][0];
                    an[k][1] = a[d][k][1];
                }
                if (is + 16 * D < ni) lda(is + 16 * D, a[d]);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    double b[RN];
#pragma unroll
                    for (int nb = 0; nb < RN; nb++) b[nb] = Q[nb * 8 * S + is + 4 * k];
#pragma unroll
                    for (int rm = 0; rm < 2; rm++)
#pragma unroll
                        for (int nb = 0; nb < RN; nb++) dmma8844(acc[rm][nb][0], acc[rm][nb][1], an[k][rm], b[nb]);
                }
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

// column-block width of the tensor-core kernels for a batch: 4, 8 or 16 fields
static int mma_rn(int batch) { return batch <= 4 ? 1 : batch <= 8 ? 2 : 4; }

// morders > 0 (real layout): the orders m = 0 .. morders - 1 alone
static int launch_synth(const Handle* h, const double2* spec, SpecMap sm, double2* F, long long ldF, int batch,
                        cudaStream_t s, int morders = 0) {
    if (batch <= 0) return SPH_OK;
    const int nm = morders > 0 ? morders : sm.cplx ? 2 * h->L + 1 : std::min(sm.lmax, h->L) + 1;
    const int rn = mma_rn(batch), cn = 8 * rn;
    const int kc = mma_chunk((sm.lmax + 2) / 2, cn, 0);
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

static int launch_anal(const Handle* h, const double2* F, long long ldF, double2* spec, SpecMap sm, int batch,
                       cudaStream_t s, const double* wts = nullptr, int morders = 0) {
    if (!wts) wts = h->w;
    if (batch <= 0) return SPH_OK;
    const int nm = morders > 0 ? morders : sm.cplx ? 2 * h->L + 1 : std::min(sm.lmax, h->L) + 1;
    const int rn = mma_rn(batch), cn = 8 * rn;
    const int cj = mma_chunk(h->nh, cn, RING_A);
    const size_t smem = (size_t)(2 * cn * (cj + 4) + RING_A) * sizeof(double);
    const dim3 grid((sm.lmax + 1 + MNT / 2 - 1) / (MNT / 2), (2 * batch + cn - 1) / cn, nm);
#define ANA_MMA(RN)                                                                                                  \
    k_legendre_analysis_mma<RN><<<grid, MNT, smem, s>>>(h->plm, h->poff, h->nh, h->nlat, wts, F, ldF, spec, sm, batch, \
                                                        cj)
    if (rn == 1) ANA_MMA(1);
    else if (rn == 2) ANA_MMA(2);
    else ANA_MMA(4);
#undef ANA_MMA
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
// the no-allocation synthesis) load nothing.  The shared-memory opt-in of the
// tensor-core kernels is set here too, before any launch, also before
// launches inside a stream capture.
int legendre_kernels_init() {
    cudaFuncAttributes fa;
    // the tensor-core kernels take up to MSMEM of dynamic shared memory
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_synthesis_mma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_synthesis_mma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_synthesis_mma<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_mma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_mma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_legendre_analysis_mma<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, MSMEM));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_zero_top));
    return SPH_OK;
}

int legendre_synthesis_real(const Handle* h, const double2* spec, long long ld_spec, int lmax, double2* F,
                            long long ldF, int batch, cudaStream_t s, int exact_m0, int nobuf) {
    SpecMap sm{0, lmax, h->L, ld_spec};
    // mixed handles: the tensor-core kernels unless the autotuner found the FP64 kernel faster (variant bit 16)
    if ((h->flags & SPH_PREC_MIXED) && !(tune_get(h, TUNE_TC_SYNTHESIS, batch, 0) & 16)) {
        if (int rc = legendre_synthesis_tc(h, spec, ld_spec, lmax, F, ldF, batch, s, nobuf)) return rc;
        if (!exact_m0) return SPH_OK;
        // the orders m = 0, 1 again, in FP64 (the plain form's kernels), over the mixed result
        return launch_synth(h, spec, sm, F, ldF, batch, s, 2);
    }
    return launch_synth(h, spec, sm, F, ldF, batch, s);
}

int legendre_analysis_real(const Handle* h, const double2* F, long long ldF, double2* spec, long long ld_spec,
                           int lmax, int batch, cudaStream_t s, int wmode) {
    if ((h->flags & SPH_PREC_MIXED) && !(tune_get(h, TUNE_TC_ANALYSIS, batch, 0) & 16)) {
        if (int rc = legendre_analysis_tc(h, F, ldF, spec, ld_spec, lmax, batch, s, wmode)) return rc;
        if (wmode) {
            // integrands of velocity-derived fields: the orders m = 0, 1 again in
            // FP64 (the plain form's kernels), over the mixed result
            SpecMap sm{0, lmax, h->L, ld_spec};
            if (int rc = launch_anal(h, F, ldF, spec, sm, batch, s, h->wc, 2)) return rc;
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
