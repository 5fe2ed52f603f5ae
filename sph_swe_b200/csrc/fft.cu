// Longitude stage of the spherical-harmonic transforms (the FFTW part of
// SHTNS spat_to_SH / SH_to_spat, SPHData.hpp:201,221): one CTA per tile of
// consecutive latitude rings of one field.  The tile is read/written with
// latitude-contiguous (coalesced) accesses of the theta-contiguous grid,
// transformed in shared memory by a mixed-radix Stockham FFT (FP64), and only
// the zonal wavenumbers m <= L are kept (analysis) / fed (synthesis).
// Two real rings are packed into one complex FFT.  Ring lengths 3 * 2^k (the
// automatic grids) use the compile-time kernels of fft_fixed.cuh.
#include "common.cuh"

namespace sphgpu {

struct FFTDev {
    int n, nrad;
    int rad[16];
};

// output k of a synthesis reads Fourier field src[k], modified by mod[k]
// (0 plain, 1 times i*m); passed by value so graph capture needs no buffers
struct RingMap {
    int use;
    int period;      // outputs per member
    int src_stride;  // Fourier fields per member
    int src[16];
    int mod[16];
    const double* rowdiv;  // nullptr, or ring j's output times 1 / rowdiv[j] (e.g. cos phi)
};

}  // namespace sphgpu

#include "fft_fixed.cuh"

namespace sphgpu {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// twiddle exp(sign * 2 pi i t / n) from the table exp(-2 pi i t / n)
__device__ __forceinline__ double2 twid(const double2* __restrict__ tw, int t, int sign) {
    double2 w = __ldg(&tw[t]);
    return sign > 0 ? cconj(w) : w;
}

// in-register DFT of length R (R in 2,3,4,5,7), sign -1 forward / +1 backward
__device__ __forceinline__ void dft_small(double2* v, int R, int sign, const double2* __restrict__ tw, int n) {
    if (R == 2) {
        double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        double2 a = v[0], b = v[1], c = v[2], d = v[3];
        double2 s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = csub(b, d);
        // multiply s3 by (sign * i)
        double2 js3 = sign < 0 ? make_double2(s3.y, -s3.x) : make_double2(-s3.y, s3.x);
        v[0] = cadd(s0, s2);
        v[2] = csub(s0, s2);
        v[1] = cadd(s1, js3);
        v[3] = csub(s1, js3);
    } else if (R == 3) {
        const double c = -0.5;
        const double sn = sign * 0.86602540378443864676372317075294;  // sin(2 pi / 3)
        double2 a = v[0], b = v[1], d = v[2];
        double2 t1 = cadd(b, d);
        double2 t2 = csub(b, d);
        double2 m1 = make_double2(a.x + c * t1.x, a.y + c * t1.y);
        double2 m2 = make_double2(-sn * t2.y, sn * t2.x);
        v[0] = cadd(a, t1);
        v[1] = cadd(m1, m2);
        v[2] = csub(m1, m2);
    } else {
        double2 o[8];
        const int step = n / R;
        for (int s = 0; s < R; s++) {
            double2 acc = make_double2(0, 0);
            for (int r = 0; r < R; r++) acc = cadd(acc, cmul(v[r], twid(tw, (int)((long long)r * s * step % n), sign)));
            o[s] = acc;
        }
        for (int s = 0; s < R; s++) v[s] = o[s];
    }
}

// nf independent length-n sequences at buf[f*n + i]; Stockham passes ping-pong
// between buf and alt.  Returns the buffer holding the (natural order) result.
__device__ double2* fft_smem(double2* buf, double2* alt, int nf, const FFTDev& p, const double2* __restrict__ tw,
                             int sign) {
    const int n = p.n;
    double2* src = buf;
    double2* dst = alt;
    int Ls = 1;
    for (int q = 0; q < p.nrad; q++) {
        const int R = p.rad[q];
        const int nR = n / R;
        const int tstep = n / (Ls * R);
        const int total = nf * nR;
        for (int t = threadIdx.x; t < total; t += blockDim.x) {
            const int f = t / nR;
            const int j = t - f * nR;
            const int k = j % Ls;
            const double2* s = src + f * n;
            double2* d = dst + f * n;
            double2 v[8];
            v[0] = s[j];
            for (int r = 1; r < R; r++) v[r] = cmul(s[j + r * nR], twid(tw, r * k * tstep, sign));
            dft_small(v, R, sign, tw, n);
            const int base = (j - k) * R + k;
            for (int r = 0; r < R; r++) d[base + r * Ls] = v[r];
        }
        __syncthreads();
        double2* tmp = src;
        src = dst;
        dst = tmp;
        Ls *= R;
    }
    return src;
}

// ------------------------------------------------------------- real analysis
// grid tile (JT rings, pairs packed) -> F[b][m][j], m = 0..mF-1 (m > L zero),
// scaled by 2 pi / n (quadrature weight in longitude).
__global__ void k_ring_analysis_real(const double* __restrict__ spat, long long ld_spat, double2* __restrict__ F,
                                     long long ldF, int mF, int L, int nlat, FFTDev p, const double2* __restrict__ tw,
                                     int JT) {
    extern __shared__ double2 smem[];
    const int n = p.n;
    const int np = JT / 2;
    double2* buf = smem;
    double2* alt = smem + np * n;
    const int j0 = blockIdx.x * JT;
    const int b = blockIdx.y;
    const double* src = spat + (long long)b * ld_spat;
    for (int idx = threadIdx.x; idx < n * JT; idx += blockDim.x) {
        const int i = idx / JT, jj = idx - (idx / JT) * JT;
        const int j = j0 + jj;
        const double val = (j < nlat) ? src[(long long)i * nlat + j] : 0.0;
        double* slot = reinterpret_cast<double*>(&buf[(jj >> 1) * n + i]);
        slot[jj & 1] = val;
    }
    __syncthreads();
    const double2* res = fft_smem(buf, alt, np, p, tw, -1);
    const double scale = 2.0 * kPi / n;
    double2* out = F + (long long)b * ldF;
    for (int idx = threadIdx.x; idx < mF * np; idx += blockDim.x) {
        const int m = idx / np, q = idx - (idx / np) * np;
        const int j = j0 + 2 * q;
        if (j >= nlat) continue;
        double2 X = make_double2(0, 0), Y = make_double2(0, 0);
        if (m <= L) {
            const double2 a = res[q * n + m];
            const double2 c = cconj(res[q * n + (n - m) % n]);
            X = make_double2(0.5 * (a.x + c.x) * scale, 0.5 * (a.y + c.y) * scale);
            // -i (a - c) / 2
            Y = make_double2(0.5 * (a.y - c.y) * scale, -0.5 * (a.x - c.x) * scale);
        }
        out[(long long)m * nlat + j] = X;
        out[(long long)m * nlat + j + 1] = Y;
    }
}

// ------------------------------------------------------------- real synthesis
// F[src[k]][m][j] (optionally times i*m) -> grid k; Re of the m = 0 term.
__global__ void k_ring_synthesis_real(const double2* __restrict__ F, long long ldF, int mF, int L, double* __restrict__ spat,
                                      long long ld_spat, int nlat, FFTDev p, const double2* __restrict__ tw, int JT,
                                      RingMap map) {
    extern __shared__ double2 smem[];
    const int n = p.n;
    const int np = JT / 2;
    double2* buf = smem;
    double2* alt = smem + np * n;
    const int j0 = blockIdx.x * JT;
    const int k = blockIdx.y;
    int fs = k, mod = 0;
    if (map.use) {
        const int mem = k / map.period, r = k - mem * map.period;
        fs = mem * map.src_stride + map.src[r];
        mod = map.mod[r];
    }
    const double2* in = F + (long long)fs * ldF;
    for (int idx = threadIdx.x; idx < np * n; idx += blockDim.x) buf[idx] = make_double2(0, 0);
    __syncthreads();
    const int mm = min(min(mF - 1, L), (n - 1) / 2);
    for (int idx = threadIdx.x; idx < (mm + 1) * np; idx += blockDim.x) {
        const int m = idx / np, q = idx - (idx / np) * np;
        const int j = j0 + 2 * q;
        double2 X = make_double2(0, 0), Y = make_double2(0, 0);
        if (j < nlat) {
            X = in[(long long)m * nlat + j];
            Y = in[(long long)m * nlat + j + 1];
        }
        if (mod == 1) {  // d/dlambda: times i*m
            X = make_double2(-m * X.y, m * X.x);
            Y = make_double2(-m * Y.y, m * Y.x);
        }
        if (m == 0) {
            buf[q * n] = make_double2(X.x, Y.x);
        } else {
            buf[q * n + m] = make_double2(X.x - Y.y, X.y + Y.x);          // X + iY
            buf[q * n + n - m] = make_double2(X.x + Y.y, -X.y + Y.x);     // conj(X) + i conj(Y)
        }
    }
    __syncthreads();
    const double2* res = fft_smem(buf, alt, np, p, tw, +1);
    double* out = spat + (long long)k * ld_spat;
    for (int idx = threadIdx.x; idx < n * JT; idx += blockDim.x) {
        const int i = idx / JT, jj = idx - (idx / JT) * JT;
        const int j = j0 + jj;
        if (j >= nlat) continue;
        const double2 z = res[(jj >> 1) * n + i];
        const double v = (jj & 1) ? z.y : z.x;
        out[(long long)i * nlat + j] = map.rowdiv ? v * (1.0 / map.rowdiv[j]) : v;
    }
}

// ------------------------------------------------------------- complex
__global__ void k_ring_analysis_cplx(const double2* __restrict__ spat, long long ld_spat, double2* __restrict__ F,
                                     long long ldF, int L, int nlat, FFTDev p, const double2* __restrict__ tw, int JT) {
    extern __shared__ double2 smem[];
    const int n = p.n;
    double2* buf = smem;
    double2* alt = smem + JT * n;
    const int j0 = blockIdx.x * JT;
    const int b = blockIdx.y;
    const double2* src = spat + (long long)b * ld_spat;
    for (int idx = threadIdx.x; idx < n * JT; idx += blockDim.x) {
        const int i = idx / JT, jj = idx - (idx / JT) * JT;
        const int j = j0 + jj;
        buf[jj * n + i] = (j < nlat) ? src[(long long)i * nlat + j] : make_double2(0, 0);
    }
    __syncthreads();
    const double2* res = fft_smem(buf, alt, JT, p, tw, -1);
    const double scale = 2.0 * kPi / n;
    double2* out = F + (long long)b * ldF;
    const int nm = 2 * L + 1;
    for (int idx = threadIdx.x; idx < nm * JT; idx += blockDim.x) {
        const int mi = idx / JT, jj = idx - (idx / JT) * JT;
        const int j = j0 + jj;
        if (j >= nlat) continue;
        const int m = mi - L;
        const double2 z = res[jj * n + ((m % n) + n) % n];
        out[(long long)mi * nlat + j] = make_double2(z.x * scale, z.y * scale);
    }
}

__global__ void k_ring_synthesis_cplx(const double2* __restrict__ F, long long ldF, int L, double2* __restrict__ spat,
                                      long long ld_spat, int nlat, FFTDev p, const double2* __restrict__ tw, int JT) {
    extern __shared__ double2 smem[];
    const int n = p.n;
    double2* buf = smem;
    double2* alt = smem + JT * n;
    const int j0 = blockIdx.x * JT;
    const int b = blockIdx.y;
    const double2* in = F + (long long)b * ldF;
    for (int idx = threadIdx.x; idx < JT * n; idx += blockDim.x) buf[idx] = make_double2(0, 0);
    __syncthreads();
    const int nm = 2 * L + 1;
    // 2L+1 <= n, so each bin receives one wavenumber: plain stores
    for (int idx = threadIdx.x; idx < nm * JT; idx += blockDim.x) {
        const int mi = idx / JT, jj = idx - (idx / JT) * JT;
        const int j = j0 + jj;
        const int m = mi - L;
        if (j < nlat) buf[jj * n + ((m % n) + n) % n] = in[(long long)mi * nlat + j];
    }
    __syncthreads();
    const double2* res = fft_smem(buf, alt, JT, p, tw, +1);
    double2* out = spat + (long long)b * ld_spat;
    for (int idx = threadIdx.x; idx < n * JT; idx += blockDim.x) {
        const int i = idx / JT, jj = idx - (idx / JT) * JT;
        const int j = j0 + jj;
        if (j < nlat) out[(long long)i * nlat + j] = res[jj * n + i];
    }
}

// ------------------------------------------------------------- launchers
static FFTDev dev_plan(const FFTPlan& p) {
    FFTDev d;
    d.n = p.n;
    d.nrad = p.nrad;
    for (int i = 0; i < 16; i++) d.rad[i] = p.rad[i];
    return d;
}

// rings per CTA: as many as fit 96 KB of ping-pong buffers (even, <= 16)
// (real rings are packed in pairs, so a real tile has at least 2 rings)
static int ring_tile(int n, int complex_rings) {
    const size_t per_ring = complex_rings ? 2 * 16 * (size_t)n : 16 * (size_t)n;  // bytes incl. ping-pong
    const int jmin = complex_rings ? 1 : 2;
    int jt = 16;
    while (jt > jmin && (size_t)jt * per_ring > 96 * 1024) jt /= 2;
    return jt;
}

// sequences per CTA of the fixed-length kernels: variant 0 the default, 1 twice
// it, 2 half of it (at least 1)
template <int N, int V>
constexpr int fixed_p() {
    return V == 0 ? fftx::seqs<N>() : (V == 1 ? 2 * fftx::seqs<N>() : (fftx::seqs<N>() > 1 ? fftx::seqs<N>() / 2 : 1));
}

template <int N, int P>
static size_t fixed_smem() {
    return (size_t)P * N * sizeof(double2);
}

template <int N, int P>
static int fixed_attr_p() {
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_ring_analysis_real_n<N, P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fixed_smem<N, P>()));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_ring_synthesis_real_n<N, P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fixed_smem<N, P>()));
    return SPH_OK;
}

template <int N>
static int fixed_attr() {
    if (int rc = fixed_attr_p<N, fixed_p<N, 0>()>()) return rc;
    if (int rc = fixed_attr_p<N, fixed_p<N, 1>()>()) return rc;
    return fixed_attr_p<N, fixed_p<N, 2>()>();
}

// every (longitude, ring pair) of every field is an aligned 16-byte chunk
static int rows16(const Handle* h, const double* spat, long long ld_spat) {
    return (h->nlat % 2 == 0 && ld_spat % 2 == 0 && reinterpret_cast<uintptr_t>(spat) % 16 == 0) ? 1 : 0;
}

template <int N, int P>
static void launch_ra(const Handle* h, const double* spat, long long ld_spat, double2* F, long long ldF, int mF, int batch,
                      cudaStream_t s) {
    k_ring_analysis_real_n<N, P><<<dim3((h->nlat + 2 * P - 1) / (2 * P), batch), fftx::nt<N, P>(), fixed_smem<N, P>(), s>>>(
        spat, ld_spat, F, ldF, mF, h->L, h->nlat, h->fft.tw, rows16(h, spat, ld_spat));
}

template <int N, int P>
static void launch_rs(const Handle* h, const double2* F, long long ldF, int mF, double* spat, long long ld_spat, int batch,
                      const RingMap& map, cudaStream_t s) {
    k_ring_synthesis_real_n<N, P><<<dim3((h->nlat + 2 * P - 1) / (2 * P), batch), fftx::nt<N, P>(), fixed_smem<N, P>(), s>>>(
        F, ldF, mF, h->L, spat, ld_spat, h->nlat, h->fft.tw, map, rows16(h, spat, ld_spat));
}

int fft_kernels_init() {
    for (int rc : {fixed_attr<96>(), fixed_attr<192>(), fixed_attr<384>(), fixed_attr<768>(), fixed_attr<1536>(),
                   fixed_attr<3072>()})
        if (rc) return rc;
    const int bytes = 200 * 1024;
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_ring_analysis_real, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_ring_synthesis_real, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_ring_analysis_cplx, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_ring_synthesis_cplx, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return SPH_OK;
}

int ring_analysis_real(const Handle* h, const double* spat, long long ld_spat, double2* F, long long ldF, int mF,
                       int batch, cudaStream_t s) {
    if (batch <= 0) return SPH_OK;
    const int var = tune_get(h, TUNE_RING_ANALYSIS, batch, 0);
    switch (h->nphi) {
#define SPH_RA(NN)                                                                                                   \
    case NN:                                                                                                         \
        if (var == 1) launch_ra<NN, fixed_p<NN, 1>()>(h, spat, ld_spat, F, ldF, mF, batch, s);                       \
        else if (var == 2) launch_ra<NN, fixed_p<NN, 2>()>(h, spat, ld_spat, F, ldF, mF, batch, s);                  \
        else launch_ra<NN, fixed_p<NN, 0>()>(h, spat, ld_spat, F, ldF, mF, batch, s);                                \
        SPH_CUDA_TRY(cudaGetLastError());                                                                            \
        return SPH_OK;
        SPH_RA(96)
        SPH_RA(192)
        SPH_RA(384)
        SPH_RA(768)
        SPH_RA(1536)
        SPH_RA(3072)
#undef SPH_RA
        default:
            break;
    }
    const int JT = ring_tile(h->nphi, 0);
    const size_t sm = (size_t)JT * h->nphi * sizeof(double2);  // 2 buffers of JT/2 sequences
    dim3 grid((h->nlat + JT - 1) / JT, batch);
    k_ring_analysis_real<<<grid, 256, sm, s>>>(spat, ld_spat, F, ldF, mF, h->L, h->nlat, dev_plan(h->fft), h->fft.tw, JT);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

int ring_synthesis_real(const Handle* h, const double2* F, long long ldF, int mF, double* spat, long long ld_spat,
                        int batch, const int* src, const int* mod, int period, int src_stride, cudaStream_t s,
                        const double* rowdiv) {
    if (batch <= 0) return SPH_OK;
    const int JT = ring_tile(h->nphi, 0);
    const size_t sm = (size_t)JT * h->nphi * sizeof(double2);
    dim3 grid((h->nlat + JT - 1) / JT, batch);
    RingMap map{};
    map.rowdiv = rowdiv;
    if (src) {
        if (period <= 0 || period > 16 || batch % period) {
            set_error("ring synthesis: bad output map");
            return SPH_ERR_ARG;
        }
        map.use = 1;
        map.period = period;
        map.src_stride = src_stride;
        for (int k = 0; k < period; k++) {
            map.src[k] = src[k];
            map.mod[k] = mod ? mod[k] : 0;
        }
    }
    const int var = tune_get(h, TUNE_RING_SYNTHESIS, batch, 0);
    switch (h->nphi) {
#define SPH_RS(NN)                                                                                                   \
    case NN:                                                                                                         \
        if (var == 1) launch_rs<NN, fixed_p<NN, 1>()>(h, F, ldF, mF, spat, ld_spat, batch, map, s);                  \
        else if (var == 2) launch_rs<NN, fixed_p<NN, 2>()>(h, F, ldF, mF, spat, ld_spat, batch, map, s);             \
        else launch_rs<NN, fixed_p<NN, 0>()>(h, F, ldF, mF, spat, ld_spat, batch, map, s);                           \
        SPH_CUDA_TRY(cudaGetLastError());                                                                            \
        return SPH_OK;
        SPH_RS(96)
        SPH_RS(192)
        SPH_RS(384)
        SPH_RS(768)
        SPH_RS(1536)
        SPH_RS(3072)
#undef SPH_RS
        default:
            break;
    }
    k_ring_synthesis_real<<<grid, 256, sm, s>>>(F, ldF, mF, h->L, spat, ld_spat, h->nlat, dev_plan(h->fft), h->fft.tw, JT,
                                                map);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

int ring_analysis_cplx(const Handle* h, const double2* spat, long long ld_spat, double2* F, long long ldF, int batch,
                       cudaStream_t s) {
    if (batch <= 0) return SPH_OK;
    const int JT = ring_tile(h->nphi, 1);
    const size_t sm = (size_t)2 * JT * h->nphi * sizeof(double2);
    dim3 grid((h->nlat + JT - 1) / JT, batch);
    k_ring_analysis_cplx<<<grid, 256, sm, s>>>(spat, ld_spat, F, ldF, h->L, h->nlat, dev_plan(h->fft), h->fft.tw, JT);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

int ring_synthesis_cplx(const Handle* h, const double2* F, long long ldF, double2* spat, long long ld_spat, int batch,
                        cudaStream_t s) {
    if (batch <= 0) return SPH_OK;
    const int JT = ring_tile(h->nphi, 1);
    const size_t sm = (size_t)2 * JT * h->nphi * sizeof(double2);
    dim3 grid((h->nlat + JT - 1) / JT, batch);
    k_ring_synthesis_cplx<<<grid, 256, sm, s>>>(F, ldF, h->L, spat, ld_spat, h->nlat, dev_plan(h->fft), h->fft.tw, JT);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

}  // namespace sphgpu
