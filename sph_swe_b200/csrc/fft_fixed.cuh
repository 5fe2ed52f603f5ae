// Real ring FFTs of compile-time length N = 3 * 2^k (the lengths the automatic
// grids use: 96, 192, 384, 768, 1536, 3072), used by fft.cu in place of the
// generic kernels for those lengths.
//
// A CTA of 256 threads transforms P complex sequences (by default P = 8 up to
// N = 768, i.e. 16 rings: every longitude row of the tile is one 128-byte run
// of the theta-contiguous grid; P is a template parameter so that the
// autotuner can trade tile width for CTAs per SM), i.e. 2P consecutive
// latitude rings of one field packed in pairs (ring 2q real part, ring 2q+1
// imaginary part).  Shared memory holds the tile element-major with the
// sequences innermost, buf[i * P + q]: element i of all P sequences is the
// 16 P bytes that longitude i of the 2P rings occupies in the grid, so the
// grid tile is copied in (analysis) and out (synthesis) as 16-byte chunks
// without rearrangement, by asynchronous copies (cp.async) on the way in.
// The Stockham passes (radix 3 first, then 8, 4, 2; all radices and strides
// compile-time) run in place in that one buffer, the sequence index fastest
// across threads so that every quarter-warp touches one contiguous row: each
// pass reads its butterfly inputs into registers, synchronises, and writes
// the outputs, so only P * N * 16 bytes of shared memory are needed.
#pragma once

// needs FFTPlan / RingMap of fft.cu (included from there)

namespace sphgpu {
namespace fftx {

constexpr int NT = 256;     // threads per CTA
// default complex sequences per CTA (2 P real rings) and the padded row stride
template <int N>
constexpr int seqs() { return N <= 768 ? 8 : (N == 1536 ? 4 : 2); }

// 16-byte asynchronous global -> shared copy; bytes = 0 writes zeros
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, int bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// multiply by sign * i
template <int SIGN>
__device__ __forceinline__ double2 mul_i(double2 a) {
    return SIGN < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

template <int SIGN>
__device__ __forceinline__ void dft2(double2& a, double2& b) {
    const double2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int SIGN>
__device__ __forceinline__ void dft4(double2& a, double2& b, double2& c, double2& d) {
    const double2 s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = mul_i<SIGN>(csub(b, d));
    a = cadd(s0, s2);
    c = csub(s0, s2);
    b = cadd(s1, s3);
    d = csub(s1, s3);
}

template <int SIGN>
__device__ __forceinline__ void dft3(double2& a, double2& b, double2& c) {
    const double s = SIGN * 0.86602540378443864676372317075294;  // sin(2 pi / 3)
    const double2 t1 = cadd(b, c), t2 = csub(b, c);
    const double2 m1 = make_double2(a.x - 0.5 * t1.x, a.y - 0.5 * t1.y);
    const double2 m2 = make_double2(-s * t2.y, s * t2.x);
    a = cadd(a, t1);
    b = cadd(m1, m2);
    c = csub(m1, m2);
}

// v[0..7] in natural order -> DFT-8 in natural order
template <int SIGN>
__device__ __forceinline__ void dft8(double2* v) {
    constexpr double h = 0.70710678118654752440084436210485;
    // radix-2 over the halves: e_k = v_k + v_{k+4}, o_k = (v_k - v_{k+4}) w8^k
    double2 e[4], o[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        e[k] = cadd(v[k], v[k + 4]);
        o[k] = csub(v[k], v[k + 4]);
    }
    // w8^1 = (h, SIGN h), w8^2 = SIGN i, w8^3 = (-h, SIGN h)
    o[1] = make_double2(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
    o[2] = mul_i<SIGN>(o[2]);
    o[3] = make_double2(-h * (o[3].x + SIGN * o[3].y), h * (SIGN * o[3].x - o[3].y));
    dft4<SIGN>(e[0], e[1], e[2], e[3]);
    dft4<SIGN>(o[0], o[1], o[2], o[3]);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[2 * k] = e[k];
        v[2 * k + 1] = o[k];
    }
}

template <int R, int SIGN>
__device__ __forceinline__ void dft(double2* v) {
    if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
    else if constexpr (R == 3) dft3<SIGN>(v[0], v[1], v[2]);
    else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
    else dft8<SIGN>(v);
}

// pass schedule of N = 3 * 2^k: radix 3, then 8s, then a 4 or a 2
constexpr int pow2_part(int n) { return n % 3 == 0 ? n / 3 : n; }
constexpr int radix_at(int N, int q) {
    if (q == 0) return 3;
    int m = pow2_part(N);
    for (int i = 1; i < q; i++) m /= (m % 8 == 0 && m != 16 && m != 4 && m != 2) ? 8 : (m % 4 == 0 ? 4 : 2);
    return (m % 8 == 0 && m != 16) ? 8 : (m % 4 == 0 ? 4 : 2);
}
constexpr int npasses(int N) {
    int m = pow2_part(N), q = 1;
    while (m > 1) {
        m /= (m % 8 == 0 && m != 16) ? 8 : (m % 4 == 0 ? 4 : 2);
        q++;
    }
    return q;
}
constexpr int ls_at(int N, int q) {
    int ls = 1;
    for (int i = 0; i < q; i++) ls *= radix_at(N, i);
    return ls;
}

// One Stockham pass on P sequences in place: butterflies t = (f, j), j < N/R,
// inputs s[j + r N/R] times w^(r k N/(Ls R)), k = j mod Ls, outputs to
// d[(j - k) R + k + r Ls]; w = exp(SIGN 2 pi i / N) from the table tw[t] = exp(-2 pi i t / N).
// Element e of sequence f is buf[e * P + f]; f = t mod P.
template <int N, int P, int Q, int SIGN>
__device__ __forceinline__ void pass(double2* buf, const double2* __restrict__ tw) {
    constexpr int R = radix_at(N, Q);
    constexpr int Ls = ls_at(N, Q);
    constexpr int NR = N / R;
    constexpr int TOT = P * NR;
    constexpr int IT = (TOT + NT - 1) / NT;
    constexpr int TS = N / (Ls * R);
    double2 v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int t = threadIdx.x + NT * it;
        if (TOT % NT == 0 || t < TOT) {
            const int f = t % P, j = t / P, k = j % Ls;
            const double2* s = buf + f;
            v[it][0] = s[j * P];
#pragma unroll
            for (int r = 1; r < R; r++) {
                double2 w = __ldg(&tw[(r * k * TS) % N]);
                if (SIGN > 0) w.y = -w.y;
                v[it][r] = cmul(s[(j + r * NR) * P], w);
            }
            dft<R, SIGN>(v[it]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int t = threadIdx.x + NT * it;
        if (TOT % NT == 0 || t < TOT) {
            const int f = t % P, j = t / P, k = j % Ls;
            double2* d = buf + ((j - k) * R + k) * P + f;
#pragma unroll
            for (int r = 0; r < R; r++) d[r * Ls * P] = v[it][r];
        }
    }
    __syncthreads();
}

template <int N, int P, int Q, int SIGN>
__device__ __forceinline__ void passes(double2* buf, const double2* __restrict__ tw) {
    if constexpr (Q < npasses(N)) {
        pass<N, P, Q, SIGN>(buf, tw);
        passes<N, P, Q + 1, SIGN>(buf, tw);
    }
}

}  // namespace fftx
}  // namespace sphgpu

namespace sphgpu {

// grid tile (2P rings, pairs packed) -> F[b][m][j], m = 0..mF-1 (m > L zero),
// scaled by 2 pi / N (quadrature weight in longitude).  vec != 0: nlat even and
// the field rows 16-byte aligned, so each (longitude, ring pair) is one
// aligned 16-byte chunk copied by cp.async.
template <int N, int P>
__global__ void __launch_bounds__(fftx::NT, 2) k_ring_analysis_real_n(const double* __restrict__ spat, long long ld_spat,
                                                                    double2* __restrict__ F, long long ldF, int mF, int L,
                                                                    int nlat, const double2* __restrict__ tw, int vec) {
    constexpr int JT = 2 * P;
    extern __shared__ double2 fbuf[];
    const int j0 = blockIdx.x * JT;
    const double* src = spat + (long long)blockIdx.y * ld_spat;
    if (vec) {
        for (int idx = threadIdx.x; idx < N * P; idx += fftx::NT) {
            const int i = idx / P, j = j0 + 2 * (idx % P);
            const bool in = j < nlat;
            fftx::cp_async16(&fbuf[idx], src + (long long)i * nlat + (in ? j : 0), in ? 16 : 0);
        }
        fftx::cp_async_wait_all();
    } else {
        // tile load in batches of U independent loads per thread
        constexpr int PER = N * JT / fftx::NT;
        constexpr int U = PER <= 12 ? PER : 8;
        static_assert((N * JT) % fftx::NT == 0 && PER % U == 0, "tile divides into batches");
        for (int base = 0; base < N * JT; base += U * fftx::NT) {
            double v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int idx = base + threadIdx.x + u * fftx::NT;
                const int i = idx / JT, j = j0 + idx % JT;
                v[u] = (j < nlat) ? __ldg(&src[(long long)i * nlat + j]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int idx = base + threadIdx.x + u * fftx::NT;
                const int i = idx / JT, jj = idx % JT;
                reinterpret_cast<double*>(&fbuf[i * P + (jj >> 1)])[jj & 1] = v[u];
            }
        }
    }
    __syncthreads();
    fftx::passes<N, P, 0, -1>(fbuf, tw);
    const double scale = 2.0 * kPi / N;
    double2* out = F + (long long)blockIdx.y * ldF;
    for (int idx = threadIdx.x; idx < mF * P; idx += fftx::NT) {
        const int m = idx / P, q = idx % P;
        const int j = j0 + 2 * q;
        if (j >= nlat) continue;
        double2 X = make_double2(0, 0), Y = make_double2(0, 0);
        if (m <= L) {
            const double2 a = fbuf[m * P + q];
            const double2 c = fbuf[((N - m) % N) * P + q];
            X = make_double2(0.5 * (a.x + c.x) * scale, 0.5 * (a.y - c.y) * scale);
            Y = make_double2(0.5 * (a.y + c.y) * scale, -0.5 * (a.x - c.x) * scale);
        }
        out[(long long)m * nlat + j] = X;
        if (j + 1 < nlat) out[(long long)m * nlat + j + 1] = Y;
    }
}

// F[fs][m][j] (optionally times i*m) -> grid k; m = 0 contributes its real part.
// vec != 0: nlat even and the field rows 16-byte aligned (16-byte stores).
template <int N, int P>
__global__ void __launch_bounds__(fftx::NT, 2) k_ring_synthesis_real_n(const double2* __restrict__ F, long long ldF, int mF,
                                                                     int L, double* __restrict__ spat, long long ld_spat,
                                                                     int nlat, const double2* __restrict__ tw,
                                                                     RingMap map, int vec) {
    constexpr int JT = 2 * P;
    extern __shared__ double2 fbuf[];
    const int j0 = blockIdx.x * JT;
    const int k = blockIdx.y;
    int fs = k, mod = 0;
    if (map.use) {
        const int mem = k / map.period, r = k - mem * map.period;
        fs = mem * map.src_stride + map.src[r];
        mod = map.mod[r];
    }
    const double2* in = F + (long long)fs * ldF;
    const int mm = min(min(mF - 1, L), (N - 1) / 2);
    // rows mm+1 .. N-mm-1 are zero; rows 0..mm and N-mm..N-1 are written below
    for (int idx = (mm + 1) * P + threadIdx.x; idx < (N - mm) * P; idx += fftx::NT) fbuf[idx] = make_double2(0, 0);
    constexpr int U = 8;
    const int tot = (mm + 1) * P;
    for (int base = threadIdx.x; base < tot; base += U * fftx::NT) {
        double2 X[U], Y[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int idx = base + u * fftx::NT;
            const int m = idx / P, j = j0 + 2 * (idx % P);
            X[u] = Y[u] = make_double2(0, 0);
            if (idx < tot && j < nlat) X[u] = __ldg(&in[(long long)m * nlat + j]);
            if (idx < tot && j + 1 < nlat) Y[u] = __ldg(&in[(long long)m * nlat + j + 1]);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int idx = base + u * fftx::NT;
            if (idx >= tot) break;
            const int m = idx / P, q = idx % P;
            double2 x = X[u], y = Y[u];
            if (mod) {  // d/dlambda: times i*m
                x = make_double2(-m * x.y, m * x.x);
                y = make_double2(-m * y.y, m * y.x);
            }
            if (m == 0) {
                fbuf[q] = make_double2(x.x, y.x);
            } else {
                fbuf[m * P + q] = make_double2(x.x - y.y, x.y + y.x);        // X + iY
                fbuf[(N - m) * P + q] = make_double2(x.x + y.y, -x.y + y.x);  // conj(X) + i conj(Y)
            }
        }
    }
    __syncthreads();
    fftx::passes<N, P, 0, +1>(fbuf, tw);
    double* out = spat + (long long)k * ld_spat;
    if (vec) {
#pragma unroll 8
        for (int idx = threadIdx.x; idx < N * P; idx += fftx::NT) {
            const int i = idx / P, j = j0 + 2 * (idx % P);
            if (j < nlat) *reinterpret_cast<double2*>(&out[(long long)i * nlat + j]) = fbuf[idx];
        }
    } else {
#pragma unroll 8
        for (int idx = threadIdx.x; idx < N * JT; idx += fftx::NT) {
            const int i = idx / JT, jj = idx % JT;
            const int j = j0 + jj;
            const double2 z = fbuf[i * P + (jj >> 1)];
            if (j < nlat) out[(long long)i * nlat + j] = (jj & 1) ? z.y : z.x;
        }
    }
}

}  // namespace sphgpu
