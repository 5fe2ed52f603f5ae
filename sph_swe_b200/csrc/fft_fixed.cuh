// Real ring FFTs of compile-time length N = 3 * 2^k (the lengths the automatic
// grids use: 96, 192, 384, 768, 1536, 3072), used by fft.cu in place of the
// generic kernels for those lengths.
//
// A CTA transforms P complex sequences, i.e. 2P consecutive latitude rings of
// one field packed in pairs (ring 2q real part, ring 2q+1 imaginary part), with
// max(128, P N / 16) threads (one radix-16 butterfly each).  By default P = 4 up
// to N = 768 (8 rings: every longitude row of the tile is one 64-byte run of
// the theta-contiguous grid, 49 KB of shared memory at N = 768), so that
// several CTAs share an SM and one CTA's loads overlap another's passes; the
// autotuner may take twice or half that.  Shared
// memory holds the tile element-major with the sequences innermost,
// buf[i * P + q]: element i of all P sequences is the 16 P bytes that
// longitude i of the 2P rings occupies in the grid.
//
// Stockham passes, all radices and strides compile-time, the sequence index
// fastest across threads so that every quarter-warp touches one contiguous
// 128-byte row of shared memory.  Shared-memory traffic is what bounds these
// kernels, so the schedule keeps the passes through shared memory few:
//   analysis   radix 3 first, fused with the tile load (global -> registers ->
//              butterfly -> shared memory; the first pass has no twiddles), then
//              radix 16 passes (and one 2, 4 or 8); the last pass writes only
//              the outputs the spectrum keeps (m <= L and N - m);
//   synthesis  radix 16 passes (and one 2, 4 or 8) first, the first one
//              reading only the nonzero Fourier rows (the rest are never
//              written), then radix 3 last, fused with the tile store.
// N = 768 takes 2 shared-memory passes (3 | 16 16) instead of 4 (3 8 8 4).
// Twiddles of a radix-16 pass come from 4 table loads (w, w^2, w^4, w^8) and
// products of them.
#pragma once

// needs FFTPlan / RingMap of fft.cu (included from there)

namespace sphgpu {
namespace fftx {

// default complex sequences per CTA (2 P real rings)
template <int N>
constexpr int seqs() { return N <= 768 ? 4 : (N == 1536 ? 2 : 1); }
// threads per CTA: one radix-16 butterfly each, at least 128
template <int N, int P>
constexpr int nt() { return P * N / 16 > 128 ? P * N / 16 : 128; }
// CTAs per SM the register budget is set for
template <int N, int P>
constexpr int minb() { return nt<N, P>() >= 384 ? 1 : (nt<N, P>() >= 192 ? 3 : 4); }

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
// a * (c + SIGN i s)
template <int SIGN>
__device__ __forceinline__ double2 rot(double2 a, double c, double s) {
    return make_double2(a.x * c - SIGN * s * a.y, a.y * c + SIGN * s * a.x);
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
    double2 e[4], o[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        e[k] = cadd(v[k], v[k + 4]);
        o[k] = csub(v[k], v[k + 4]);
    }
    // w8^1 = (h, SIGN h), w8^2 = SIGN i, w8^3 = (-h, SIGN h)
    o[1] = rot<SIGN>(o[1], h, h);
    o[2] = mul_i<SIGN>(o[2]);
    o[3] = rot<SIGN>(o[3], -h, h);
    dft4<SIGN>(e[0], e[1], e[2], e[3]);
    dft4<SIGN>(o[0], o[1], o[2], o[3]);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[2 * k] = e[k];
        v[2 * k + 1] = o[k];
    }
}

// v[0..15] in natural order -> DFT-16 in natural order: n = n2 + 4 n1,
// k = k1 + 4 k2; DFT-4 over n1, twiddles w16^(n2 k1), DFT-4 over n2
template <int SIGN>
__device__ __forceinline__ void dft16(double2* v) {
    constexpr double c1 = 0.92387953251128675612818318939679;  // cos(pi / 8)
    constexpr double s1 = 0.38268343236508977172845998403040;  // sin(pi / 8)
    constexpr double h = 0.70710678118654752440084436210485;
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4<SIGN>(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
    // v[n2 + 4 k1] *= w16^(n2 k1), w16 = exp(SIGN 2 pi i / 16)
    v[5] = rot<SIGN>(v[5], c1, s1);     // w^1
    v[9] = rot<SIGN>(v[9], h, h);       // w^2
    v[13] = rot<SIGN>(v[13], s1, c1);   // w^3
    v[6] = rot<SIGN>(v[6], h, h);       // w^2
    v[10] = mul_i<SIGN>(v[10]);         // w^4
    v[14] = rot<SIGN>(v[14], -h, h);    // w^6
    v[7] = rot<SIGN>(v[7], s1, c1);     // w^3
    v[11] = rot<SIGN>(v[11], -h, h);    // w^6
    v[15] = rot<SIGN>(v[15], -c1, -s1); // w^9
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft4<SIGN>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // X[k1 + 4 k2] sits at v[4 k1 + k2]: transpose
    double2 t[16];
#pragma unroll
    for (int i = 0; i < 16; i++) t[i] = v[i];
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[4 * k1 + k2];
}

template <int R, int SIGN>
__device__ __forceinline__ void dft(double2* v) {
    if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
    else if constexpr (R == 3) dft3<SIGN>(v[0], v[1], v[2]);
    else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 8) dft8<SIGN>(v);
    else dft16<SIGN>(v);
}

// twiddles w^(r b), r = 1..R-1, applied to v[r]; w = exp(SIGN 2 pi i / N) from
// the table tw[t] = exp(-2 pi i t / N).  Radix 16 and 8 load w^b, w^2b, w^4b
// (and w^8b) and form the other powers as products of at most four of them.
template <int N, int R, int SIGN>
__device__ __forceinline__ void twiddle(double2* v, int b, const double2* __restrict__ tw) {
    auto ld = [&](int e) {
        double2 w = __ldg(&tw[e % N]);
        if (SIGN > 0) w.y = -w.y;
        return w;
    };
    if constexpr (R == 2) {
        v[1] = cmul(v[1], ld(b));
    } else if constexpr (R == 3 || R == 4) {
#pragma unroll
        for (int r = 1; r < R; r++) v[r] = cmul(v[r], ld(r * b));
    } else {
        double2 p[R];
        p[1] = ld(b);
        p[2] = ld(2 * b);
        p[4] = ld(4 * b);
        p[3] = cmul(p[1], p[2]);
        p[5] = cmul(p[1], p[4]);
        p[6] = cmul(p[2], p[4]);
        p[7] = cmul(p[3], p[4]);
        if constexpr (R == 16) {
            p[8] = ld(8 * b);
#pragma unroll
            for (int r = 9; r < 16; r++) p[r] = cmul(p[r - 8], p[8]);
        }
#pragma unroll
        for (int r = 1; r < R; r++) v[r] = cmul(v[r], p[r]);
    }
}

// pass schedules.  Power-of-two part M = N / 3 as radix 16s, then one 2, 4 or 8.
constexpr int p2_count(int M) {
    int q = 0;
    while (M >= 16) {
        M /= 16;
        q++;
    }
    return q + (M > 1 ? 1 : 0);
}
constexpr int p2_radix(int M, int i) {
    int q = 0;
    while (M >= 16) {
        if (q == i) return 16;
        M /= 16;
        q++;
    }
    return M;
}
constexpr int npasses(int N) { return 1 + p2_count(N / 3); }
// DIR -1 (analysis): 3 first; +1 (synthesis): 3 last
template <int DIR>
constexpr int radix_at(int N, int q) {
    if (DIR < 0) return q == 0 ? 3 : p2_radix(N / 3, q - 1);
    return q == npasses(N) - 1 ? 3 : p2_radix(N / 3, q);
}
template <int DIR>
constexpr int ls_at(int N, int q) {
    int ls = 1;
    for (int i = 0; i < q; i++) ls *= radix_at<DIR>(N, i);
    return ls;
}

// One Stockham pass through shared memory on P sequences, in place: butterflies
// t = (f, j), j < N/R, inputs s[j + r N/R] times w^(r k N/(Ls R)), k = j mod Ls,
// outputs to d[(j - k) R + k + r Ls].  Element e of sequence f is buf[e * P + f].
// Every thread holds at most 16 complex values across the barrier.
//   ZMASK (first synthesis pass): elements mm < e < N - mm were never written
//         and read as zeros;
//   WMASK (last analysis pass, k = j): only outputs e <= mm or e >= N - mm
//         are written.
template <int N, int P, int Q, int SIGN, int DIR, bool ZMASK, bool WMASK>
__device__ __forceinline__ void pass(double2* buf, const double2* __restrict__ tw, int mm) {
    constexpr int NT = nt<N, P>();
    constexpr int R = radix_at<DIR>(N, Q);
    constexpr int Ls = ls_at<DIR>(N, Q);
    constexpr int NR = N / R;
    constexpr int TOT = P * NR;
    constexpr int IT = (TOT + NT - 1) / NT;
    constexpr int TS = N / (Ls * R);
    static_assert(IT * R <= 16, "at most 16 complex values per thread");
    double2 v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int t = threadIdx.x + NT * it;
        if (TOT % NT == 0 || t < TOT) {
            const int f = t % P, j = t / P, k = j % Ls;
            const double2* s = buf + f;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int e = j + r * NR;
                v[it][r] = (!ZMASK || e <= mm || e >= N - mm) ? s[e * P] : make_double2(0, 0);
            }
            if constexpr (Ls > 1) twiddle<N, R, SIGN>(v[it], k * TS, tw);
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
            for (int r = 0; r < R; r++) {
                const int e = (j - k) * R + k + r * Ls;
                if (!WMASK || e <= mm || e >= N - mm) d[r * Ls * P] = v[it][r];
            }
        }
    }
    __syncthreads();
}

// the shared-memory passes Q .. QE-1
template <int N, int P, int Q, int QE, int SIGN, int DIR>
__device__ __forceinline__ void passes(double2* buf, const double2* __restrict__ tw, int mm) {
    if constexpr (Q < QE) {
        constexpr bool zm = DIR > 0 && Q == 0;
        constexpr bool wm = DIR < 0 && Q == npasses(N) - 1;
        pass<N, P, Q, SIGN, DIR, zm, wm>(buf, tw, mm);
        passes<N, P, Q + 1, QE, SIGN, DIR>(buf, tw, mm);
    }
}

}  // namespace fftx
}  // namespace sphgpu

namespace sphgpu {

// grid tile (2P rings, pairs packed) -> F[b][m][j], m = 0..mF-1 (m > L zero),
// scaled by 2 pi / N (quadrature weight in longitude).  vec != 0: nlat even and
// the field rows 16-byte aligned, so each (longitude, ring pair) is one aligned
// 16-byte load.
template <int N, int P>
__global__ void __launch_bounds__(fftx::nt<N, P>(), fftx::minb<N, P>()) k_ring_analysis_real_n(const double* __restrict__ spat, long long ld_spat,
                                                                    double2* __restrict__ F, long long ldF, int mF, int L,
                                                                    int nlat, const double2* __restrict__ tw, int vec) {
    constexpr int JT = 2 * P, N3 = N / 3, TOT = P * N3, NT = fftx::nt<N, P>();
    constexpr int U = 3;  // radix-3 butterflies whose loads are in flight together
    extern __shared__ double2 fbuf[];
    const int j0 = blockIdx.x * JT;
    const double* src = spat + (long long)blockIdx.y * ld_spat;
    const int mk = min(mF - 1, L);  // the last pass writes elements m <= mk and N - m
    // first pass (radix 3, Ls = 1: no twiddles) straight from the grid:
    // butterfly (f, j) reads longitudes j, j + N/3, j + 2N/3 of ring pair f and
    // writes elements 3j, 3j + 1, 3j + 2
    for (int base = threadIdx.x; base < TOT; base += U * NT) {
        double2 x[U][3];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = base + u * NT;
            const int f = t % P, j = t / P, jr = j0 + 2 * f;
            const bool in = t < TOT && jr < nlat;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const double* p = src + (long long)(j + r * N3) * nlat + jr;
                if (!in) x[u][r] = make_double2(0, 0);
                else if (vec) x[u][r] = __ldg(reinterpret_cast<const double2*>(p));
                else x[u][r] = make_double2(__ldg(p), jr + 1 < nlat ? __ldg(p + 1) : 0.0);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = base + u * NT;
            if (TOT % (U * NT) == 0 || t < TOT) {
                const int f = t % P, j = t / P;
                fftx::dft3<-1>(x[u][0], x[u][1], x[u][2]);
#pragma unroll
                for (int r = 0; r < 3; r++) fbuf[(3 * j + r) * P + f] = x[u][r];
            }
        }
    }
    __syncthreads();
    fftx::passes<N, P, 1, fftx::npasses(N), -1, -1>(fbuf, tw, mk);
    const double scale = 2.0 * kPi / N;
    double2* out = F + (long long)blockIdx.y * ldF;
    for (int idx = threadIdx.x; idx < mF * P; idx += NT) {
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
__global__ void __launch_bounds__(fftx::nt<N, P>(), fftx::minb<N, P>()) k_ring_synthesis_real_n(const double2* __restrict__ F, long long ldF, int mF,
                                                                     int L, double* __restrict__ spat, long long ld_spat,
                                                                     int nlat, const double2* __restrict__ tw,
                                                                     RingMap map, int vec) {
    constexpr int JT = 2 * P, N3 = N / 3, TOT = P * N3, NT = fftx::nt<N, P>();
    constexpr int U = 3;
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
    // rows 0..mm and N-mm..N-1; the rows between are never written (the first
    // pass reads them as zeros)
    constexpr int UL = 8;
    const int tot = (mm + 1) * P;
    for (int base = threadIdx.x; base < tot; base += UL * NT) {
        double2 X[UL], Y[UL];
#pragma unroll
        for (int u = 0; u < UL; u++) {
            const int idx = base + u * NT;
            const int m = idx / P, j = j0 + 2 * (idx % P);
            X[u] = Y[u] = make_double2(0, 0);
            if (idx < tot && j < nlat) X[u] = __ldg(&in[(long long)m * nlat + j]);
            if (idx < tot && j + 1 < nlat) Y[u] = __ldg(&in[(long long)m * nlat + j + 1]);
        }
#pragma unroll
        for (int u = 0; u < UL; u++) {
            const int idx = base + u * NT;
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
    constexpr int NP = fftx::npasses(N);
    fftx::passes<N, P, 0, NP - 1, +1, +1>(fbuf, tw, mm);
    // last pass (radix 3, Ls = N/3, k = j) straight to the grid: butterfly
    // (f, j) reads elements j, j + N/3, j + 2N/3 and writes longitudes
    // j, j + N/3, j + 2N/3 of ring pair f
    double* out = spat + (long long)k * ld_spat;
    for (int base = threadIdx.x; base < TOT; base += U * NT) {
        double2 x[U][3];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = base + u * NT;
            if (TOT % (U * NT) == 0 || t < TOT) {
                const int f = t % P, j = t / P;
#pragma unroll
                for (int r = 0; r < 3; r++) x[u][r] = fbuf[(j + r * N3) * P + f];
                fftx::twiddle<N, 3, +1>(x[u], j, tw);
                fftx::dft3<+1>(x[u][0], x[u][1], x[u][2]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = base + u * NT;
            const int f = t % P, j = t / P, jr = j0 + 2 * f;
            if ((TOT % (U * NT) == 0 || t < TOT) && jr < nlat) {
                if (map.rowdiv) {  // rings jr, jr + 1 times 1 / rowdiv
                    const double s0 = 1.0 / map.rowdiv[jr], s1 = jr + 1 < nlat ? 1.0 / map.rowdiv[jr + 1] : 0.0;
#pragma unroll
                    for (int r = 0; r < 3; r++) x[u][r] = make_double2(x[u][r].x * s0, x[u][r].y * s1);
                }
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    double* p = out + (long long)(j + r * N3) * nlat + jr;
                    if (vec) {
                        *reinterpret_cast<double2*>(p) = x[u][r];
                    } else {
                        p[0] = x[u][r].x;
                        if (jr + 1 < nlat) p[1] = x[u][r].y;
                    }
                }
            }
        }
    }
}

}  // namespace sphgpu
