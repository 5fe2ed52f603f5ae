// Legendre stage on tcgen05 kind::i8: the integer split (Ozaki scheme) with
// exact int32 sums in tensor memory.
//
// Included by legendre_tc.cu after legendre_tcs.cuh (PTX helpers, TMA loads).
//
// Per order m and parity the contraction C = A B (synthesis: A = P_l^m(mu_j),
// rows = northern latitudes, K = degrees of the parity, B = spectra; analysis:
// A = P_l^m(mu_j) w_j, rows = degrees, K = latitudes, B = north +/- south
// Fourier sums; columns = fields x re/im) is evaluated exactly in integers:
//   * every row of A carries a power-of-two scale 2^ea, every column of B one
//     of 2^eb (frexp exponent of (1 + 2^-7) times the largest magnitude: the
//     synthesis row over all degrees of order m up to the table degree, the
//     analysis row its own, the synthesis column over all degrees of the call,
//     the analysis column max_j |north_j| + |south_j|, which bounds both
//     parities), so the scaled entries a satisfy |a| < 128/129;
//   * v = rint(a 2^31) is written in balanced base 256,
//     v = d0 2^24 + d1 2^16 + d2 2^8 + d3 with every digit in [-128, 127]; the
//     digit word is (v + 0x808080) ^ 0x808080 (its bytes 3..0 are d0..d3);
//   * one kind::i8 MMA (signed x signed, int32 accumulator) per digit product
//     d_s(A) d_t(B) with s + t < 4 (10 products), accumulated in tensor memory
//     per group g = s + t over the whole K range of the tile: the dropped
//     products are zero-mean, and no partial sum is ever rounded;
//   * one FP64 combination per finished tile,
//     C = 2^(ea + eb - 14) (((G0 + G1 2^-8) + G2 2^-16) + G3 2^-24).
// The A digits (P tables) are built once per handle; the B digits are formed
// per tile by the producer warps: a first pass takes the column maxima over
// the tile's whole K range, a second pass writes the digit planes of one K
// segment at a time into a two-slot ring, in the tensor core's K-major
// no-swizzle layout.
//
// Tables (int8 digit planes, 16-byte rows of 16 K values, 64 rows = 1 KB):
//   synthesis  SY[d][z][j][16]: z = zoff(m) + parity * 2 nch(m) + l'/16,
//              nch(m) = 32-degree chunks of parity 0 of order m (both parities
//              padded to it), rows j padded to a multiple of 64;
//   analysis   AN[d][j/16][y][16]: y = aoff(m) + parity * pad64(nlp0) + l',
//              each (m, parity) block padded with zero rows to a multiple of 64.
// A 4-D tensor map (1 KB row blocks as 256 words, row block, z, digit) makes a
// chunk's A operand of one parity one TMA box {256, 2, 2, 4}: 128 rows x 32 K
// x 4 digit planes, in shared memory [digit][z][128 rows][16 B] (core matrices
// 128 B apart along M, 2 KB apart along K).
//
// One persistent CTA of 14 warps per SM: producers (warps 0-7) stage B, warp
// 12 issues the A loads, warp 13 the MMAs, consumers (warps 8-11, warp 8 + q
// reading tensor-memory lane quadrant q) combine and write finished tiles.
// Every wait is bounded as in the split-TF32 kernels.

namespace li8 {
constexpr int M = 128;                // rows per tile (TMEM lanes)
constexpr int KC = 32;                // K per chunk: one kind::i8 MMA K step
constexpr int ND = 4;                 // digit planes
constexpr int NG = 4;                 // product groups kept (s + t < NG)
constexpr int NSTAGE = 3;             // A stages
constexpr int A_PAR = M * KC * ND;    // 16 KB: one parity's A operand of a chunk
constexpr int A_STAGE = 2 * A_PAR;    // 32 KB
constexpr int NPROD = 256;            // producer threads (warps 0-7)
constexpr int NCONS = 128;            // consumer threads (warps 8-11)
constexpr int TMA_WARP = 12;
constexpr int MMA_WARP = 13;
constexpr int NT = 448;
constexpr int B_SLOT = 48 * 1024;     // one B segment: 2 parities x 4 planes x NC columns x KSEG
constexpr int OFF_B = NSTAGE * A_STAGE;
constexpr int OFF_MAX = OFF_B + 2 * B_SLOT;     // unsigned long long colmax[64]
constexpr int OFF_EXP = OFF_MAX + 64 * 8;       // int exps[2][64]
constexpr int OFF_SCL = OFF_EXP + 2 * 64 * 4;   // double2 scl[64]
constexpr int OFF_BAR = OFF_SCL + 64 * 16;
constexpr int BYTES = OFF_BAR + 256;
static_assert(OFF_B % 1024 == 0 && B_SLOT % 1024 == 0 && OFF_MAX % 16 == 0, "aligned buffers");
}  // namespace li8

// degrees of one parity of order m up to degree T, 32-degree chunks of parity 0
__host__ __device__ inline int i8_nlp(int T, int m, int par) { return T - m - par >= 0 ? (T - m - par) / 2 + 1 : 0; }
__host__ __device__ inline int i8_nch(int T, int m) { return (i8_nlp(T, m, 0) + li8::KC - 1) / li8::KC; }
// prepared-B chunks (kernels with both operands by TMA, legendre_i8b.cuh):
// synthesis chunks of the orders below m (degree lmax), sum_{m' < m} ((lmax - m') / 64 + 1)
__host__ __device__ inline long long i8b_syn_coff(int lmax, int m) {
    auto fs = [](int n) -> long long {  // sum_{x = 0..n} floor(x / 64)
        if (n < 0) return 0;
        const long long q = n / 64, r = n % 64;
        return 32 * q * (q - 1) + q * (r + 1);
    };
    return (long long)m + fs(lmax) - fs(lmax - m);
}
// analysis chunks of one order: the latitudes of one hemisphere in steps of 32
__host__ __device__ inline int i8b_ana_nch(int nh) { return (nh + li8::KC - 1) / li8::KC; }

// instruction descriptor: D = S32, A = B = S8, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_s8(int m, int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_s8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}

// balanced base-256 digit word of v = rint(t s1 s2), s1 s2 = 2^(31 - e) split in
// two powers of two so that neither overflows (|v| < 2^31): t s1 is exact, and
// adding 1.5 2^52 in the same FMA rounds t s1 s2 to the nearest integer (half
// to even), which then sits in the low 32 bits of the result
__device__ __forceinline__ uint32_t i8_word(double t, double s1, double s2) {
    const uint32_t v = (uint32_t)__double2loint(fma(t * s1, s2, 0x1.8p52));
    return (v + 0x808080u) ^ 0x808080u;
}
// the powers of two 2^(31 - e) as two factors
__device__ __forceinline__ double2 i8_scale(int e) {
    const int k = 31 - e, k1 = k / 2, k2 = k - k1;
    return make_double2(ldexp(1.0, k1), ldexp(1.0, k2));
}
// frexp exponent of (1 + 2^-7) mx, 0 for mx = 0
__device__ __forceinline__ int i8_exp(double mx) {
    if (!(mx > 0.0)) return 0;
    int e;
    frexp(mx * (1.0 + 0x1p-7), &e);
    return e;
}
// 2^k as a double (k may leave the normal range)
__device__ __forceinline__ double i8_pow2(int k) {
    if (k >= -1022 && k <= 1023) return __hiloint2double((k + 1023) << 20, 0);
    return ldexp(1.0, k);
}

// unsigned 64-bit pattern of a non-negative double (ordered like the values)
__device__ __forceinline__ unsigned long long i8_bits(double x) { return (unsigned long long)__double_as_longlong(x); }

// the digit planes of 4 words (values of 4 consecutive K indices): o[d] holds
// digit d (0 = most significant) of the 4 values, value k at byte k
__device__ __forceinline__ void i8_planes4(uint32_t a, uint32_t b, uint32_t c, uint32_t e, uint32_t* o) {
    const uint32_t t0 = __byte_perm(a, b, 0x5140), t1 = __byte_perm(a, b, 0x7362);
    const uint32_t t2 = __byte_perm(c, e, 0x5140), t3 = __byte_perm(c, e, 0x7362);
    o[3] = __byte_perm(t0, t2, 0x5410);  // byte 0 of each word: d3
    o[2] = __byte_perm(t0, t2, 0x7632);  // byte 1: d2
    o[1] = __byte_perm(t1, t3, 0x5410);  // byte 2: d1
    o[0] = __byte_perm(t1, t3, 0x7632);  // byte 3: d0
}

// Producer micro-tasks: one task = one field and 4 consecutive K indices of
// both parities; task t -> (q = t & 3, fl = (t >> 2) % NF, zl = (t >> 2) / NF)
// with K indices 16 zl + 4 q + (0..3), so that 4 neighbouring lanes fill one
// 16-byte row of a digit plane.  Every producer runs the same number of loop
// trips (tasks beyond the count contribute nothing), so the column-maximum
// reduction can use warp shuffles.
__device__ __forceinline__ int i8_trips(int ntasks) { return (ntasks + li8::NPROD - 1) / li8::NPROD; }

// column maxima (bit patterns of non-negative doubles) of a task's two columns,
// reduced over the 4 lanes of one field before one shared-memory atomic each
__device__ __forceinline__ void i8_colmax(double mr, double mi, bool lead, int fl, unsigned long long* colmax) {
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
        mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        mi = fmax(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    }
    if (lead) {
        atomicMax(&colmax[2 * fl], i8_bits(mr));
        atomicMax(&colmax[2 * fl + 1], i8_bits(mi));
    }
}

// store the 4 plane words of one (parity, column) stream of a task
template <int NC, int ZSEG>
__device__ __forceinline__ void i8_put(unsigned char* Bs, int par, int zl, int c, int q, const uint32_t* o) {
#pragma unroll
    for (int d = 0; d < li8::ND; d++)
        *reinterpret_cast<uint32_t*>(Bs + ((size_t)((par * li8::ND + d) * ZSEG + zl) * NC + c) * 16 + 4 * q) = o[d];
}

struct I8Args {
    const int* erow;        // row exponents: synthesis esy[m * nh + j]; analysis ean[pidx(tlmax, l, m)]
    unsigned char* B;       // prepared B chunks (kernels with both operands by TMA)
    int* ecol;              // their column exponents [ct][m][NC]
    long long cpt;          // B chunks per column tile
    const long long* zoff;  // synthesis table: first z of order m
    const long long* aoff;  // analysis table: first row of order m
    int tlmax, lmax, nh, nlat, batch;
    int nct, nrt, nm, ntiles, order;
    long long ld_spec, ldF;
    int* flag;
};

struct I8Tile {
    int t;           // tile index (>= ntiles: none)
    int m, rt, ct;
    int nch;         // chunks of K
};

__device__ __forceinline__ int i8_order_m(const I8Args& a, int mi) {
    // order 0: m ascending (longest K first in the synthesis); 1: m paired with
    // its complement (0, L, 1, L-1, ...), alternating long and short tiles
    if (a.order == 1) return (mi & 1) ? a.nm - 1 - (mi >> 1) : (mi >> 1);
    return mi;
}

template <class Dir>
__device__ __forceinline__ I8Tile i8_tile(const I8Args& a, int t) {
    I8Tile p;
    for (; t < a.ntiles; t += gridDim.x) {
        p.ct = t % a.nct;
        const int rest = t / a.nct;
        p.rt = rest % a.nrt;
        p.m = i8_order_m(a, rest / a.nrt);
        p.nch = Dir::nch(a, p.m, p.rt);
        if (p.nch > 0) break;
    }
    p.t = t;
    return p;
}


// ------------------------------------------------------------------ synthesis
template <int NC>
struct SynI8 {
    static constexpr int NF = NC / 2;
    static constexpr int KSEG = li8::B_SLOT / (2 * li8::ND * NC);  // K per B segment
    static constexpr int ZSEG = KSEG / 16;
    __device__ static int nch(const I8Args& a, int m, int) { return (i8_nlp(a.lmax, m, 0) + li8::KC - 1) / li8::KC; }
    // prepared B: chunks of order m and their first chunk within the column tile
    __device__ static int prep_nch(const I8Args& a, int m) { return nch(a, m, 0); }
    __device__ static long long prep_coff(const I8Args& a, int m) { return i8b_syn_coff(a.lmax, m); }
    __device__ static int3 box(const I8Args& a, const I8Tile& p, int kc, int par) {
        const long long z = a.zoff[p.m] + (long long)par * 2 * i8_nch(a.tlmax, p.m) + 2 * kc;
        return make_int3(0, 2 * p.rt, (int)z);
    }
    // tasks of a K range of nz z groups (16 K indices each, per parity)
    __device__ static int tasks(int nz) { return NF * 4 * nz; }
    // the 8 coefficients l = m + 2 k0 .. m + 2 k0 + 7 (K indices k0..k0+3 of both parities)
    __device__ static void load(const I8Args& a, const I8Tile& p, int f, int k0, const double2* __restrict__ spec,
                                double2* q) {
        const double2* src = spec + (long long)(f < a.batch ? f : 0) * a.ld_spec;
        const int l0 = p.m + 2 * k0;
#pragma unroll
        for (int i = 0; i < 8; i++)
            q[i] = (f < a.batch && l0 + i <= a.lmax) ? src[pidx(a.lmax, l0 + i, p.m)] : make_double2(0.0, 0.0);
    }
    // pass 1: column maxima of |re|, |im| over all degrees of the tile
    __device__ static void scan(const I8Args& a, const I8Tile& p, int task, bool live, const double2* __restrict__ spec,
                                unsigned long long* colmax) {
        const int q = task & 3, fl = (task >> 2) % NF, zl = (task >> 2) / NF;
        double mr = 0.0, mi = 0.0;
        if (live) {
            double2 v[8];
            load(a, p, p.ct * NF + fl, 16 * zl + 4 * q, spec, v);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                mr = fmax(mr, fabs(v[i].x));
                mi = fmax(mi, fabs(v[i].y));
            }
        }
        i8_colmax(mr, mi, live && q == 0, fl, colmax);
    }
    // pass 2: the digit planes of 4 K indices of both parities, both columns,
    // handed to put(parity, z group, column, lane q, plane words)
    template <class Put>
    __device__ static void digits(const I8Args& a, const I8Tile& p, int task, int z0, const double2* __restrict__ spec,
                                  const double2* scl, Put&& put) {
        const int q = task & 3, fl = (task >> 2) % NF, zl = (task >> 2) / NF;
        double2 v[8];
        load(a, p, p.ct * NF + fl, 16 * (z0 + zl) + 4 * q, spec, v);
        const double2 sr = scl[2 * fl], si = scl[2 * fl + 1];
#pragma unroll
        for (int par = 0; par < 2; par++) {
            uint32_t o[4];
            i8_planes4(i8_word(v[par].x, sr.x, sr.y), i8_word(v[2 + par].x, sr.x, sr.y),
                       i8_word(v[4 + par].x, sr.x, sr.y), i8_word(v[6 + par].x, sr.x, sr.y), o);
            put(par, zl, 2 * fl, q, o);
            i8_planes4(i8_word(v[par].y, si.x, si.y), i8_word(v[2 + par].y, si.x, si.y),
                       i8_word(v[4 + par].y, si.x, si.y), i8_word(v[6 + par].y, si.x, si.y), o);
            put(par, zl, 2 * fl + 1, q, o);
        }
    }
    // consumer: the row exponent of TMEM lane r (latitude 128 rt + r), less
    // the 14 of the combination, loaded ahead of the accumulator
    __device__ static void row_exp(const I8Args& a, const I8Tile& p, int r, int* er) {
        const int j = p.rt * li8::M + r;
        er[0] = j < a.nh ? a.erow[(long long)p.m * a.nh + j] - 14 : 0;
        er[1] = 0;
    }
    // consumer: TMEM lane r = latitude 128 rt + r; e, o: 8 columns c0.. of
    // parity 0 / 1, ec8 their column exponents
    __device__ static void epilogue(const I8Args& a, const I8Tile& p, int r, int c0, const int* er, const int* ec8,
                                    const double* e, const double* o, double2* __restrict__ F) {
        const int j = p.rt * li8::M + r;
        if (j >= a.nh) return;
        const int ea = er[0];
        const int fb = p.ct * NF + c0 / 2;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int f = fb + u;
            if (f >= a.batch) continue;
            const double sr = i8_pow2(ea + ec8[2 * u]), si = i8_pow2(ea + ec8[2 * u + 1]);
            const double er = e[2 * u] * sr, ei = e[2 * u + 1] * si, orr = o[2 * u] * sr, oi = o[2 * u + 1] * si;
            double2* out = F + (long long)f * a.ldF + (long long)p.m * a.nlat;
            out[j] = make_double2(er + orr, ei + oi);
            out[a.nlat - 1 - j] = make_double2(er - orr, ei - oi);
        }
    }
};

// ------------------------------------------------------------------ analysis
template <int NC>
struct AnaI8 {
    static constexpr int NF = NC / 2;
    static constexpr int KSEG = li8::B_SLOT / (2 * li8::ND * NC);
    static constexpr int ZSEG = KSEG / 16;
    __device__ static int nch(const I8Args& a, int m, int rt) {
        return li8::M * rt < i8_nlp(a.lmax, m, 0) ? (a.nh + li8::KC - 1) / li8::KC : 0;
    }
    __device__ static int prep_nch(const I8Args& a, int) { return i8b_ana_nch(a.nh); }
    __device__ static long long prep_coff(const I8Args& a, int m) { return (long long)m * i8b_ana_nch(a.nh); }
    __device__ static int3 box(const I8Args& a, const I8Tile& p, int kc, int par) {
        const long long y = a.aoff[p.m] + (long long)par * tcs_pad64(i8_nlp(a.tlmax, p.m, 0)) + li8::M * p.rt;
        return make_int3(0, (int)(y >> 6), 2 * kc);
    }
    __device__ static int tasks(int nz) { return NF * 4 * nz; }
    // north and south Fourier values of the latitudes j0..j0+3
    __device__ static void load(const I8Args& a, const I8Tile& p, int f, int j0, const double2* __restrict__ F,
                                double2* n, double2* s) {
        const double2* src = F + (long long)(f < a.batch ? f : 0) * a.ldF + (long long)p.m * a.nlat;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const bool v = f < a.batch && j0 + i < a.nh;
            n[i] = v ? src[j0 + i] : make_double2(0.0, 0.0);
            s[i] = v ? src[a.nlat - 1 - j0 - i] : make_double2(0.0, 0.0);
        }
    }
    // pass 1: column maxima of |north| + |south| (re, im) over all latitudes
    __device__ static void scan(const I8Args& a, const I8Tile& p, int task, bool live, const double2* __restrict__ F,
                                unsigned long long* colmax) {
        const int q = task & 3, fl = (task >> 2) % NF, zl = (task >> 2) / NF;
        double mr = 0.0, mi = 0.0;
        if (live) {
            double2 n[4], s[4];
            load(a, p, p.ct * NF + fl, 16 * zl + 4 * q, F, n, s);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                mr = fmax(mr, fabs(n[i].x) + fabs(s[i].x));
                mi = fmax(mi, fabs(n[i].y) + fabs(s[i].y));
            }
        }
        i8_colmax(mr, mi, live && q == 0, fl, colmax);
    }
    // pass 2: digits of north + south (parity 0) and north - south (parity 1)
    // of 4 latitudes, both columns; the scale is applied to north and south
    // first (exact), so the sum is rounded once, as (north +/- south) would be
    template <class Put>
    __device__ static void digits(const I8Args& a, const I8Tile& p, int task, int z0, const double2* __restrict__ F,
                                  const double2* scl, Put&& put) {
        const int q = task & 3, fl = (task >> 2) % NF, zl = (task >> 2) / NF;
        double2 n[4], s[4];
        load(a, p, p.ct * NF + fl, 16 * (z0 + zl) + 4 * q, F, n, s);
        const double2 sr = scl[2 * fl], si = scl[2 * fl + 1];
        double nr[4], sre[4], ni[4], sim[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            nr[i] = n[i].x * sr.x;
            sre[i] = s[i].x * sr.x;
            ni[i] = n[i].y * si.x;
            sim[i] = s[i].y * si.x;
        }
        auto w = [](double t, double s2) {
            const uint32_t v = (uint32_t)__double2loint(fma(t, s2, 0x1.8p52));
            return (v + 0x808080u) ^ 0x808080u;
        };
        uint32_t o[4];
        i8_planes4(w(nr[0] + sre[0], sr.y), w(nr[1] + sre[1], sr.y), w(nr[2] + sre[2], sr.y), w(nr[3] + sre[3], sr.y), o);
        put(0, zl, 2 * fl, q, o);
        i8_planes4(w(ni[0] + sim[0], si.y), w(ni[1] + sim[1], si.y), w(ni[2] + sim[2], si.y), w(ni[3] + sim[3], si.y), o);
        put(0, zl, 2 * fl + 1, q, o);
        i8_planes4(w(nr[0] - sre[0], sr.y), w(nr[1] - sre[1], sr.y), w(nr[2] - sre[2], sr.y), w(nr[3] - sre[3], sr.y), o);
        put(1, zl, 2 * fl, q, o);
        i8_planes4(w(ni[0] - sim[0], si.y), w(ni[1] - sim[1], si.y), w(ni[2] - sim[2], si.y), w(ni[3] - sim[3], si.y), o);
        put(1, zl, 2 * fl + 1, q, o);
    }
    // consumer: row exponents (less 14) of the degrees l' = 128 rt + r of both
    // parities, loaded ahead of the accumulator
    __device__ static void row_exp(const I8Args& a, const I8Tile& p, int r, int* er) {
        const int le = p.m + 2 * (li8::M * p.rt + r);
        er[0] = le <= a.lmax ? a.erow[pidx(a.tlmax, le, p.m)] - 14 : 0;
        er[1] = le + 1 <= a.lmax ? a.erow[pidx(a.tlmax, le + 1, p.m)] - 14 : 0;
    }
    // consumer: TMEM lane r = degree index l' = 128 rt + r of both parities
    __device__ static void epilogue(const I8Args& a, const I8Tile& p, int r, int c0, const int* er, const int* ec8,
                                    const double* e, const double* o, double2* __restrict__ spec) {
        const int lp = li8::M * p.rt + r;
        const int le = p.m + 2 * lp;
        if (le > a.lmax) return;
        const bool odd = le + 1 <= a.lmax;
        const int eae = er[0], eao = er[1];
        const int fb = p.ct * NF + c0 / 2;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int f = fb + u;
            if (f >= a.batch) continue;
            double2* out = spec + (long long)f * a.ld_spec;
            const int cr = ec8[2 * u], ci = ec8[2 * u + 1];
            out[pidx(a.lmax, le, p.m)] = make_double2(e[2 * u] * i8_pow2(eae + cr), e[2 * u + 1] * i8_pow2(eae + ci));
            if (odd)
                out[pidx(a.lmax, le + 1, p.m)] =
                    make_double2(o[2 * u] * i8_pow2(eao + cr), o[2 * u + 1] * i8_pow2(eao + ci));
        }
    }
};

// the 10 MMAs of one parity and one K step: A digit planes 4 KB apart
// (descriptor in the TMA layout), B digit planes `bplane` bytes apart.  The
// descriptors differ only in their start-address field (address / 16 in the
// low 14 bits, which no addition here carries out of), so they are formed
// once and advanced by adds, and all 10 MMAs go out in one asm block with the
// accumulate predicate set once: the single issuing thread spent ~0.7 us per
// chunk building descriptors MMA by MMA.
template <int NC>
__device__ __forceinline__ void i8_issue(uint32_t a_addr, uint32_t b_addr, uint32_t bplane, uint32_t tacc, bool first) {
    constexpr uint32_t idesc = idesc_s8(li8::M, NC);
    const uint64_t da = sdesc2(a_addr, 2048u, 128u);
    const uint64_t db = sdesc2(b_addr, (uint32_t)NC * 16u, 128u);
    const uint64_t ps = 4096u >> 4, pt = (uint64_t)(bplane >> 4);
    // (g, s, t) in issue order: g = s + t < 4
    asm volatile(
        "{\n\t.reg .pred pf, pa;\n\t"
        "setp.ne.b32 pf, %12, 0;\n\t"
        "setp.eq.b32 pa, %12, %12;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %4, %8, %13, pf;\n\t"   // g0: s0 t0
        "tcgen05.mma.cta_group::1.kind::i8 [%1], %4, %9, %13, pf;\n\t"   // g1: s0 t1
        "tcgen05.mma.cta_group::1.kind::i8 [%1], %5, %8, %13, pa;\n\t"   // g1: s1 t0
        "tcgen05.mma.cta_group::1.kind::i8 [%2], %4, %10, %13, pf;\n\t"  // g2: s0 t2
        "tcgen05.mma.cta_group::1.kind::i8 [%2], %5, %9, %13, pa;\n\t"   // g2: s1 t1
        "tcgen05.mma.cta_group::1.kind::i8 [%2], %6, %8, %13, pa;\n\t"   // g2: s2 t0
        "tcgen05.mma.cta_group::1.kind::i8 [%3], %4, %11, %13, pf;\n\t"  // g3: s0 t3
        "tcgen05.mma.cta_group::1.kind::i8 [%3], %5, %10, %13, pa;\n\t"  // g3: s1 t2
        "tcgen05.mma.cta_group::1.kind::i8 [%3], %6, %9, %13, pa;\n\t"   // g3: s2 t1
        "tcgen05.mma.cta_group::1.kind::i8 [%3], %7, %8, %13, pa;\n\t"   // g3: s3 t0
        "}\n" ::"r"(tacc), "r"(tacc + (uint32_t)NC), "r"(tacc + 2u * NC), "r"(tacc + 3u * NC),
        "l"(da), "l"(da + ps), "l"(da + 2 * ps), "l"(da + 3 * ps),
        "l"(db), "l"(db + pt), "l"(db + 2 * pt), "l"(db + 3 * pt),
        "r"(first ? 0u : 1u), "r"(idesc));
}

// 4 groups x 8 int32 columns of one parity at TMEM address ta (groups NC apart),
// converted to the 8 combined FP64 values (((G0 + G1 2^-8) + G2 2^-16) + G3 2^-24)
template <int NC>
__device__ __forceinline__ void i8_ld_combine(uint32_t ta, double* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%32];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%33];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16,%17,%18,%19,%20,%21,%22,%23}, [%34];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%24,%25,%26,%27,%28,%29,%30,%31}, [%35];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(ta), "r"(ta + (uint32_t)NC), "r"(ta + 2u * NC), "r"(ta + 3u * NC)
        : "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) {
        double x = (double)(int)r[i];
        x = fma((double)(int)r[8 + i], 0x1p-8, x);
        x = fma((double)(int)r[16 + i], 0x1p-16, x);
        v[i] = fma((double)(int)r[24 + i], 0x1p-24, x);
    }
}

template <class Dir, int NC>
__global__ void __launch_bounds__(li8::NT, 1) k_legendre_i8(const __grid_constant__ CUtensorMap map, I8Args a,
                                                             const double2* __restrict__ in, double2* __restrict__ out) {
    constexpr int TCOLS = 2 * li8::NG * NC;                  // tensor-memory columns per tile
    constexpr int NACC = TCOLS <= 256 ? 2 : 1;               // tiles in flight in tensor memory
    constexpr uint32_t NCOLS = (uint32_t)(NACC * TCOLS) <= 256u ? 256u : 512u;
    constexpr int KSEG = Dir::KSEG, ZSEG = Dir::ZSEG, CPS = KSEG / li8::KC;  // chunks per segment
    static_assert(KSEG % li8::KC == 0 && NC % 16 == 0 && NC <= 64, "tile shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned long long* colmax = reinterpret_cast<unsigned long long*>(smem + li8::OFF_MAX);
    int* exps = reinterpret_cast<int*>(smem + li8::OFF_EXP);  // [2][64]
    double2* scl = reinterpret_cast<double2*>(smem + li8::OFF_SCL);
    unsigned long long* afull = reinterpret_cast<unsigned long long*>(smem + li8::OFF_BAR);
    unsigned long long* aempty = afull + li8::NSTAGE;
    unsigned long long* bfull = aempty + li8::NSTAGE;   // [2]
    unsigned long long* bempty = bfull + 2;             // [2]
    unsigned long long* accfull = bempty + 2;           // [NACC]
    unsigned long long* accempty = accfull + 2;         // [NACC]
    unsigned long long* expempty = accempty + 2;        // [2] column exponents of a tile read
    unsigned long long* expfull = expempty + 2;         // [2] column exponents of a tile written
    volatile int* abort = reinterpret_cast<volatile int*>(expfull + 2);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(expfull + 2) + 1;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    const I8Tile first = i8_tile<Dir>(a, blockIdx.x);
    if (first.t >= a.ntiles) return;

    if (warp == 0) tmem_alloc(smem_u32(tslot), NCOLS);
    if (tid == 0) {
        for (int i = 0; i < li8::NSTAGE; i++) {
            mbar_init(smem_u32(&afull[i]), 1);
            mbar_init(smem_u32(&aempty[i]), 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(smem_u32(&bfull[i]), 1);
            mbar_init(smem_u32(&bempty[i]), 1);
            mbar_init(smem_u32(&accfull[i]), 1);
            mbar_init(smem_u32(&accempty[i]), li8::NCONS);
            mbar_init(smem_u32(&expempty[i]), li8::NCONS);
            mbar_init(smem_u32(&expfull[i]), 1);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    int issued = -1;  // last chunk whose MMAs were issued (MMA thread)
    int loaded = 0;   // A chunk loads issued (TMA thread)

    if (tid < li8::NPROD) {
        // ---------------------------------------------------------------- producers: B digits
        int j = 0, g = 0;  // tile and segment counters
        bool ok = true;
        for (I8Tile p = first; p.t < a.ntiles && ok; p = i8_tile<Dir>(a, p.t + gridDim.x), j++) {
            if (tid < 64) colmax[tid] = 0ull;
            producers_sync_s();
            const int ns = Dir::tasks(2 * p.nch), trips = i8_trips(ns);
            for (int it = 0; it < trips; it++) {
                const int task = tid + it * li8::NPROD;
                Dir::scan(a, p, task, task < ns, in, colmax);
            }
            // the exponent slot of this tile is free once the consumers have read tile j - 2's
            bool v = true;
            if (tid == 0 && j >= 2)
                v = mbar_wait_abort(smem_u32(&expempty[j & 1]), (uint32_t)(((j >> 1) - 1) & 1), abort);
            if (!producers_and_s(v)) {  // also publishes the column maxima
                ok = false;
                break;
            }
            if (tid < NC) {
                const int e = i8_exp(__longlong_as_double((long long)colmax[tid]));
                exps[(j & 1) * 64 + tid] = e;
                scl[tid] = i8_scale(e);
            }
            producers_sync_s();
            if (tid == 0) mbar_arrive(smem_u32(&expfull[j & 1]));
            const int nseg = (p.nch + CPS - 1) / CPS;
            for (int sg = 0; sg < nseg; sg++, g++) {
                const int slot = g & 1;
                v = true;
                if (tid == 0 && g >= 2)
                    v = mbar_wait_abort(smem_u32(&bempty[slot]), (uint32_t)(((g >> 1) - 1) & 1), abort);
                if (!producers_and_s(v)) {
                    ok = false;
                    break;
                }
                const int z0 = sg * ZSEG, nz = min(ZSEG, 2 * p.nch - z0);
                unsigned char* Bs = smem + li8::OFF_B + slot * li8::B_SLOT;
                const int nt = Dir::tasks(nz);
                auto put = [Bs](int par, int zl, int c, int q, const uint32_t* o) {
                    i8_put<NC, ZSEG>(Bs, par, zl, c, q, o);
                };
                for (int task = tid; task < nt; task += li8::NPROD) Dir::digits(a, p, task, z0, in, scl, put);
                fence_async_smem();
                producers_sync_s();
                if (tid == 0) mbar_arrive(smem_u32(&bfull[slot]));
            }
        }
    } else if (warp == li8::TMA_WARP) {
        // ---------------------------------------------------------------- A loads
        if (lane == 0) {
            int q = 0;
            bool ok = true;
            for (I8Tile p = first; p.t < a.ntiles && ok; p = i8_tile<Dir>(a, p.t + gridDim.x)) {
                for (int kc = 0; kc < p.nch; kc++, q++) {
                    const int s = q % li8::NSTAGE;
                    if (q >= li8::NSTAGE &&
                        !mbar_wait_abort(smem_u32(&aempty[s]), (uint32_t)((q / li8::NSTAGE - 1) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    const uint32_t tb = smem_u32(&afull[s]);
                    mbar_expect_tx(tb, (uint32_t)li8::A_STAGE);
#pragma unroll
                    for (int par = 0; par < 2; par++) {
                        const int3 o = Dir::box(a, p, kc, par);
                        tma_load_4d(smem_u32(smem + s * li8::A_STAGE + par * li8::A_PAR), &map, o.x, o.y, o.z, 0, tb);
                    }
                    loaded = q + 1;
                }
            }
        }
        __syncwarp();
    } else if (warp == li8::MMA_WARP) {
        // ---------------------------------------------------------------- MMAs
        if (lane == 0) {
            int q = 0, g = 0, j = 0;
            bool ok = true;
            for (I8Tile p = first; p.t < a.ntiles && ok; p = i8_tile<Dir>(a, p.t + gridDim.x), j++) {
                const int b = j % NACC;
                if (j >= NACC &&
                    !mbar_wait_abort(smem_u32(&accempty[b]), (uint32_t)((j / NACC - 1) & 1), abort)) {
                    ok = false;
                    break;
                }
                const uint32_t tacc = tmem + (uint32_t)(b * TCOLS);
                for (int kc = 0; kc < p.nch && ok; kc++, q++) {
                    const int kcs = kc % CPS, slot = g & 1;
                    if (kcs == 0 && !mbar_wait_abort(smem_u32(&bfull[slot]), (uint32_t)((g >> 1) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    const int s = q % li8::NSTAGE;
                    if (!mbar_wait_abort(smem_u32(&afull[s]), (uint32_t)((q / li8::NSTAGE) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t As = smem_u32(smem + s * li8::A_STAGE);
                    const uint32_t Bs = smem_u32(smem + li8::OFF_B + slot * li8::B_SLOT);
                    constexpr uint32_t bplane = (uint32_t)ZSEG * NC * 16u;
#pragma unroll
                    for (int par = 0; par < 2; par++)
                        i8_issue<NC>(As + par * li8::A_PAR, Bs + (uint32_t)(par * li8::ND) * bplane + kcs * 2u * NC * 16u,
                                     bplane, tacc + (uint32_t)(par * li8::NG * NC), kc == 0);
                    mma_commit(smem_u32(&aempty[s]));
                    issued = q;
                    if (kcs == CPS - 1 || kc == p.nch - 1) {
                        mma_commit(smem_u32(&bempty[slot]));
                        g++;
                    }
                    if (kc == p.nch - 1) mma_commit(smem_u32(&accfull[b]));
                }
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- consumers
        const int qd = warp - li8::NPROD / 32;  // lane quadrant
        const int r = qd * 32 + lane;
        int j = 0;
        for (I8Tile p = first; p.t < a.ntiles; p = i8_tile<Dir>(a, p.t + gridDim.x), j++) {
            const int b = j % NACC;
            bool v = mbar_wait_abort(smem_u32(&accfull[b]), (uint32_t)((j / NACC) & 1), abort);
            v = v && mbar_wait_abort(smem_u32(&expfull[j & 1]), (uint32_t)((j >> 1) & 1), abort);
            if (!__all_sync(0xffffffffu, v)) break;
            tc_fence_after();
            int ecol[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) ecol[c] = exps[(j & 1) * 64 + c];
            mbar_arrive(smem_u32(&expempty[j & 1]));
            const uint32_t base = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(b * TCOLS);
            int er[2];
            Dir::row_exp(a, p, r, er);
#pragma unroll
            for (int c0 = 0; c0 < NC; c0 += 8) {
                double e[8], o[8];
                i8_ld_combine<NC>(base + (uint32_t)c0, e);
                i8_ld_combine<NC>(base + (uint32_t)(li8::NG * NC + c0), o);
                Dir::epilogue(a, p, r, c0, er, ecol + c0, e, o, out);
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&accempty[b]));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort) {
        if (tid == li8::MMA_WARP * 32) {
            // let the last issued chunk finish before its tensor memory is freed
            if (issued >= 0) {
                const uint32_t bar = smem_u32(&aempty[issued % li8::NSTAGE]);
                const uint32_t ph = (uint32_t)((issued / li8::NSTAGE) & 1);
                const uint64_t t0 = globaltimer();
                while (!mbar_try(bar, ph) && globaltimer() - t0 < tc::WAIT_NS) {
                }
            }
            atomicOr(a.flag, 1);
        }
        if (tid == li8::TMA_WARP * 32) {
            // the A loads still in flight land before the CTA's shared memory is released
            for (int c = loaded - 1; c >= 0 && c >= loaded - li8::NSTAGE; c--) {
                const uint32_t bar = smem_u32(&afull[c % li8::NSTAGE]);
                const uint32_t ph = (uint32_t)((c / li8::NSTAGE) & 1);
                const uint64_t t0 = globaltimer();
                while (!mbar_try(bar, ph) && globaltimer() - t0 < tc::WAIT_NS) {
                }
            }
        }
        __syncthreads();
    }
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, NCOLS);
    }
}

// ------------------------------------------------------------------ tables
// The FP64 recurrence of the P table (same steps and scaling) for one thread
// (northern latitude j, order m), calling put(l, value) for l = m..T.
template <class Put>
__device__ __forceinline__ void i8_recurrence(double z, int m, int T, Put&& put) {
    const double sn = sqrt((1.0 - z) * (1.0 + z));
    const double BIG = 0x1p600, SMALL = 0x1p-600;
    double pmm = sqrt(1.0 / (4.0 * kPi));
    int e = 0;
    for (int k = 1; k <= m; k++) {
        pmm *= -sqrt((2.0 * k + 1.0) / (2.0 * k)) * sn;
        if (fabs(pmm) < SMALL && pmm != 0.0) {
            pmm *= BIG;
            e -= 600;
        }
    }
    double p0 = pmm;
    int el = e;
    put(m, ldexp(p0, el));
    if (m + 1 > T) return;
    double p1 = z * sqrt(2.0 * m + 3.0) * p0;
    put(m + 1, ldexp(p1, el));
    for (int l = m + 2; l <= T; l++) {
        const double ll = l, mm_ = m;
        const double ca = sqrt((4.0 * ll * ll - 1.0) / (ll * ll - mm_ * mm_));
        const double cb = sqrt(((ll - 1.0) * (ll - 1.0) - mm_ * mm_) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0));
        const double p2 = ca * (z * p1 - cb * p0);
        p0 = p1;
        p1 = p2;
        if (el < 0 && fabs(p1) > BIG) {
            p0 *= SMALL;
            p1 *= SMALL;
            el += 600;
        }
        put(l, ldexp(p1, el));
    }
}

// row maxima: synthesis row (m, j) over all degrees -> esy (null: skipped);
// analysis row (m, l) over the latitudes of |P w| -> amax (bit patterns, atomic max)
__global__ void k_i8_rowmax(int nh, int T, int mm, const double* __restrict__ x, const double* __restrict__ w,
                            int* __restrict__ esy, unsigned long long* __restrict__ amax) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, m = blockIdx.y;
    if (j >= nh || m > mm) return;
    const double wj = w[j];
    double smax = 0.0;
    i8_recurrence(x[j], m, T, [&](int l, double v) {
        smax = fmax(smax, fabs(v));
        atomicMax(&amax[pidx(T, l, m)], i8_bits(fabs(v * wj)));
    });
    if (esy) esy[(long long)m * nh + j] = i8_exp(smax);
}

__global__ void k_i8_anexp(long long n, const unsigned long long* __restrict__ amax, int* __restrict__ ean) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ean[i] = i8_exp(__longlong_as_double((long long)amax[i]));
}

// digit words of P (synthesis rows, skipped when SY is null) and P w (analysis
// rows) into the two tables
__global__ void k_i8_tables(int nh, int nhP, int T, int mm, const double* __restrict__ x, const double* __restrict__ w,
                            const int* __restrict__ esy, const int* __restrict__ ean,
                            const long long* __restrict__ zoff, const long long* __restrict__ aoff, long long zS,
                            long long rowsA, int zA, unsigned char* __restrict__ SY, unsigned char* __restrict__ AN) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, m = blockIdx.y;
    if (j >= nh || m > mm) return;
    const double wj = w[j];
    const int es = esy[(long long)m * nh + j];
    const long long plS = zS * nhP * 16, plA = (long long)zA * rowsA * 16;  // bytes per digit plane
    const long long s0 = zoff[m], a0 = aoff[m], a1 = a0 + tcs_pad64(i8_nlp(T, m, 0));
    const int nchm = i8_nch(T, m);
    i8_recurrence(x[j], m, T, [&](int l, double v) {
        const int d = l - m, par = d & 1, lp = d >> 1;
        const uint32_t ws = (uint32_t)(__double2int_rn(ldexp(v, 31 - es)) + 0x808080) ^ 0x808080u;
        const uint32_t wa =
            (uint32_t)(__double2int_rn(ldexp(v * wj, 31 - ean[pidx(T, l, m)])) + 0x808080) ^ 0x808080u;
        const long long is = ((s0 + (long long)par * 2 * nchm + (lp >> 4)) * nhP + j) * 16 + (lp & 15);
        const long long ia = ((long long)(j >> 4) * rowsA + (par ? a1 : a0) + lp) * 16 + (j & 15);
#pragma unroll
        for (int dp = 0; dp < 4; dp++) {
            if (SY) SY[dp * plS + is] = (unsigned char)(ws >> (24 - 8 * dp));
            AN[dp * plA + ia] = (unsigned char)(wa >> (24 - 8 * dp));
        }
    });
}
