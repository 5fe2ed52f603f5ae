// Legendre stage on tcgen05 with the A operand (P_l^m) streamed by TMA.
//
// Included by legendre_tc.cu after its helpers.  The split-TF32 P_l^m of the
// handle are stored once, at set-up, in two tables whose 4-D tensor maps make
// every chunk's A operand (both parities, hi and lo: 32 KB) two TMA box
// loads that land directly in the tensor core's K-major no-swizzle layout:
//
//   synthesis  S[w][z][j][x]  x = l' mod 4, z = zoff(m, parity) + l' / 4
//              (rows = latitudes j, padded to a multiple of 64; K = degrees
//               l = m + 2 l' + parity; each (m, parity) block padded with
//               zeros to whole chunks)
//   analysis   A[w][z][y][x]  x = j mod 4, z = j / 4,
//              y = yoff(m, parity) + l' (rows = degrees, each (m, parity)
//              block padded with zero rows to a multiple of 64; K = latitudes)
//
// with w = 0 hi, 1 lo.  A row is 16 B and 64 rows are 1 KB of contiguous
// memory, so the tensor maps see (64 rows x 4 floats, row block, z, w) and a
// box {256, 2, 4, 2} is 128 rows x 16 K x {hi, lo} with a 1 KB inner extent:
// in shared memory four 2 KB slices of 128 rows x 16 B per part, i.e. core
// matrices 128 B apart along M/N (SBO) and 2 KB apart along K (LBO).  Row
// blocks beyond a table's extent are zero filled by the TMA unit; padded rows
// are zero or land in output rows the epilogue discards.
//
// Per SM one persistent CTA of 17 warps: producers (warps 0-7) stage the
// split B operand from a cp.async prefetch ring, thread 0 also issues the A
// loads of each stage; warp 16 issues the MMAs; consumers (warps 8-15, two per
// tensor-memory lane quadrant, each half of the columns) fold the FP32 group
// sums into FP64 sums in tensor memory and write finished tiles, with one
// tensor-memory load wait per 8 columns.  Every wait is bounded as in the
// generator kernel.

namespace tss {
constexpr int NPROD = 256;                 // producer threads (B staging; thread 0 issues the A loads)
constexpr int NCONS = 256;                 // consumer threads: warp 8 + q + 4 h = lane quadrant q, column half h
constexpr int MMA_WARP = 16;
constexpr int NT = 544;
constexpr int NSTAGE = 3;
constexpr int NRAW = 3;
constexpr int STAGE_B = 4 * tc::STAGE_F;  // 48 KB: A (32 KB) then B (16 KB)
constexpr int A_BYTES = 4 * tc::ATILE * 4;
constexpr int RAW_B = 32 * (32 + 4) * 16 + 16 * 8 + 128;  // B rows, weights, pad to 128 B
constexpr int OFF_RAW = NSTAGE * STAGE_B;
constexpr int OFF_BAR = OFF_RAW + NRAW * RAW_B;
constexpr int BYTES = OFF_BAR + 512;
static_assert(RAW_B % 128 == 0 && STAGE_B % 1024 == 0, "aligned buffers");
}  // namespace tss

// chunks of 16 degrees per parity of order m up to degree T, degrees of one
// parity, and a row count rounded up to whole 64-row blocks
__host__ __device__ inline int tcs_nchunks(int T, int m) { return (T - m) / (2 * tc::KC) + 1; }
__host__ __device__ inline int tcs_nlp(int T, int m, int par) { return T - m - par >= 0 ? (T - m - par) / 2 + 1 : 0; }
__host__ __device__ inline int tcs_pad64(int n) { return (n + 63) & ~63; }

// K-major no-swizzle descriptor with explicit core-matrix strides (bytes)
__device__ __forceinline__ uint64_t sdesc2(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ bool producers_and_s(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 256, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void producers_sync_s() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

struct TsArgs {
    const long long* soff;  // synthesis table: first z row of order m (parity 0; parity 1 follows)
    const long long* aoff;  // analysis table: first row of order m (parity 0; parity 1 follows)
    const double* w;
    int tlmax, lmax, nh, nlat, batch;
    int nct, nrt, ntiles, group;
    long long ld_spec, ldF;
    int* flag;
};

__device__ __forceinline__ double2* raw_b(unsigned char* smem, int buf) {
    return reinterpret_cast<double2*>(smem + tss::OFF_RAW + buf * tss::RAW_B);
}

// item decomposition of the B operand (as the generator kernel's)
template <int NC>
struct SynS {
    static constexpr int NF = NC / 2;
    static constexpr int BIT = NC * 2 * tc::KC / tss::NPROD;
    __device__ static int nchunks(const TsArgs& a, int m, int) { return (a.lmax - m) / (2 * tc::KC) + 1; }
    __device__ static int item_f(int idx) { return ((idx >> 3) & 3) | ((idx >> 7) % (NF / 4)) * 4; }
    __device__ static int item_par(int idx) { return (idx >> 7) / (NF / 4); }

    __device__ static void prefetch(const TsArgs& a, const double2* __restrict__ spec, const TcPos& p,
                                    unsigned char* smem, int buf) {
        const int l0 = p.m + 2 * tc::KC * p.kc;
        double2* b = raw_b(smem, buf);
#pragma unroll
        for (int it = 0; it < NF * 32 / tss::NPROD; it++) {
            const int idx = threadIdx.x + tss::NPROD * it;
            const int d = idx & 31, fl = idx >> 5;
            const int l = l0 + d, f = p.ct * NF + fl;
            const bool v = l <= a.lmax && f < a.batch;
            cp_async(&b[((d & 1) * 16 + (d >> 1)) * (NF + 4) + fl],
                     v ? (const void*)(spec + (long long)f * a.ld_spec + pidx(a.lmax, l, p.m)) : (const void*)spec, 16,
                     v);
        }
    }
    __device__ static void fill_b(const TsArgs&, float* Bs, unsigned char* smem, int buf) {
        const double2* b = raw_b(smem, buf);
#pragma unroll
        for (int it = 0; it < BIT; it++) {
            const int idx = threadIdx.x + tss::NPROD * it;
            const double2 q = b[(item_par(idx) * 16 + item_k(idx)) * (NF + 4) + item_f(idx)];
            float hi, lo;
            split_tf32(item_ri(idx) ? q.y : q.x, hi, lo);
            float* bp = Bs + item_par(idx) * 2 * tc::BTILE + tile_off(2 * item_f(idx) + item_ri(idx), item_k(idx), NC);
            bp[0] = hi;
            bp[tc::BTILE] = lo;
        }
    }
    // TMA box origin (x, row block, z) of parity par's A part
    __device__ static int3 box(const TsArgs& a, const TcPos& p, int par) {
        const long long z = a.soff[p.m] + (long long)par * 4 * tcs_nchunks(a.tlmax, p.m) + 4 * p.kc;
        return make_int3(0, 2 * p.rt, (int)z);
    }
    __device__ static void epilogue(const TsArgs& a, const TcPos& p, int cw, int col, double2* __restrict__ F,
                                    const double* e, const double* o) {
        const int j = p.rt * tc::M + (cw & 3) * 32 + (threadIdx.x & 31);
        if (j >= a.nh) return;
        const int fb = p.ct * NF + col / 2;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int f = fb + u;
            if (f < a.batch) {
                double2* out = F + (long long)f * a.ldF + (long long)p.m * a.nlat;
                out[j] = make_double2(e[2 * u] + o[2 * u], e[2 * u + 1] + o[2 * u + 1]);
                out[a.nlat - 1 - j] = make_double2(e[2 * u] - o[2 * u], e[2 * u + 1] - o[2 * u + 1]);
            }
        }
    }
};

template <int NC>
struct AnaS {
    static constexpr int NF = NC / 2;
    static constexpr int BIT = NC * tc::KC / tss::NPROD;
    __device__ static int nchunks(const TsArgs& a, int m, int rt) {
        return m + 2 * tc::M * rt > a.lmax ? 0 : (a.nh + tc::KC - 1) / tc::KC;
    }
    __device__ static int item_f(int idx) { return ((idx >> 3) & 3) | ((idx >> 7) << 2); }

    __device__ static void prefetch(const TsArgs& a, const double2* __restrict__ F, const TcPos& p, unsigned char* smem,
                                    int buf) {
        double2* b = raw_b(smem, buf);
        const int j0 = p.kc * tc::KC;
#pragma unroll
        for (int it = 0; it < NF * 32 / tss::NPROD; it++) {
            const int idx = threadIdx.x + tss::NPROD * it;
            const int k = idx & 15, hs = (idx >> 4) & 1, fl = idx >> 5;
            const int j = j0 + k, f = p.ct * NF + fl;
            const bool v = j < a.nh && f < a.batch;
            const double2* src = F + (long long)f * a.ldF + (long long)p.m * a.nlat + (hs ? a.nlat - 1 - j : j);
            cp_async(&b[(hs * 16 + k) * (NF + 4) + fl], v ? (const void*)src : (const void*)F, 16, v);
        }
        if (threadIdx.x < tc::KC) {
            double* wr = reinterpret_cast<double*>(b + 32 * (NF + 4));
            const int j = j0 + threadIdx.x;
            cp_async(&wr[threadIdx.x], j < a.nh ? (const void*)(a.w + j) : (const void*)a.w, 8, j < a.nh);
        }
    }
    __device__ static void fill_b(const TsArgs&, float* Bs, unsigned char* smem, int buf) {
        const double2* b = raw_b(smem, buf);
        const int k = item_k(threadIdx.x), ri = item_ri(threadIdx.x);
        const double wj = reinterpret_cast<const double*>(b + 32 * (NF + 4))[k];
#pragma unroll
        for (int it = 0; it < BIT; it++) {
            const int idx = threadIdx.x + tss::NPROD * it;
            const double2 qn = b[k * (NF + 4) + item_f(idx)], qs = b[(16 + k) * (NF + 4) + item_f(idx)];
            const double n = ri ? qn.y : qn.x, sv = ri ? qs.y : qs.x;
            float hi, lo;
            const int o = tile_off(2 * item_f(idx) + ri, k, NC);
            split_tf32(wj * (n + sv), hi, lo);
            Bs[o] = hi;
            Bs[tc::BTILE + o] = lo;
            split_tf32(wj * (n - sv), hi, lo);
            Bs[2 * tc::BTILE + o] = hi;
            Bs[3 * tc::BTILE + o] = lo;
        }
    }
    __device__ static int3 box(const TsArgs& a, const TcPos& p, int par) {
        const long long y = a.aoff[p.m] + (long long)par * tcs_pad64(tcs_nlp(a.tlmax, p.m, 0)) + tc::M * p.rt;
        return make_int3(0, (int)(y >> 6), 4 * p.kc);
    }
    // consumer thread: TMEM lane r = degree index l' = 128 rt + r of both parities
    __device__ static void epilogue(const TsArgs& a, const TcPos& p, int cw, int col, double2* __restrict__ spec,
                                    const double* e, const double* o) {
        const int r = (cw & 3) * 32 + (threadIdx.x & 31);
        const int le = p.m + 2 * (tc::M * p.rt + r);
        const int fb = p.ct * NF + col / 2;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int f = fb + u;
            if (f >= a.batch) continue;
            double2* out = spec + (long long)f * a.ld_spec;
            if (le <= a.lmax) out[pidx(a.lmax, le, p.m)] = make_double2(e[2 * u], e[2 * u + 1]);
            if (le + 1 <= a.lmax) out[pidx(a.lmax, le + 1, p.m)] = make_double2(o[2 * u], o[2 * u + 1]);
        }
    }
};

// the MMAs of one staged chunk: A in the TMA layout, B in the generator kernel's
// layout with its four parts BPART floats apart
template <int NC, int BPART = tc::BTILE>
__device__ __forceinline__ void tcs_issue_chunk(const float* As, const float* Bs, uint32_t tacc, bool acc) {
    constexpr uint32_t idesc = idesc_tf32(tc::M, NC);
    const uint64_t dA = sdesc2(smem_u32(As), 2048u, 128u), dB = sdesc(smem_u32(Bs));
#pragma unroll
    for (int s = 0; s < tc::KC / 8; s++) {
#pragma unroll
        for (int par = 0; par < 2; par++) {
            const uint64_t ah = dA + (uint64_t)((par * 2 * tc::ATILE * 4 + s * 4096) >> 4);
            const uint64_t al = ah + (uint64_t)((tc::ATILE * 4) >> 4);
            const uint64_t bh = dB + (uint64_t)((par * 2 * BPART * 4 + s * NC * 32) >> 4);
            const uint64_t bl = bh + (uint64_t)((BPART * 4) >> 4);
            const uint32_t d = tacc + par * NC;
            mma_tf32(d, ah, bh, idesc, (s > 0 || acc) ? 1u : 0u);
            mma_tf32(d, ah, bl, idesc, 1u);
            mma_tf32(d, al, bh, idesc, 1u);
        }
    }
}

template <class Dir>
__device__ __forceinline__ TcPos ts_tile(const TsArgs& a, int t) {
    TcPos p;
    for (; t < a.ntiles; t += gridDim.x) {
        p.ct = t % a.nct;
        const int rest = t / a.nct;
        p.rt = rest % a.nrt;
        p.m = rest / a.nrt;
        p.nk = Dir::nchunks(a, p.m, p.rt);
        if (p.nk > 0) break;
    }
    p.t = t;
    p.kc = 0;
    return p;
}

template <class Dir>
__device__ __forceinline__ TcPos ts_next(const TsArgs& a, TcPos p) {
    if (p.kc + 1 < p.nk) {
        p.kc++;
        return p;
    }
    return ts_tile<Dir>(a, p.t + gridDim.x);
}

// 8 FP32 columns of E and O and, unless first, their FP64 running sums
// (16 + 16 words), one wait
__device__ __forceinline__ void tmem_ld_block(uint32_t pe, uint32_t po, uint32_t se, uint32_t so, bool first, float* e,
                                              float* o, float* we, float* wo) {
    uint32_t r[48];
    if (first) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%16];\n\t"
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%17];\n\t"
            "tcgen05.wait::ld.sync.aligned;"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(pe), "r"(po)
            : "memory");
    } else {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%48];\n\t"
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%49];\n\t"
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
            "[%50];\n\t"
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47}, "
            "[%51];\n\t"
            "tcgen05.wait::ld.sync.aligned;"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
              "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
              "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
              "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
              "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47])
            : "r"(pe), "r"(po), "r"(se), "r"(so)
            : "memory");
#pragma unroll
        for (int i = 0; i < 16; i++) {
            we[i] = __uint_as_float(r[16 + i]);
            wo[i] = __uint_as_float(r[32 + i]);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        e[i] = __uint_as_float(r[i]);
        o[i] = __uint_as_float(r[8 + i]);
    }
}

// consumer warp cw (0..7): lane quadrant cw & 3, columns of half cw >> 2; fold a
// group's FP32 sums into the FP64 sums, or hand the totals to the epilogue
template <class Dir, int NC>
__device__ __forceinline__ void ts_consume(const TsArgs& a, const TcPos& p, uint32_t tmem, int b, int cw, bool first,
                                           bool last, double2* __restrict__ out) {
    constexpr int HALF = NC / 2;
    const uint32_t lane = (uint32_t)((cw & 3) * 32) << 16;
    const int c_begin = (cw >> 2) * HALF;
    const uint32_t part = tmem + lane + (uint32_t)(b * 2 * NC);
    const uint32_t sum = tmem + lane + TcCfg<NC>::ACC64;
#pragma unroll
    for (int c0 = c_begin; c0 < c_begin + HALF; c0 += 8) {
        float e[8], o[8], we[16], wo[16];
        tmem_ld_block(part + c0, part + NC + c0, sum + 2 * c0, sum + 2 * NC + 2 * c0, first, e, o, we, wo);
        double se[8], so[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            se[i] = (double)e[i];
            so[i] = (double)o[i];
            if (!first) {
                se[i] += __hiloint2double(__float_as_int(we[2 * i + 1]), __float_as_int(we[2 * i]));
                so[i] += __hiloint2double(__float_as_int(wo[2 * i + 1]), __float_as_int(wo[2 * i]));
            }
        }
        if (last) {
            Dir::epilogue(a, p, cw, c0, out, se, so);
        } else {
            uint32_t ve[16], vo[16];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                ve[2 * i] = (uint32_t)__double2loint(se[i]);
                ve[2 * i + 1] = (uint32_t)__double2hiint(se[i]);
                vo[2 * i] = (uint32_t)__double2loint(so[i]);
                vo[2 * i + 1] = (uint32_t)__double2hiint(so[i]);
            }
            tmem_st16(sum + 2 * c0, ve);
            tmem_st16(sum + 2 * NC + 2 * c0, vo);
        }
    }
    if (!last) tmem_wait_st();
}

template <class Dir, int NC>
__global__ void __launch_bounds__(tss::NT, 1) k_legendre_tcs(const __grid_constant__ CUtensorMap map, TsArgs a,
                                                              const double2* __restrict__ in, double2* __restrict__ out) {
    constexpr int NACC = TcCfg<NC>::NACC;
    constexpr uint32_t NCOLS = TcCfg<NC>::NCOLS;
    extern __shared__ __align__(1024) unsigned char smem[];
    float* stages = reinterpret_cast<float*>(smem);
    unsigned long long* empty = reinterpret_cast<unsigned long long*>(smem + tss::OFF_BAR);  // [NSTAGE]
    unsigned long long* full = empty + tss::NSTAGE;                                           // [NSTAGE] B staged
    unsigned long long* tfull = full + tss::NSTAGE;                                           // [NSTAGE] A landed
    unsigned long long* accfull = tfull + tss::NSTAGE;                                        // [NACC]
    unsigned long long* accempty = accfull + NACC;                                            // [NACC]
    volatile int* abort = reinterpret_cast<volatile int*>(accempty + NACC);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(accempty + NACC) + 1;
    const int tid = threadIdx.x, warp = tid >> 5;

    const TcPos first = ts_tile<Dir>(a, blockIdx.x);
    if (first.t >= a.ntiles) return;

    if (warp == 0) tmem_alloc(smem_u32(tslot), NCOLS);
    if (tid == 0) {
        for (int i = 0; i < tss::NSTAGE; i++) {
            mbar_init(smem_u32(&empty[i]), 1);
            mbar_init(smem_u32(&full[i]), 1);
            mbar_init(smem_u32(&tfull[i]), 1);
        }
        for (int i = 0; i < NACC; i++) {
            mbar_init(smem_u32(&accfull[i]), 1);
            mbar_init(smem_u32(&accempty[i]), tss::NCONS);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    int issued = -1;   // last chunk whose MMAs were issued (MMA thread)
    int loaded = 0;    // A loads issued (producer thread 0)

    if (tid < tss::NPROD) {
        TcPos cur = first, pf = first;
#pragma unroll
        for (int i = 0; i < tss::NRAW - 1; i++) {
            if (pf.t < a.ntiles) {
                Dir::prefetch(a, in, pf, smem, i);
                pf = ts_next<Dir>(a, pf);
            }
            cp_async_commit();
        }
        int q = 0;
        while (cur.t < a.ntiles) {
            if (pf.t < a.ntiles) {
                Dir::prefetch(a, in, pf, smem, (q + tss::NRAW - 1) % tss::NRAW);
                pf = ts_next<Dir>(a, pf);
            }
            cp_async_commit();
            const int s = q % tss::NSTAGE;
            float* As = stages + s * (tss::STAGE_B / 4);
            float* Bs = As + 4 * tc::ATILE;
            bool v = true;
            if (tid == 0) {
                if (q >= tss::NSTAGE)
                    v = mbar_wait_abort(smem_u32(&empty[s]), (uint32_t)((q / tss::NSTAGE - 1) & 1), abort);
                if (v) {
                    const uint32_t tb = smem_u32(&tfull[s]);
                    mbar_expect_tx(tb, (uint32_t)tss::A_BYTES);
#pragma unroll
                    for (int par = 0; par < 2; par++) {
                        const int3 o = Dir::box(a, cur, par);
                        tma_load_4d(smem_u32(As + par * 2 * tc::ATILE), &map, o.x, o.y, o.z, 0, tb);
                    }
                    loaded = q + 1;
                }
            }
            cp_async_wait<tss::NRAW - 1>();
            if (!producers_and_s(v)) break;  // also publishes every producer's prefetched data
            Dir::fill_b(a, Bs, smem, q % tss::NRAW);
            fence_async_smem();
            producers_sync_s();
            if (tid == 0) mbar_arrive(smem_u32(&full[s]));
            q++;
            cur = ts_next<Dir>(a, cur);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp == tss::MMA_WARP) {
        if (tid == tss::MMA_WARP * 32) {
            TcPos cur = first;
            int q = 0, gq = -1;
            while (cur.t < a.ntiles) {
                const int s = q % tss::NSTAGE;
                const bool gfirst = cur.kc % a.group == 0;
                const bool glast = cur.kc % a.group == a.group - 1 || cur.kc == cur.nk - 1;
                if (gfirst) gq++;
                const int b = gq % NACC;
                const uint32_t ph = (uint32_t)((q / tss::NSTAGE) & 1);
                if (!mbar_wait_abort(smem_u32(&full[s]), ph, abort)) break;
                if (!mbar_wait_abort(smem_u32(&tfull[s]), ph, abort)) break;
                if (gfirst && gq >= NACC &&
                    !mbar_wait_abort(smem_u32(&accempty[b]), (uint32_t)(((gq - NACC) / NACC) & 1), abort))
                    break;
                tc_fence_after();
                float* As = stages + s * (tss::STAGE_B / 4);
                tcs_issue_chunk<NC>(As, As + 4 * tc::ATILE, tmem + b * 2 * NC, !gfirst);
                mma_commit(smem_u32(&empty[s]));
                if (glast) mma_commit(smem_u32(&accfull[b]));
                issued = q;
                q++;
                cur = ts_next<Dir>(a, cur);
            }
        }
        __syncwarp();
    } else {
        const int cw = warp - tss::NPROD / 32;
        TcPos cur = first;
        int g = -1;
        while (cur.t < a.ntiles) {
            const bool gfirst = cur.kc % a.group == 0;
            const bool glast = cur.kc % a.group == a.group - 1 || cur.kc == cur.nk - 1;
            if (gfirst) g++;
            if (glast) {
                const int b = g % NACC;
                const bool v = mbar_wait_abort(smem_u32(&accfull[b]), (uint32_t)((g / NACC) & 1), abort);
                if (!__all_sync(0xffffffffu, v)) break;
                tc_fence_after();
                ts_consume<Dir, NC>(a, cur, tmem, b, cw, cur.kc < a.group, cur.kc == cur.nk - 1, out);
                tc_fence_before();
                mbar_arrive(smem_u32(&accempty[b]));
            }
            cur = ts_next<Dir>(a, cur);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort) {
        if (tid == tss::MMA_WARP * 32) {
            // let the last issued chunk finish before its tensor memory is freed
            if (issued >= 0) {
                const uint32_t bar = smem_u32(&empty[issued % tss::NSTAGE]);
                const uint32_t ph = (uint32_t)((issued / tss::NSTAGE) & 1);
                const uint64_t t0 = globaltimer();
                while (!mbar_try(bar, ph) && globaltimer() - t0 < tc::WAIT_NS) {
                }
            }
            atomicOr(a.flag, 1);
        }
        if (tid == 0) {
            // the A loads still in flight land before the CTA's shared memory is released
            for (int c = loaded - 1; c >= 0 && c >= loaded - tss::NSTAGE; c--) {
                const uint32_t bar = smem_u32(&tfull[c % tss::NSTAGE]);
                const uint32_t ph = (uint32_t)((c / tss::NSTAGE) & 1);
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
// thread per (northern latitude j, order m): the FP64 recurrence of the P
// table (same steps and scaling), split into TF32 hi/lo, written to both tables
__global__ void k_tcs_tables(int nh, int nhP, int tlmax, int mm, const double* __restrict__ x,
                             const long long* __restrict__ soff, const long long* __restrict__ aoff, long long zS,
                             long long rowsA, int zA, float* __restrict__ S, float* __restrict__ A) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (j >= nh || m > mm) return;
    const double z = x[j];
    const double sn = sqrt((1.0 - z) * (1.0 + z));
    const long long sw = zS * nhP * 4, aw = (long long)zA * rowsA * 4;
    const long long s0 = soff[m], s1 = s0 + 4LL * tcs_nchunks(tlmax, m);
    const long long a0 = aoff[m], a1 = a0 + tcs_pad64(tcs_nlp(tlmax, m, 0));
    auto put = [&](int l, double v) {
        const int d = l - m, par = d & 1, lp = d >> 1;
        float hi, lo;
        split_tf32(v, hi, lo);
        const long long is = (((par ? s1 : s0) + (lp >> 2)) * nhP + j) * 4 + (lp & 3);
        S[is] = hi;
        S[is + sw] = lo;
        const long long ia = (((long long)(j >> 2)) * rowsA + (par ? a1 : a0) + lp) * 4 + (j & 3);
        A[ia] = hi;
        A[ia + aw] = lo;
    };
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
    if (m + 1 > tlmax) return;
    double p1 = z * sqrt(2.0 * m + 3.0) * p0;
    put(m + 1, ldexp(p1, el));
    for (int l = m + 2; l <= tlmax; l++) {
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
