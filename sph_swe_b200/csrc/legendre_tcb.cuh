// Legendre stage on tcgen05 with both operands moved by the TMA unit.
//
// Included by legendre_tc.cu after legendre_tcs.cuh.  The P operand comes
// from the split-TF32 tables of legendre_tcs.cuh (two 4-D tensor-map boxes
// per chunk); the B operand is split into TF32 hi/lo once per call by a
// bandwidth-bound preparation kernel that writes every chunk's B stage in the
// tensor core's K-major layout, so each chunk's B is one contiguous bulk copy:
//
//   synthesis  B[ct][m][kc] = split spectra of the column tile's fields,
//              degrees l = m + 32 kc + 2 k + parity (k < 16), both parities
//   analysis   B[ct][m][kc] = split w_j (F_north +- F_south), latitudes
//              j = 16 kc + k (even / odd parity)
//
// With no per-chunk work left for the producers, one thread issues all loads
// and 16 consumer warps (four per tensor-memory lane quadrant, a quarter of
// the columns each) fold the FP32 chunk sums into the FP64 running sums.
// Warp 0: loads (thread 0) and tensor-memory allocation; warp 1: MMAs (one
// thread); warps 2-17: consumers.  Every wait is bounded as in the other
// tensor-core kernels.

namespace tsb {
constexpr int NCONS = 512;
constexpr int MMA_WARP = 1;
constexpr int CONS_WARP0 = 2;
constexpr int NT = 576;
constexpr int NSTAGE = 4;
constexpr int STAGE_B = 4 * tc::STAGE_F;  // 48 KB: A (32 KB) then B (up to 16 KB)
constexpr int OFF_BAR = NSTAGE * STAGE_B;
constexpr int BYTES = OFF_BAR + 512;
static_assert(STAGE_B % 1024 == 0 && BYTES <= 227 * 1024, "shared memory plan");
}  // namespace tsb

// bytes of one chunk's B stage with NC columns (4 parts of NC x 16 floats)
__host__ __device__ constexpr int tcb_bbytes(int nc) { return 4 * nc * tc::KC * 4; }

// chunks of order m before m (synthesis, degree lmax): sum_{m' < m} ((lmax - m') / 32 + 1)
__host__ __device__ inline long long tcb_syn_coff(int lmax, int m) {
    auto fs = [](int n) -> long long {  // sum_{x=0..n} floor(x / 32)
        if (n < 0) return 0;
        const long long q = n / 32, r = n % 32;
        return 16 * q * (q - 1) + q * (r + 1);
    };
    return (long long)m + fs(lmax) - fs(lmax - m);
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(mbar)
                 : "memory");
}

struct TbArgs {
    const long long* soff;  // synthesis P table rows of order m
    const long long* aoff;  // analysis P table rows of order m
    const float* B;         // prepared B stages
    int tlmax, lmax, nh, nlat, batch;
    int nct, nrt, ntiles, group, nkA, nm;
    long long csyn;         // synthesis chunks per column tile
    long long ld_spec, ldF;
    int* flag;
};

// ------------------------------------------------------------------ B preparation
// thread per (chunk, element of one part): element e = (k, col) of the
// NC x 16 part; writes the four parts (parity 0 hi, lo, parity 1 hi, lo)
template <int NC>
__global__ void k_tcb_prep_syn(const double2* __restrict__ spec, long long ld_spec, int lmax, int batch,
                               long long csyn, float* __restrict__ B) {
    constexpr int NF = NC / 2, PART = NC * tc::KC;
    const long long chunk = blockIdx.y;  // within the column tile
    const int ct = blockIdx.z;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= PART) return;
    // order m and chunk kc of this chunk index (m ascending): small search over m
    int m = 0;
    {
        int lo = 0, hi = lmax;  // largest m with coff(m) <= chunk
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tcb_syn_coff(lmax, mid) <= chunk) lo = mid;
            else hi = mid - 1;
        }
        m = lo;
    }
    const int kc = (int)(chunk - tcb_syn_coff(lmax, m));
    const int col = e % NC, k = e / NC;
    const int f = ct * NF + (col >> 1), ri = col & 1;
    float* out = B + ((long long)ct * csyn + chunk) * (4 * PART);
    const int o = tile_off(col, k, NC);
#pragma unroll
    for (int par = 0; par < 2; par++) {
        const int l = m + 2 * tc::KC * kc + 2 * k + par;
        double v = 0.0;
        if (l <= lmax && f < batch) {
            const double2 q = spec[(long long)f * ld_spec + pidx(lmax, l, m)];
            v = ri ? q.y : q.x;
        }
        float hi, lo;
        split_tf32(v, hi, lo);
        out[(2 * par) * PART + o] = hi;
        out[(2 * par + 1) * PART + o] = lo;
    }
}

template <int NC>
__global__ void k_tcb_prep_ana(const double2* __restrict__ F, long long ldF, int nlat, int nh, int nm, int nkA,
                               const double* __restrict__ w, int batch, float* __restrict__ B) {
    constexpr int NF = NC / 2, PART = NC * tc::KC;
    const int m = blockIdx.y / nkA, kc = blockIdx.y % nkA;
    const int ct = blockIdx.z;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= PART || m >= nm) return;
    const int col = e % NC, k = e / NC;
    const int f = ct * NF + (col >> 1), ri = col & 1;
    const int j = tc::KC * kc + k;
    double ev = 0.0, od = 0.0;
    if (j < nh && f < batch) {
        const double2* src = F + (long long)f * ldF + (long long)m * nlat;
        const double2 qn = src[j], qs = src[nlat - 1 - j];
        const double n = ri ? qn.y : qn.x, s = ri ? qs.y : qs.x, wj = w[j];
        ev = wj * (n + s);
        od = wj * (n - s);
    }
    float* out = B + (((long long)ct * nm + m) * nkA + kc) * (4 * PART);
    const int o = tile_off(col, k, NC);
    float hi, lo;
    split_tf32(ev, hi, lo);
    out[o] = hi;
    out[PART + o] = lo;
    split_tf32(od, hi, lo);
    out[2 * PART + o] = hi;
    out[3 * PART + o] = lo;
}

// ------------------------------------------------------------------ directions
template <int NC>
struct SynB {
    __device__ static int nchunks(const TbArgs& a, int m, int) { return (a.lmax - m) / (2 * tc::KC) + 1; }
    __device__ static const float* bsrc(const TbArgs& a, const TcPos& p) {
        return a.B + ((long long)p.ct * a.csyn + tcb_syn_coff(a.lmax, p.m) + p.kc) * (tcb_bbytes(NC) / 4);
    }
    __device__ static int3 box(const TbArgs& a, const TcPos& p, int par) {
        const long long z = a.soff[p.m] + (long long)par * 4 * tcs_nchunks(a.tlmax, p.m) + 4 * p.kc;
        return make_int3(0, 2 * p.rt, (int)z);
    }
    __device__ static void epilogue(const TbArgs& a, const TcPos& p, int r, int col, double2* __restrict__ F,
                                    const double* e, const double* o) {
        constexpr int NF = NC / 2;
        const int j = p.rt * tc::M + r;
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
struct AnaB {
    __device__ static int nchunks(const TbArgs& a, int m, int rt) { return m + 2 * tc::M * rt > a.lmax ? 0 : a.nkA; }
    __device__ static const float* bsrc(const TbArgs& a, const TcPos& p) {
        return a.B + (((long long)p.ct * a.nm + p.m) * a.nkA + p.kc) * (tcb_bbytes(NC) / 4);
    }
    __device__ static int3 box(const TbArgs& a, const TcPos& p, int par) {
        const long long y = a.aoff[p.m] + (long long)par * tcs_pad64(tcs_nlp(a.tlmax, p.m, 0)) + tc::M * p.rt;
        return make_int3(0, (int)(y >> 6), 4 * p.kc);
    }
    __device__ static void epilogue(const TbArgs& a, const TcPos& p, int r, int col, double2* __restrict__ spec,
                                    const double* e, const double* o) {
        constexpr int NF = NC / 2;
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

template <class Dir>
__device__ __forceinline__ TcPos tb_tile(const TbArgs& a, int t) {
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
__device__ __forceinline__ TcPos tb_next(const TbArgs& a, TcPos p) {
    if (p.kc + 1 < p.nk) {
        p.kc++;
        return p;
    }
    return tb_tile<Dir>(a, p.t + gridDim.x);
}

// consumer warp: lane quadrant q, columns [c_begin, c_begin + ncols) in blocks of 8
template <class Dir, int NC>
__device__ __forceinline__ void tb_consume(const TbArgs& a, const TcPos& p, uint32_t tmem, int b, int q, int c_begin,
                                           int ncols, bool first, bool last, double2* __restrict__ out) {
    const uint32_t lane = (uint32_t)(q * 32) << 16;
    const uint32_t part = tmem + lane + (uint32_t)(b * 2 * NC);
    const uint32_t sum = tmem + lane + TcCfg<NC>::ACC64;
    const int r = q * 32 + (threadIdx.x & 31);
    for (int c0 = c_begin; c0 < c_begin + ncols; c0 += 8) {
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
            Dir::epilogue(a, p, r, c0, out, se, so);
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
__global__ void __launch_bounds__(tsb::NT, 1) k_legendre_tcb(const __grid_constant__ CUtensorMap map, TbArgs a,
                                                              double2* __restrict__ out) {
    constexpr int NACC = TcCfg<NC>::NACC;
    constexpr uint32_t NCOLS = TcCfg<NC>::NCOLS;
    constexpr uint32_t BB = (uint32_t)tcb_bbytes(NC);
    extern __shared__ __align__(1024) unsigned char smem[];
    float* stages = reinterpret_cast<float*>(smem);
    unsigned long long* empty = reinterpret_cast<unsigned long long*>(smem + tsb::OFF_BAR);  // [NSTAGE]
    unsigned long long* full = empty + tsb::NSTAGE;                                           // [NSTAGE] A and B landed
    unsigned long long* accfull = full + tsb::NSTAGE;                                         // [NACC]
    unsigned long long* accempty = accfull + NACC;                                            // [NACC]
    volatile int* abort = reinterpret_cast<volatile int*>(accempty + NACC);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(accempty + NACC) + 1;
    const int tid = threadIdx.x, warp = tid >> 5;

    const TcPos first = tb_tile<Dir>(a, blockIdx.x);
    if (first.t >= a.ntiles) return;

    if (warp == 0) tmem_alloc(smem_u32(tslot), NCOLS);
    if (tid == 0) {
        for (int i = 0; i < tsb::NSTAGE; i++) {
            mbar_init(smem_u32(&empty[i]), 1);
            mbar_init(smem_u32(&full[i]), 1);
        }
        for (int i = 0; i < NACC; i++) {
            mbar_init(smem_u32(&accfull[i]), 1);
            mbar_init(smem_u32(&accempty[i]), tsb::NCONS);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    int issued = -1;  // last chunk whose MMAs were issued (MMA thread)
    int loaded = 0;   // chunks whose loads were issued (thread 0)

    if (warp == 0) {
        if (tid == 0) {
            TcPos cur = first;
            int q = 0;
            while (cur.t < a.ntiles) {
                const int s = q % tsb::NSTAGE;
                if (q >= tsb::NSTAGE &&
                    !mbar_wait_abort(smem_u32(&empty[s]), (uint32_t)((q / tsb::NSTAGE - 1) & 1), abort))
                    break;
                float* As = stages + s * (tsb::STAGE_B / 4);
                float* Bs = As + 4 * tc::ATILE;
                const uint32_t fb = smem_u32(&full[s]);
                mbar_expect_tx(fb, (uint32_t)tss::A_BYTES + BB);
#pragma unroll
                for (int par = 0; par < 2; par++) {
                    const int3 o = Dir::box(a, cur, par);
                    tma_load_4d(smem_u32(As + par * 2 * tc::ATILE), &map, o.x, o.y, o.z, 0, fb);
                }
                bulk_load(smem_u32(Bs), Dir::bsrc(a, cur), BB, fb);
                loaded = q + 1;
                q++;
                cur = tb_next<Dir>(a, cur);
            }
        }
        __syncwarp();
    } else if (warp == tsb::MMA_WARP) {
        if ((tid & 31) == 0) {
            TcPos cur = first;
            int q = 0, gq = -1;
            while (cur.t < a.ntiles) {
                const int s = q % tsb::NSTAGE;
                const bool gfirst = cur.kc % a.group == 0;
                const bool glast = cur.kc % a.group == a.group - 1 || cur.kc == cur.nk - 1;
                if (gfirst) gq++;
                const int b = gq % NACC;
                if (!mbar_wait_abort(smem_u32(&full[s]), (uint32_t)((q / tsb::NSTAGE) & 1), abort)) break;
                if (gfirst && gq >= NACC &&
                    !mbar_wait_abort(smem_u32(&accempty[b]), (uint32_t)(((gq - NACC) / NACC) & 1), abort))
                    break;
                tc_fence_after();
                float* As = stages + s * (tsb::STAGE_B / 4);
                tcs_issue_chunk<NC, NC * tc::KC>(As, As + 4 * tc::ATILE, tmem + b * 2 * NC, !gfirst);
                mma_commit(smem_u32(&empty[s]));
                if (glast) mma_commit(smem_u32(&accfull[b]));
                issued = q;
                q++;
                cur = tb_next<Dir>(a, cur);
            }
        }
        __syncwarp();
    } else {
        // consumer warps 2..17: lane quadrant warp % 4, column quarter (warp - 2) / 4
        const int qd = warp & 3, slice = (warp - tsb::CONS_WARP0) >> 2;
        constexpr int PER = NC / 4 >= 8 ? NC / 4 : 8;  // columns per warp, whole blocks of 8
        const int c_begin = slice * PER;
        const int ncols = c_begin < NC ? PER : 0;
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
                tb_consume<Dir, NC>(a, cur, tmem, b, qd, c_begin, ncols, cur.kc < a.group, cur.kc == cur.nk - 1, out);
                tc_fence_before();
                mbar_arrive(smem_u32(&accempty[b]));
            }
            cur = tb_next<Dir>(a, cur);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort) {
        if (tid == tsb::MMA_WARP * 32) {
            if (issued >= 0) {
                const uint32_t bar = smem_u32(&empty[issued % tsb::NSTAGE]);
                const uint32_t ph = (uint32_t)((issued / tsb::NSTAGE) & 1);
                const uint64_t t0 = globaltimer();
                while (!mbar_try(bar, ph) && globaltimer() - t0 < tc::WAIT_NS) {
                }
            }
            atomicOr(a.flag, 1);
        }
        if (tid == 0) {
            // the loads still in flight land before the CTA's shared memory is released
            for (int c = loaded - 1; c >= 0 && c >= loaded - tsb::NSTAGE; c--) {
                const uint32_t bar = smem_u32(&full[c % tsb::NSTAGE]);
                const uint32_t ph = (uint32_t)((c / tsb::NSTAGE) & 1);
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
