// Legendre stage on tcgen05 kind::i8 with both operands moved by the TMA unit.
//
// Included by legendre_tc.cu after legendre_i8.cuh, whose integer split, P
// digit tables and tile epilogues it shares.  The B operand (spectra for the
// synthesis, north +/- south Fourier sums for the analysis) is turned into
// balanced int8 digit planes once per call by a preparation kernel, one CTA
// per (order m, column tile): a first pass takes every column's maximum over
// the whole K range of the order, a second writes the digits, chunk by chunk,
// in the tensor core's K-major no-swizzle layout and the column exponents
// beside them.  Each chunk's B stage is then one contiguous bulk copy:
//
//   chunk (ct, m, kc) = [parity][digit plane][2 groups of 16 K][NC][16 B]
//   synthesis  K = degrees l = m + 2 (32 kc + k) + parity, chunks of order m
//              at i8b_syn_coff(lmax, m) within the column tile
//   analysis   K = latitudes j = 32 kc + k, parity 0 north + south, 1 north -
//              south; chunks of order m at m * nchA
//
// The main kernel has no per-chunk work besides the MMAs: warp 0 issues the
// loads (A by the 4-D tensor map of the digit tables, B by one bulk copy into
// the same stage), warp 1 the 10 digit-product MMAs per parity, and 16
// consumer warps (four per tensor-memory lane quadrant, a quarter of the
// columns each) combine the four exact int32 group sums of a finished tile in
// FP64 and write it: the stores of a tile, not the MMAs, pace the kernel, so
// they are spread over as many warps as possible.  Every wait is bounded as in the other tensor-core kernels.

// bytes of one B chunk of nc columns
__host__ __device__ constexpr int i8b_chunk(int nc) { return 2 * li8::ND * 2 * nc * 16; }

namespace li8b {
constexpr int A_STAGE = li8::A_STAGE;  // 32 KB: both parities' A of a chunk
constexpr int SMEM_MAX = 227 * 1024;
// A load takes ~2 us to land under full load, so the ring holds as many
// stages (A + B of one chunk) as the shared memory allows: 6, 5 or 4 at 16,
// 32 or 64 columns
template <int NC>
constexpr int stage() { return A_STAGE + i8b_chunk(NC); }
template <int NC>
constexpr int nstage() { return (SMEM_MAX - 256) / stage<NC>(); }
template <int NC>
constexpr int off_bar() { return nstage<NC>() * stage<NC>(); }
template <int NC>
constexpr int bytes() { return off_bar<NC>() + 256; }
constexpr int MAXSTAGE = 8;
constexpr int NCONS = 512;  // 16 consumer warps: 4 per tensor-memory lane quadrant
constexpr int CONS_WARP0 = 2;
constexpr int NT = 64 + NCONS;
constexpr int PREP_NT = 256;
static_assert(stage<16>() % 1024 == 0 && stage<32>() % 1024 == 0 && stage<64>() % 1024 == 0, "stage alignment");
static_assert(nstage<16>() <= MAXSTAGE && nstage<64>() >= 4, "stage count");
}  // namespace li8b

// ------------------------------------------------------------------ B preparation
// CTA per (order m = blockIdx.x, column tile ct = blockIdx.y).  Dir is SynI8 or
// AnaI8: their scan / digits are the producer passes of the kernel that stages
// B itself, here over the whole K range of the order at once (a first pass
// takes the column maxima, a second re-reads the values, mostly from L1/L2,
// and writes the digits).  Small CTAs of 64 registers a thread keep several
// per SM; tasks that kept their values in registers between the passes, with
// 16-byte digit rows, measured slower (their larger CTAs fit once per SM).
template <class Dir, int NC>
__global__ void __launch_bounds__(li8b::PREP_NT) k_i8b_prep(I8Args a, const double2* __restrict__ in) {
    __shared__ unsigned long long cmax[NC];
    __shared__ double2 scl[NC];
    I8Tile p;
    p.t = 0;
    p.m = blockIdx.x;
    p.ct = blockIdx.y;
    p.rt = 0;
    p.nch = Dir::prep_nch(a, p.m);
    if (threadIdx.x < NC) cmax[threadIdx.x] = 0ull;
    __syncthreads();
    const int ns = Dir::tasks(2 * p.nch);
    // the same trip count on every thread: the maxima are reduced with warp shuffles
    const int trips = (ns + li8b::PREP_NT - 1) / li8b::PREP_NT;
    for (int it = 0; it < trips; it++) {
        const int task = threadIdx.x + it * li8b::PREP_NT;
        Dir::scan(a, p, task, task < ns, in, cmax);
    }
    __syncthreads();
    if (threadIdx.x < NC) {
        const int e = i8_exp(__longlong_as_double((long long)cmax[threadIdx.x]));
        a.ecol[((long long)p.ct * a.nm + p.m) * NC + threadIdx.x] = e;
        scl[threadIdx.x] = i8_scale(e);
    }
    __syncthreads();
    unsigned char* out = a.B + ((long long)p.ct * a.cpt + Dir::prep_coff(a, p.m)) * i8b_chunk(NC);
    auto put = [out](int par, int zl, int c, int q, const uint32_t* o) {
        unsigned char* ch = out + (long long)(zl >> 1) * i8b_chunk(NC);
#pragma unroll
        for (int d = 0; d < li8::ND; d++)
            *reinterpret_cast<uint32_t*>(ch + (((par * li8::ND + d) * 2 + (zl & 1)) * NC + c) * 16 + 4 * q) = o[d];
    };
    for (int task = threadIdx.x; task < ns; task += li8b::PREP_NT) Dir::digits(a, p, task, 0, in, scl, put);
}

// ------------------------------------------------------------------ main kernel
template <class Dir, int NC>
__global__ void __launch_bounds__(li8b::NT, 1) k_legendre_i8b(const __grid_constant__ CUtensorMap map, I8Args a,
                                                              double2* __restrict__ out) {
    constexpr int TCOLS = 2 * li8::NG * NC;                  // tensor-memory columns per tile
    constexpr int NACC = TCOLS <= 256 ? 2 : 1;               // tiles in flight in tensor memory
    constexpr uint32_t NCOLS = (uint32_t)(NACC * TCOLS) <= 256u ? 256u : 512u;
    constexpr int BCH = i8b_chunk(NC);
    constexpr int PART = NC >= 32 ? NC / 4 : NC / 2;  // columns per consumer warp (multiples of 8)
    constexpr int NPART = NC / PART;
    constexpr int NSTAGE = li8b::nstage<NC>(), STAGE = li8b::stage<NC>();
    static_assert(NC % 16 == 0 && NC <= 64, "tile shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned long long* full = reinterpret_cast<unsigned long long*>(smem + li8b::off_bar<NC>());
    unsigned long long* empty = full + NSTAGE;
    unsigned long long* accfull = empty + NSTAGE;  // [NACC]
    unsigned long long* accempty = accfull + 2;           // [NACC]
    volatile int* abort = reinterpret_cast<volatile int*>(accempty + 2);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(accempty + 2) + 1;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    const I8Tile first = i8_tile<Dir>(a, blockIdx.x);
    if (first.t >= a.ntiles) return;

    if (warp == 0) tmem_alloc(smem_u32(tslot), NCOLS);
    if (tid == 32) {
        for (int i = 0; i < NSTAGE; i++) {
            mbar_init(smem_u32(&full[i]), 1);
            mbar_init(smem_u32(&empty[i]), 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(smem_u32(&accfull[i]), 1);
            mbar_init(smem_u32(&accempty[i]), li8b::NCONS);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    int issued = -1;  // last chunk whose MMAs were issued (MMA thread)
    int loaded = 0;   // chunk loads issued (load thread)

    if (warp == 0) {
        // ---------------------------------------------------------------- loads
        if (lane == 0) {
            int q = 0;
            bool ok = true;
            for (I8Tile p = first; p.t < a.ntiles && ok; p = i8_tile<Dir>(a, p.t + gridDim.x)) {
                const unsigned char* bsrc = a.B + ((long long)p.ct * a.cpt + Dir::prep_coff(a, p.m)) * BCH;
                for (int kc = 0; kc < p.nch; kc++, q++) {
                    const int s = q % NSTAGE;
                    if (q >= NSTAGE &&
                        !mbar_wait_abort(smem_u32(&empty[s]), (uint32_t)((q / NSTAGE - 1) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&full[s]);
                    unsigned char* st = smem + s * STAGE;
                    mbar_expect_tx(fb, (uint32_t)(li8::A_STAGE + BCH));
#pragma unroll
                    for (int par = 0; par < 2; par++) {
                        const int3 o = Dir::box(a, p, kc, par);
                        tma_load_4d(smem_u32(st + par * li8::A_PAR), &map, o.x, o.y, o.z, 0, fb);
                    }
                    bulk_load(smem_u32(st + li8b::A_STAGE), bsrc + (long long)kc * BCH, (uint32_t)BCH, fb);
                    loaded = q + 1;
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------------------------------------------------------- MMAs
        if (lane == 0) {
            int q = 0, j = 0;
            bool ok = true;
            for (I8Tile p = first; p.t < a.ntiles && ok; p = i8_tile<Dir>(a, p.t + gridDim.x), j++) {
                const int b = j % NACC;
                if (j >= NACC &&
                    !mbar_wait_abort(smem_u32(&accempty[b]), (uint32_t)((j / NACC - 1) & 1), abort)) {
                    ok = false;
                    break;
                }
                const uint32_t tacc = tmem + (uint32_t)(b * TCOLS);
                for (int kc = 0; kc < p.nch; kc++, q++) {
                    const int s = q % NSTAGE;
                    if (!mbar_wait_abort(smem_u32(&full[s]), (uint32_t)((q / NSTAGE) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t As = smem_u32(smem + s * STAGE);
                    const uint32_t Bs = As + (uint32_t)li8b::A_STAGE;
                    constexpr uint32_t bplane = 2u * NC * 16u;
#pragma unroll
                    for (int par = 0; par < 2; par++)
                        i8_issue<NC>(As + par * li8::A_PAR, Bs + (uint32_t)(par * li8::ND) * bplane, bplane,
                                     tacc + (uint32_t)(par * li8::NG * NC), kc == 0);
                    mma_commit(smem_u32(&empty[s]));
                    issued = q;
                }
                if (ok) mma_commit(smem_u32(&accfull[b]));
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- consumers
        // a warp reads the tensor-memory lane quadrant warp % 4 (the only one
        // tcgen05.ld lets it access); warps 2-5 take the first part of the
        // columns, warps 6-9 the second, ...; with fewer parts than warp sets
        // (16 columns) the last sets only release the accumulator
        const int cw = warp - li8b::CONS_WARP0;
        const int qd = warp & 3, half = cw >> 2;
        const bool active = half < NPART;
        const int r = qd * 32 + lane;
        int j = 0;
        for (I8Tile p = first; p.t < a.ntiles; p = i8_tile<Dir>(a, p.t + gridDim.x), j++) {
            const int b = j % NACC;
            // row and column exponents of this thread's outputs: loaded before the
            // wait, so their latency overlaps the tile's MMAs
            int er[2], ec[PART];
            Dir::row_exp(a, p, r, er);
            const int* ecol = a.ecol + ((long long)p.ct * a.nm + p.m) * NC + (active ? half : 0) * PART;
#pragma unroll
            for (int c = 0; c < PART; c++) ec[c] = __ldg(ecol + c);
            const bool v = mbar_wait_abort(smem_u32(&accfull[b]), (uint32_t)((j / NACC) & 1), abort);
            if (!__all_sync(0xffffffffu, v)) break;
            tc_fence_after();
            const uint32_t base = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(b * TCOLS);
            if (active) {
#pragma unroll
                for (int cb = 0; cb < PART; cb += 8) {
                    const int c0 = half * PART + cb;
                    double e[8], o[8];
                    i8_ld_combine<NC>(base + (uint32_t)c0, e);
                    i8_ld_combine<NC>(base + (uint32_t)(li8::NG * NC + c0), o);
                    Dir::epilogue(a, p, r, c0, er, ec + cb, e, o, out);
                }
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&accempty[b]));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort) {
        if (tid == 32) {
            // let the last issued chunk finish before its tensor memory is freed
            if (issued >= 0) {
                const uint32_t bar = smem_u32(&empty[issued % NSTAGE]);
                const uint32_t ph = (uint32_t)((issued / NSTAGE) & 1);
                const uint64_t t0 = globaltimer();
                while (!mbar_try(bar, ph) && globaltimer() - t0 < tc::WAIT_NS) {
                }
            }
            atomicOr(a.flag, 1);
        }
        if (tid == 0) {
            // the loads still in flight land before the CTA's shared memory is released
            for (int c = loaded - 1; c >= 0 && c >= loaded - NSTAGE; c--) {
                const uint32_t bar = smem_u32(&full[c % NSTAGE]);
                const uint32_t ph = (uint32_t)((c / NSTAGE) & 1);
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
