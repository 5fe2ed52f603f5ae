// Legendre stage on the 5th-generation tensor cores (mixed-precision form).
//
// Per zonal wavenumber m the Legendre transforms are dense contractions
//   synthesis  E/O[j][c] = sum_{l' in parity} P[l(l')][j] Q[l'][c]     (rows = latitudes)
//   analysis   Q_p[l'][c] = sum_j P[l(l')][j] G_p[j][c]                 (rows = degrees)
// with columns c = 2 f + (0 re, 1 im) and l = m + 2 l' + p.  Each is run as
// a tcgen05.mma kind::tf32 GEMM in split-TF32 form: every operand x is
// written as hi + lo with hi, lo representable in TF32, and
// hi*hi + hi*lo + lo*hi is accumulated (lo*lo is below 2^-22 relative).
//
// P_l^m is not streamed from a table.  It is regenerated in FP64 on the CUDA
// cores by the three-term recurrence, restarted from checkpoints
// (P_l, P_{l+1}, binary scale) stored every 16 degrees, and split into TF32
// hi/lo directly into the canonical K-major no-swizzle shared-memory layout
// of the tensor core.  HBM traffic is the spectral and Fourier data plus the
// checkpoints (1/8 of a P table).
//
// Precision: the tensor core accumulates a group of K chunks (16 terms per
// parity and chunk) in FP32 starting from zero; each group's accumulator is
// then added into an FP64 running sum kept in tensor memory, so FP32
// rounding acts on short partial sums only.
//
// One persistent CTA of 17 warps per SM walks its tiles as one stream of
// chunks.  Producers (warps 0-11) prefetch a chunk's raw data NRAW-1 chunks
// ahead with cp.async, then warps 0-7 regenerate P and warps 8-11 stage B
// into one of NSTAGE smem stages; one thread of warp 16
// issues each staged chunk's MMAs and commits them; consumers (warps 12-15)
// fold finished groups into the FP64 sums and write finished tiles.  The
// roles are decoupled by mbarriers; all
// waits are bounded: on timeout the CTA raises an abort flag, waits (bounded)
// for its last MMA, records the error in the handle's flag, frees its tensor
// memory and returns.
#include "common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

namespace sphgpu {

namespace tc {
constexpr int M = 128;            // tile rows (TMEM lanes)
constexpr int KC = 16;            // K per chunk and parity (two MMA K-steps of 8)
constexpr int SEG = 16;           // degrees per recurrence checkpoint
constexpr int NGEN = 256;         // producer threads regenerating P (warps 0-7)
constexpr int NBST = 128;         // producer threads staging B (warps 8-11)
constexpr int NPROD = NGEN + NBST;
constexpr int NCONS = 128;        // consumer threads (warps 12-15)
constexpr int MMA_WARP = 16;
constexpr int NT = 544;           // threads per CTA
constexpr int ATILE = M * KC;     // floats per A part (8 KB)
constexpr int NMAX = 64;          // max columns per CTA (32 complex fields)
constexpr int BTILE = NMAX * KC;  // floats per B part (4 KB)
constexpr int STAGE_F = 4 * ATILE + 4 * BTILE;  // floats per stage: A,B x {par0 hi, par0 lo, par1 hi, par1 lo}
constexpr double BIG = 0x1p600, SMALL = 0x1p-600;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s limit of every wait
}  // namespace tc

// Recurrence coefficients of degree l (order m):
//   P_l = a (mu P_{l-1} - b P_{l-2})                        (l >= m + 2)
//   P_l = (alpha mu^2 + beta) P_{l-2} + gamma P_{l-4}       (l >= m + 4)
// the second form is the first applied twice with P_{l-1}, P_{l-3} eliminated:
//   alpha = a_l a_{l-1}, beta = -a_l (a_{l-1} b_{l-1} / a_{l-2} + b_l),
//   gamma = -a_l a_{l-1} b_{l-1} b_{l-2}; it advances the even and the odd
// degrees as two independent chains.
struct TcCoef {
    double2 ab;   // (a, b)
    double2 ag;   // (alpha, beta)
    double2 g;    // (gamma, 0)
};

struct MixedTables {
    TcCoef* ab = nullptr;         // recurrence coefficients of (l, m) at ab[abo(m) + l - m]
    long long* abo = nullptr;     // [m]
    double2* ck = nullptr;        // checkpoints (P_l, P_{l+1}), scaled, at ck[(cko(m) + c) * nhp + j], l = m + SEG c
    int* ckx = nullptr;           // binary exponent of each checkpoint's scale (0, -600, ...)
    long long* cko = nullptr;     // [m]
    int lmax = 0;
    int nhp = 0;                  // checkpoint row stride: nh rounded up to a multiple of 4 (16 B rows of ints)
    int* flag = nullptr;          // device error flag (bit 0: a wait gave up)
    // split-TF32 P tables streamed by TMA (legendre_tcs.cuh)
    float* S = nullptr;           // synthesis layout
    float* A = nullptr;           // analysis layout
    long long* soff = nullptr;    // [m] first z row of order m in S
    long long* aoff = nullptr;    // [m] first row of order m in A
    long long zS = 0, rowsA = 0;
    int zA = 0;
    bool streamed = false;
    CUtensorMap mapS, mapA;
    // B operand prepared by the loader-only kernel (legendre_tcb.cuh)
    // (also the prepared B chunks and column exponents of the int8 kernels with
    // both operands by TMA, legendre_i8b.cuh)
    float* Bbuf = nullptr;
    size_t Bcap = 0;
    // buffers replaced by larger ones: a captured graph may still hold their
    // addresses, so they live until the tables are freed
    std::vector<void*> retired;
    // int8 digit tables of the integer-split kernels (legendre_i8.cuh)
    unsigned char* SY = nullptr;  // synthesis digit planes
    unsigned char* AN = nullptr;  // analysis digit planes (P w)
    unsigned char* ANc = nullptr; // analysis digit planes (P w / cos(phi))
    int* esy = nullptr;           // synthesis row exponents [m][j]
    int* ean = nullptr;           // analysis row exponents [pidx(lmax, l, m)]
    int* eanc = nullptr;          // the same for ANc
    long long* i8zoff = nullptr;  // [m] first z of order m in SY
    long long* i8aoff = nullptr;  // [m] first row of order m in AN
    long long zSY = 0, rowsAN = 0;
    int zAN = 0;
    bool i8 = false;
    CUtensorMap mapSY, mapAN, mapANc;
};

// Offsets of degree m's blocks in the coefficient and checkpoint tables of
// degree T (closed forms of the prefix sums of T - m + 1 and (T - m) / SEG + 1).
__host__ __device__ inline long long tc_abo(int T, int m) {
    return (long long)m * (T + 1) - (long long)m * (m - 1) / 2;
}
__host__ __device__ inline long long tc_floor_sum(int n) {  // sum_{x=0..n} floor(x / SEG)
    const long long q = n / tc::SEG, r = n % tc::SEG;
    return (tc::SEG / 2) * q * (q - 1) + q * (r + 1);
}
__host__ __device__ inline long long tc_cko(int T, int m) { return m + tc_floor_sum(T) - tc_floor_sum(T - m); }

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no-swizzle shared-memory matrix descriptor: 8-row x 16 B core
// matrices, the two 16 B K-halves of an 8-row group 128 B apart (LBO), 8-row
// groups 256 B apart (SBO); descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((256u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: D = F32, A = B = TF32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for a phase with a time limit; gives up early when another thread has
// raised the CTA's abort flag, and raises it on its own timeout.
__device__ __forceinline__ bool mbar_wait_abort(uint32_t mbar, uint32_t phase, volatile int* abort,
                                                unsigned long long limit_ns = tc::WAIT_NS) {
    if (mbar_try(mbar, phase)) return true;
    const uint64_t t0 = globaltimer();
    for (uint32_t i = 0;; i++) {
        if (mbar_try(mbar, phase)) return true;
        if ((i & 63) == 63) {
            if (*abort) return false;
            if (globaltimer() - t0 > limit_ns) {
                *abort = 1;
                return false;
            }
        }
    }
}

// One CTA waits, with the bounded wait of the tensor-core kernels, for a
// barrier phase that nothing completes: the wait gives up after limit_ns and
// the CTA records the failure in the handle's flag exactly as a timed-out
// tensor-core kernel does, then returns.  This exercises the SPH_ERR_TIMEOUT
// path without a faulty kernel.
__global__ void k_wait_selftest(unsigned long long limit_ns, int* flag) {
    __shared__ __align__(8) unsigned long long bar;
    __shared__ int abort;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0 && !mbar_wait_abort(smem_u32(&bar), 0, &abort, limit_ns)) atomicOr(flag, 1);
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t slot_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// N consecutive 32-bit columns of this thread's lane at two TMEM addresses, one wait
template <int N>
__device__ __forceinline__ void tmem_ld_pair(uint32_t ta, uint32_t tb, float* va, float* vb);

template <>
__device__ __forceinline__ void tmem_ld_pair<16>(uint32_t ta, uint32_t tb, float* va, float* vb) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%32];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
        "[%33];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(ta), "r"(tb)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) {
        va[i] = __uint_as_float(r[i]);
        vb[i] = __uint_as_float(r[16 + i]);
    }
}

template <>
__device__ __forceinline__ void tmem_ld_pair<8>(uint32_t ta, uint32_t tb, float* va, float* vb) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%16];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%17];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(ta), "r"(tb)
        : "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) {
        va[i] = __uint_as_float(r[i]);
        vb[i] = __uint_as_float(r[8 + i]);
    }
}

// 16 consecutive 32-bit columns of this thread's lane
__device__ __forceinline__ void tmem_st16(uint32_t ta, const uint32_t* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(ta),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// x = hi + lo with hi, lo representable in TF32 (10 explicit mantissa bits):
// x is rounded once to FP32, hi keeps its top 11 significant bits (round half
// away from zero on the bit pattern), lo = xf - hi is exact in FP32 and is
// rounded the same way.  Bit operations instead of conversions: one cvt per value.
__device__ __forceinline__ float tf32_bits_round(float v) {
    return __uint_as_float((__float_as_uint(v) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
    const float xf = __double2float_rn(x);
    hi = tf32_bits_round(xf);
    lo = tf32_bits_round(xf - hi);
}

// float offset of element (row r, k) in a K-major tile with `rows` rows per K step of 8
__host__ __device__ __forceinline__ int tile_off(int r, int k, int rows) {
    return (k >> 3) * (rows * 8) + (r >> 3) * 64 + ((k & 7) >> 2) * 32 + (r & 7) * 4 + (k & 3);
}

// ------------------------------------------------------------------ P_l^m recurrence
// Same recurrence and scaling as the FP64 table: P_l = a_l (mu P_{l-1} - b_l P_{l-2}),
// values kept scaled by 2^el with el in {0, -600, ...} to survive underflow of P_mm.
__device__ __forceinline__ double plm_a(int l, int m) {
    const double ll = l, mm = m;
    return sqrt((4.0 * ll * ll - 1.0) / (ll * ll - mm * mm));
}
__device__ __forceinline__ double plm_b(int l, int m) {
    const double ll = l, mm = m;
    return sqrt(((ll - 1.0) * (ll - 1.0) - mm * mm) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0));
}
__device__ __forceinline__ void plm_step(double z, double2 ab, double& p0, double& p1, int& el) {
    const double p2 = ab.x * (z * p1 - ab.y * p0);
    p0 = p1;
    p1 = p2;
    if (el < 0 && fabs(p1) > tc::BIG) {
        p0 *= tc::SMALL;
        p1 *= tc::SMALL;
        el += 600;
    }
}
__device__ __forceinline__ double plm_value(double p, int el) {
    return el == 0 ? p : (el == -600 ? p * tc::SMALL : 0.0);
}

// thread per (l, m): recurrence coefficients
__global__ void k_tc_ab(int lmax, int mm, TcCoef* __restrict__ ab) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (m > mm || l < m || l > lmax) return;
    TcCoef c;
    c.ab = l >= m + 2 ? make_double2(plm_a(l, m), plm_b(l, m)) : make_double2(0.0, 0.0);
    c.ag = make_double2(0.0, 0.0);
    c.g = make_double2(0.0, 0.0);
    if (l >= m + 4) {
        const double a0 = plm_a(l, m), b0 = plm_b(l, m);
        const double a1 = plm_a(l - 1, m), b1 = plm_b(l - 1, m);
        const double a2 = plm_a(l - 2, m), b2 = plm_b(l - 2, m);
        c.ag = make_double2(a0 * a1, -a0 * (a1 * b1 / a2 + b0));
        c.g = make_double2(-a0 * a1 * b1 * b2, 0.0);
    }
    ab[tc_abo(lmax, m) + (l - m)] = c;
}

// thread per (j, m): runs the recurrence over all degrees and stores a checkpoint every SEG degrees
__global__ void k_tc_ck(int nh, int nhp, int lmax, int mm, const double* __restrict__ x,
                        const TcCoef* __restrict__ ab, double2* __restrict__ ck, int* __restrict__ ckx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (j >= nh || m > mm) return;
    const double z = x[j];
    const double s = sqrt((1.0 - z) * (1.0 + z));
    double pmm = sqrt(1.0 / (4.0 * kPi));
    int el = 0;
    for (int k = 1; k <= m; k++) {
        pmm *= -sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
        if (fabs(pmm) < tc::SMALL && pmm != 0.0) {
            pmm *= tc::BIG;
            el -= 600;
        }
    }
    double p0 = pmm;
    double p1 = m + 1 <= lmax ? z * sqrt(2.0 * m + 3.0) * p0 : 0.0;
    double2* ckm = ck + tc_cko(lmax, m) * nhp + j;
    int* ckxm = ckx + tc_cko(lmax, m) * nhp + j;
    ckm[0] = make_double2(p0, p1);
    ckxm[0] = el;
    const TcCoef* abm = ab + tc_abo(lmax, m);
    for (int l = m + 2; l <= lmax; l++) {
        plm_step(z, abm[l - m].ab, p0, p1, el);  // state (P_{l-1}, P_l)
        const int d = l - 1 - m;
        if (d % tc::SEG == 0) {
            ckm[(size_t)(d / tc::SEG) * nhp] = make_double2(p0, p1);
            ckxm[(size_t)(d / tc::SEG) * nhp] = el;
        }
    }
    // a checkpoint at l = lmax itself has no successor inside the range
    const int d = lmax - m;
    if (d > 0 && d % tc::SEG == 0) {
        ckm[(size_t)(d / tc::SEG) * nhp] = make_double2(p1, 0.0);
        ckxm[(size_t)(d / tc::SEG) * nhp] = el;
    }
}

static int tcs_tables_build(Handle* h, MixedTables* T);
static int i8_tables_build(Handle* h, MixedTables* T);
static bool g_tc_stream = true;
static bool g_tc_i8 = true;

int tc_tables_build(Handle* h, int lmax) {
    if (h->mixed) return SPH_OK;
    MixedTables* T = new MixedTables();
    h->mixed = T;
    const int nh = h->nh;
    T->lmax = lmax;
    const int mm = std::min(lmax, h->L);
    const long long na = tc_abo(lmax, mm + 1), nc = tc_cko(lmax, mm + 1);
    SPH_CUDA_TRY(cudaMalloc(&T->ab, sizeof(TcCoef) * na));
    T->nhp = (nh + 3) & ~3;
    SPH_CUDA_TRY(cudaMalloc(&T->ck, sizeof(double2) * nc * T->nhp));
    SPH_CUDA_TRY(cudaMalloc(&T->ckx, sizeof(int) * nc * T->nhp));
    SPH_CUDA_TRY(cudaMemset(T->ckx, 0, sizeof(int) * nc * T->nhp));
    SPH_CUDA_TRY(cudaMalloc(&T->flag, sizeof(int)));
    SPH_CUDA_TRY(cudaMemset(T->flag, 0, sizeof(int)));
    k_tc_ab<<<dim3((lmax + 128) / 128, mm + 1), 128>>>(lmax, mm, T->ab);
    SPH_CUDA_TRY(cudaGetLastError());
    k_tc_ck<<<dim3((nh + 127) / 128, mm + 1), 128>>>(nh, T->nhp, lmax, mm, h->mu, T->ab, T->ck, T->ckx);
    SPH_CUDA_TRY(cudaGetLastError());
    if (g_tc_stream)
        if (int rc = tcs_tables_build(h, T)) return rc;
    if (g_tc_i8)
        if (int rc = i8_tables_build(h, T)) return rc;
    SPH_CUDA_TRY(cudaDeviceSynchronize());
    return SPH_OK;
}

void tc_tables_free(Handle* h) {
    MixedTables* T = static_cast<MixedTables*>(h->mixed);
    if (!T) return;
    void* bufs[] = {T->ab, T->ck,   T->ckx, T->flag,   T->S,      T->A,     T->soff,
                    T->aoff, T->Bbuf, T->SY, T->AN, T->ANc, T->esy, T->ean, T->eanc, T->i8zoff, T->i8aoff};
    for (void* p : bufs)
        if (p) cudaFree(p);
    for (void* p : T->retired) cudaFree(p);
    delete T;
    h->mixed = nullptr;
}

// ------------------------------------------------------------------ kernels
struct TcArgs {
    const TcCoef* ab;
    const double2* ck;
    const int* ckx;
    const double* mu;
    const double* w;
    int tlmax;      // degree of the coefficient / checkpoint tables
    int lmax;       // degree of this call's packed layout (<= tlmax)
    int nh, nhp, nlat;
    int batch;      // fields
    int nct, nrt;   // column tiles, row tiles (latitude tiles or degree tiles)
    int ntiles;     // nct * nrt * (number of m)
    int group;      // chunks accumulated in FP32 before each FP64 update (1 or 2)
    long long ld_spec;
    long long ldF;
    int* flag;
};

// Shared-memory map: NSTAGE operand stages, NRAW raw prefetch buffers (the
// producers prefetch NRAW-1 chunks ahead with cp.async), barriers.  A raw
// buffer holds the generators' checkpoints, mu and scale exponents, the
// recurrence coefficients of the chunk's degrees (segment h at row 17 h), and
// the B-operand data.
namespace tcs {
constexpr int NSTAGE = 2;
constexpr int NRAW = 3;
constexpr int STAGE_B = 4 * tc::STAGE_F;                  // 48 KB
constexpr int R_CK = 0;                                   // double2[256]
constexpr int R_MU = R_CK + 256 * 16;                     // double[256]
constexpr int R_EX = R_MU + 256 * 8;                      // int[256]
constexpr int R_AB = R_EX + 256 * 4;                      // TcCoef[16][17]
constexpr int R_B = R_AB + 16 * 17 * 48;                  // double2[32][NF + 4], then double[16]
constexpr int RAW_B = R_B + 32 * (32 + 4) * 16 + 16 * 8;  // 38 KB
constexpr int OFF_RAW = NSTAGE * STAGE_B;
constexpr int OFF_BAR = OFF_RAW + NRAW * RAW_B;
constexpr int BYTES = OFF_BAR + 256;
}  // namespace tcs
constexpr size_t tc_smem_bytes() { return (size_t)tcs::BYTES; }

// position of a chunk in the CTA's sequence of tiles
struct TcPos {
    int t;    // tile index (>= ntiles: none)
    int m, rt, ct;
    int kc, nk;
};

__device__ __forceinline__ void cp_async(void* dst, const void* src, int bytes, bool valid) {
    const uint32_t d = smem_u32(dst);
    const int n = valid ? bytes : 0;  // 0: zero fill, nothing read
    if (bytes == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// named barrier over the producer warpgroups, with an AND of v
__device__ __forceinline__ bool producers_and(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 384, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void producers_sync() { asm volatile("bar.sync 1, 384;" ::: "memory"); }

// raw prefetch slots of one buffer
struct Raw {
    double2* ck;
    double* mu;
    int* ex;
    TcCoef* ab;
    double2* b;  // [32][NF + 4]: spectral (parity 16 + k) or Fourier (hemisphere 16 + k) rows
};
__device__ __forceinline__ Raw raw_buf(unsigned char* smem, int buf) {
    unsigned char* p = smem + tcs::OFF_RAW + buf * tcs::RAW_B;
    return Raw{reinterpret_cast<double2*>(p + tcs::R_CK), reinterpret_cast<double*>(p + tcs::R_MU),
               reinterpret_cast<int*>(p + tcs::R_EX), reinterpret_cast<TcCoef*>(p + tcs::R_AB),
               reinterpret_cast<double2*>(p + tcs::R_B)};
}

// The SEG values P_l(mu), l = l0 .. l0+SEG-1 (zero above lmax), from the
// checkpoint at l0 and the coefficients abl[t] of degree l0 + t (shared
// memory), handed to emit(t, hi, lo) with t = l - l0 a compile-time constant.
// Unscaled full segments (the common case) take the branch-free path: two
// ordinary steps, then the even and odd degrees as two independent chains of
// the mu^2 form, one dependent FMA per step.
template <typename Emit>
__device__ __forceinline__ void plm_segment(double z, double2 c, int el, const TcCoef* abl, int l0, int lmax,
                                            Emit&& emit) {
    float hi, lo;
    if (el == 0 && l0 + tc::SEG - 1 <= lmax) {
        double v[tc::SEG];
        v[0] = c.x;
        v[1] = c.y;
        v[2] = abl[2].ab.x * (z * v[1] - abl[2].ab.y * v[0]);
        v[3] = abl[3].ab.x * (z * v[2] - abl[3].ab.y * v[1]);
        const double z2 = z * z;
#pragma unroll
        for (int t = 4; t < tc::SEG; t++) {
            const double2 ag = abl[t].ag;
            v[t] = fma(fma(ag.x, z2, ag.y), v[t - 2], abl[t].g.x * v[t - 4]);
        }
#pragma unroll
        for (int t = 0; t < tc::SEG; t++) {
            split_tf32(v[t], hi, lo);
            emit(t, hi, lo);
        }
        return;
    }
    double p0 = c.x, p1 = c.y;
    split_tf32(l0 <= lmax ? plm_value(p0, el) : 0.0, hi, lo);
    emit(0, hi, lo);
    split_tf32(l0 + 1 <= lmax ? plm_value(p1, el) : 0.0, hi, lo);
    emit(1, hi, lo);
#pragma unroll
    for (int t = 2; t < tc::SEG; t++) {
        const int l = l0 + t;
        double v = 0.0;
        if (l <= lmax) {
            plm_step(z, abl[t].ab, p0, p1, el);
            v = plm_value(p1, el);
        }
        split_tf32(v, hi, lo);
        emit(t, hi, lo);
    }
}

// Issue the split-TF32 products of one staged chunk for both parities (one
// thread) into the accumulator buffer (E at column 0, O at NC); the first
// product starts from zero unless `acc`.  Descriptors differ only in their
// start-address field, so each is the stage's base descriptor plus a
// compile-time offset (in 16 B units).
template <int NC>
__device__ __forceinline__ void tc_issue_chunk(const float* As, const float* Bs, uint32_t tacc, bool acc) {
    constexpr uint32_t idesc = idesc_tf32(tc::M, NC);
    const uint64_t dA = sdesc(smem_u32(As)), dB = sdesc(smem_u32(Bs));
#pragma unroll
    for (int s = 0; s < tc::KC / 8; s++) {
#pragma unroll
        for (int par = 0; par < 2; par++) {
            const uint64_t ah = dA + (uint64_t)((par * 2 * tc::ATILE * 4 + s * tc::M * 32) >> 4);
            const uint64_t al = ah + (uint64_t)((tc::ATILE * 4) >> 4);
            const uint64_t bh = dB + (uint64_t)((par * 2 * tc::BTILE * 4 + s * NC * 32) >> 4);
            const uint64_t bl = bh + (uint64_t)((tc::BTILE * 4) >> 4);
            const uint32_t d = tacc + par * NC;
            mma_tf32(d, ah, bh, idesc, (s > 0 || acc) ? 1u : 0u);
            mma_tf32(d, ah, bl, idesc, 1u);
            mma_tf32(d, al, bh, idesc, 1u);
        }
    }
}

// TMEM plan per column count: NACC FP32 accumulator buffers of 2 NC columns
// (E at 0, O at NC), then the FP64 running sums, two 32-bit columns per value
// (E at ACC64, O at ACC64 + 2 NC).
template <int NC>
struct TcCfg {
    static constexpr int NACC = NC == 64 ? 2 : 4;
    static constexpr uint32_t ACC64 = (uint32_t)(NACC * 2 * NC);
    static constexpr uint32_t USED = ACC64 + 4 * NC;
    static constexpr uint32_t NCOLS = USED <= 32 ? 32u : USED <= 64 ? 64u : USED <= 128 ? 128u : USED <= 256 ? 256u : 512u;
};


// B-operand item decomposition: lanes cover (re/im, k & 3, f & 3) so that the
// scalar stores into the K-major tile hit 32 distinct banks.  k depends on the
// B thread only (idx = bt + 128 it).
__device__ __forceinline__ int item_ri(int idx) { return idx & 1; }
__device__ __forceinline__ int item_k(int idx) { return ((idx >> 1) & 3) | (((idx >> 5) & 3) << 2); }

// Synthesis: tile = (column tile, latitude tile of 128, m); chunk k = degrees
// l = m + 32k .. m + 32k + 31 (16 per parity = K of the chunk).  Generator
// thread t < 256: P row t & 127, half h = t >> 7 (degrees 16h .. 16h+15);
// B thread bt = t - 256: NC/4 coefficient items.
template <int NC>
struct SynDir {
    static constexpr int NF = NC / 2;
    static constexpr int BIT = NC * 2 * tc::KC / tc::NBST;  // B items per B thread
    __device__ static int nchunks(const TcArgs& a, int m, int) { return (a.lmax - m) / (2 * tc::KC) + 1; }
    __device__ static int item_f(int idx) { return ((idx >> 3) & 3) | ((idx >> 7) % (NF / 4)) * 4; }
    __device__ static int item_par(int idx) { return (idx >> 7) / (NF / 4); }

    __device__ static void prefetch(const TcArgs& a, const double2* __restrict__ spec, const TcPos& p,
                                    unsigned char* smem, int buf) {
        const int tid = threadIdx.x;
        const int l0 = p.m + 2 * tc::KC * p.kc;
        const Raw r = raw_buf(smem, buf);
        if (tid >= tc::NGEN) {
            // coefficients (f, l0 + d), d = 0..31: consecutive threads read consecutive degrees
            const int bt = tid - tc::NGEN;
#pragma unroll
            for (int it = 0; it < NF * 32 / tc::NBST; it++) {
                const int idx = bt + tc::NBST * it;
                const int d = idx & 31, fl = idx >> 5;
                const int l = l0 + d, f = p.ct * NF + fl;
                const bool v = l <= a.lmax && f < a.batch;
                cp_async(&r.b[((d & 1) * 16 + (d >> 1)) * (NF + 4) + fl],
                         v ? (const void*)(spec + (long long)f * a.ld_spec + pidx(a.lmax, l, p.m)) : (const void*)spec,
                         16, v);
            }
            return;
        }
        {
            const int gr = tid & (tc::M - 1), gh = tid >> 7;
            const int gj = p.rt * tc::M + gr;
            const bool v = gj < a.nh && l0 + tc::SEG * gh <= a.lmax;
            const long long ci = (tc_cko(a.tlmax, p.m) + 2 * p.kc + gh) * (long long)a.nhp + gj;
            cp_async(&r.ck[tid], v ? (const void*)(a.ck + ci) : (const void*)a.ck, 16, v);
            cp_async(&r.ex[tid], v ? (const void*)(a.ckx + ci) : (const void*)a.ckx, 4, v);
            cp_async(&r.mu[tid], v ? (const void*)(a.mu + gj) : (const void*)a.mu, 8, v);
        }
        if (tid < 3 * 2 * tc::KC) {  // coefficients of degrees l0 .. l0+31 (segment h at 17 h), 3 x 16 B each
            const int e = tid / 3, part = tid % 3;
            const int l = l0 + e;
            const bool v = l <= a.lmax;
            const double2* src = reinterpret_cast<const double2*>(a.ab + tc_abo(a.tlmax, p.m) + (l - p.m)) + part;
            cp_async(reinterpret_cast<double2*>(&r.ab[(e >> 4) * 17 + (e & 15)]) + part,
                     v ? (const void*)src : (const void*)a.ab, 16, v);
        }
    }

    __device__ static void fill(const TcArgs& a, const TcPos& p, float* As, float* Bs, unsigned char* smem, int buf) {
        const int tid = threadIdx.x;
        const int l0 = p.m + 2 * tc::KC * p.kc;
        const Raw r = raw_buf(smem, buf);
        if (tid >= tc::NGEN) {
            const int bt = tid - tc::NGEN;
#pragma unroll
            for (int it = 0; it < BIT; it++) {
                const int idx = bt + tc::NBST * it;
                const double2 q = r.b[(item_par(idx) * 16 + item_k(idx)) * (NF + 4) + item_f(idx)];
                float hi, lo;
                split_tf32(item_ri(idx) ? q.y : q.x, hi, lo);
                float* bp =
                    Bs + item_par(idx) * 2 * tc::BTILE + tile_off(2 * item_f(idx) + item_ri(idx), item_k(idx), NC);
                bp[0] = hi;
                bp[tc::BTILE] = lo;
            }
            return;
        }
        const int gr = tid & (tc::M - 1), gh = tid >> 7;
        const int gj = p.rt * tc::M + gr;
        float h[8], g[8];
        auto emit = [&](int t, float hi, float lo) {
            h[t & 7] = hi;
            g[t & 7] = lo;
            if ((t & 7) == 7) {
                const int k0 = 8 * gh + (t >> 3) * 4;
#pragma unroll
                for (int par = 0; par < 2; par++) {
                    float* ap = As + par * 2 * tc::ATILE + tile_off(gr, k0, tc::M);
                    *reinterpret_cast<float4*>(ap) = make_float4(h[par], h[par + 2], h[par + 4], h[par + 6]);
                    *reinterpret_cast<float4*>(ap + tc::ATILE) = make_float4(g[par], g[par + 2], g[par + 4], g[par + 6]);
                }
            }
        };
        const int lseg = l0 + tc::SEG * gh;
        if (gj < a.nh && lseg <= a.lmax) {
            plm_segment(r.mu[tid], r.ck[tid], r.ex[tid], r.ab + 17 * gh, lseg, a.lmax, emit);
        } else {
#pragma unroll
            for (int t = 0; t < tc::SEG; t++) emit(t, 0.f, 0.f);
        }
    }

    // consumer thread: row 32 (cw & 3) + lane; columns col .. col+7 = fields col/2 .. col/2+3
    __device__ static void epilogue(const TcArgs& a, const TcPos& p, int cw, int col, double2* __restrict__ F,
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

// Analysis: tile = (column tile, degree tile of 256 = 128 rows per parity, m);
// chunk k = latitudes j = 16k .. 16k+15.  Generator thread (s, jj), s, jj = 0..15,
// regenerates degrees l = lbase + 16 s + t at latitude 16k + jj; the i-th degree
// of parity p of segment s sits in row 8 s + ((i + s) & 7), a rotation that keeps
// the scalar shared-memory stores free of bank conflicts.
template <int NC>
struct AnaDir {
    static constexpr int NF = NC / 2;
    static constexpr int BIT = NC * tc::KC / tc::NBST;  // B items per B thread
    __device__ static int nchunks(const TcArgs& a, int m, int rt) {
        return m + 2 * tc::M * rt > a.lmax ? 0 : (a.nh + tc::KC - 1) / tc::KC;
    }
    __device__ static int gs() { return (threadIdx.x & 7) | (((threadIdx.x >> 5) & 1) << 3); }
    __device__ static int gjj() { return ((threadIdx.x >> 3) & 3) | ((threadIdx.x >> 6) << 2); }
    __device__ static int item_f(int idx) { return ((idx >> 3) & 3) | ((idx >> 7) << 2); }

    __device__ static void prefetch(const TcArgs& a, const double2* __restrict__ F, const TcPos& p, unsigned char* smem,
                                    int buf) {
        const int tid = threadIdx.x;
        const int lbase = p.m + 2 * tc::M * p.rt;
        const Raw r = raw_buf(smem, buf);
        if (tid >= tc::NGEN) {
            // Fourier data (f, hemisphere, j0 + k): consecutive threads read consecutive latitudes
            const int bt = tid - tc::NGEN;
            const int j0 = p.kc * tc::KC;
#pragma unroll
            for (int it = 0; it < NF * 32 / tc::NBST; it++) {
                const int idx = bt + tc::NBST * it;
                const int k = idx & 15, hs = (idx >> 4) & 1, fl = idx >> 5;
                const int j = j0 + k, f = p.ct * NF + fl;
                const bool v = j < a.nh && f < a.batch;
                const double2* src = F + (long long)f * a.ldF + (long long)p.m * a.nlat + (hs ? a.nlat - 1 - j : j);
                cp_async(&r.b[(hs * 16 + k) * (NF + 4) + fl], v ? (const void*)src : (const void*)F, 16, v);
            }
            if (bt < tc::KC) {
                double* wr = reinterpret_cast<double*>(r.b + 32 * (NF + 4));
                cp_async(&wr[bt], j0 + bt < a.nh ? (const void*)(a.w + j0 + bt) : (const void*)a.w, 8, j0 + bt < a.nh);
            }
            return;
        }
        {
            const int s = gs();
            const int j = p.kc * tc::KC + gjj();
            const bool v = j < a.nh && lbase + tc::SEG * s <= a.lmax;
            const long long ci = (tc_cko(a.tlmax, p.m) + (2 * tc::M / tc::SEG) * p.rt + s) * (long long)a.nhp + j;
            cp_async(&r.ck[tid], v ? (const void*)(a.ck + ci) : (const void*)a.ck, 16, v);
            cp_async(&r.ex[tid], v ? (const void*)(a.ckx + ci) : (const void*)a.ckx, 4, v);
            cp_async(&r.mu[tid], v ? (const void*)(a.mu + j) : (const void*)a.mu, 8, v);
        }
#pragma unroll
        for (int it = 0; it < 3; it++) {  // coefficients of the tile's 256 degrees, segment s at 17 s, 3 x 16 B each
            const int idx = tid + tc::NGEN * it;
            const int e = idx / 3, part = idx % 3;
            const int l = lbase + e;
            const bool v = l <= a.lmax;
            const double2* src = reinterpret_cast<const double2*>(a.ab + tc_abo(a.tlmax, p.m) + (l - p.m)) + part;
            cp_async(reinterpret_cast<double2*>(&r.ab[(e >> 4) * 17 + (e & 15)]) + part,
                     v ? (const void*)src : (const void*)a.ab, 16, v);
        }
    }

    __device__ static void fill(const TcArgs& a, const TcPos& p, float* As, float* Bs, unsigned char* smem, int buf) {
        const int tid = threadIdx.x;
        const Raw r = raw_buf(smem, buf);
        if (tid >= tc::NGEN) {
            // G_S = w (F_j + F_mirror) (even parity), G_A = w (F_j - F_mirror) (odd), K = latitude
            const int bt = tid - tc::NGEN;
            const int k = item_k(bt), ri = item_ri(bt);
            const double wj = reinterpret_cast<const double*>(r.b + 32 * (NF + 4))[k];
#pragma unroll
            for (int it = 0; it < BIT; it++) {
                const int idx = bt + tc::NBST * it;
                const double2 qn = r.b[k * (NF + 4) + item_f(idx)], qs = r.b[(16 + k) * (NF + 4) + item_f(idx)];
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
            return;
        }
        const int s = gs(), jj = gjj();
        const int j = p.kc * tc::KC + jj;
        const int l0 = p.m + 2 * tc::M * p.rt + tc::SEG * s;
        auto emit = [&](int t, float hi, float lo) {
            const int par = t & 1, i = t >> 1;
            float* ap = As + par * 2 * tc::ATILE + tile_off(8 * s + ((i + s) & 7), jj, tc::M);
            ap[0] = hi;
            ap[tc::ATILE] = lo;
        };
        if (j < a.nh && l0 <= a.lmax) {
            plm_segment(r.mu[tid], r.ck[tid], r.ex[tid], r.ab + 17 * s, l0, a.lmax, emit);
        } else {
#pragma unroll
            for (int t = 0; t < tc::SEG; t++) emit(t, 0.f, 0.f);
        }
    }

    // consumer thread: TMEM lane r = row r (segment s = r >> 3, position i = ((r & 7) - s) & 7);
    // columns col .. col+7 = fields col/2 .. col/2+3
    __device__ static void epilogue(const TcArgs& a, const TcPos& p, int cw, int col, double2* __restrict__ spec,
                                    const double* e, const double* o) {
        const int r = (cw & 3) * 32 + (threadIdx.x & 31);
        const int rs = r >> 3;
        const int i = ((r & 7) - rs) & 7;
        const int le = p.m + 2 * tc::M * p.rt + tc::SEG * rs + 2 * i;  // even-parity degree of this row
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

// Consumer warp cw (0..3): TMEM lanes 32 cw .. +31, all NC columns of E and of O,
// in pieces of 8.  The group's FP32 partial sums
// are added to the FP64 running sums kept in TMEM; the tile's first group starts
// them, its last group hands the totals to the epilogue instead of storing them.
template <class Dir, int NC>
__device__ __forceinline__ void tc_consume(const TcArgs& a, const TcPos& p, uint32_t tmem, int b, int cw, bool first,
                                           bool last, double2* __restrict__ out) {
    constexpr int H = NC;
    const uint32_t lane = (uint32_t)((cw & 3) * 32) << 16;
    const int col0 = 0;
    const uint32_t part = tmem + lane + (uint32_t)(b * 2 * NC + col0);
    const uint32_t sum = tmem + lane + TcCfg<NC>::ACC64 + (uint32_t)(2 * col0);
#pragma unroll
    for (int c0 = 0; c0 < H; c0 += 8) {
        float e[8], o[8];
        tmem_ld_pair<8>(part + c0, part + NC + c0, e, o);
        double se[8], so[8];
        if (first) {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                se[i] = (double)e[i];
                so[i] = (double)o[i];
            }
        } else {
            float we[16], wo[16];
            tmem_ld_pair<16>(sum + 2 * c0, sum + 2 * NC + 2 * c0, we, wo);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                se[i] = __hiloint2double(__float_as_int(we[2 * i + 1]), __float_as_int(we[2 * i])) + (double)e[i];
                so[i] = __hiloint2double(__float_as_int(wo[2 * i + 1]), __float_as_int(wo[2 * i])) + (double)o[i];
            }
        }
        if (last) {
            Dir::epilogue(a, p, cw, col0 + c0, out, se, so);
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

template <class Dir>
__device__ __forceinline__ TcPos tc_tile(const TcArgs& a, int t) {
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
__device__ __forceinline__ TcPos tc_next(const TcArgs& a, TcPos p) {
    if (p.kc + 1 < p.nk) {
        p.kc++;
        return p;
    }
    return tc_tile<Dir>(a, p.t + gridDim.x);
}

// Persistent, warp-specialised CTA (one per SM) walking tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... as one stream of chunks q.
//   producers (warps 0-7): prefetch the raw data of chunk q + NRAW - 1
//     (cp.async), wait for stage q % NSTAGE to be free, regenerate P and stage B
//     for chunk q and mark the stage full;
//   MMA warp (warp 16, one thread): wait for the stage and, at a group's first
//     chunk, for its accumulator buffer to be drained; issue the chunk's MMAs
//     and commit stage-free / group-ready;
//   consumers (warps 8-15): per group, wait until ready, fold the accumulator
//     into the FP64 sums, release the buffer, and write a finished tile out.
template <class Dir, int NC>
__global__ void __launch_bounds__(tc::NT, 1) k_legendre_tc(TcArgs a, const double2* __restrict__ in,
                                                            double2* __restrict__ out) {
    constexpr int NACC = TcCfg<NC>::NACC;
    constexpr uint32_t NCOLS = TcCfg<NC>::NCOLS;
    extern __shared__ __align__(1024) unsigned char smem[];
    float* stages = reinterpret_cast<float*>(smem);
    unsigned long long* empty = reinterpret_cast<unsigned long long*>(smem + tcs::OFF_BAR);  // [NSTAGE]
    unsigned long long* full = empty + tcs::NSTAGE;                                           // [NSTAGE]
    unsigned long long* accfull = full + tcs::NSTAGE;                                         // [NACC]
    unsigned long long* accempty = accfull + NACC;                                            // [NACC]
    volatile int* abort = reinterpret_cast<volatile int*>(accempty + NACC);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(accempty + NACC) + 1;
    const int tid = threadIdx.x, warp = tid >> 5;

    const TcPos first = tc_tile<Dir>(a, blockIdx.x);
    if (first.t >= a.ntiles) return;

    if (warp == 0) tmem_alloc(smem_u32(tslot), NCOLS);
    if (tid == 0) {
        for (int i = 0; i < tcs::NSTAGE; i++) {
            mbar_init(smem_u32(&empty[i]), 1);
            mbar_init(smem_u32(&full[i]), 1);
        }
        for (int i = 0; i < NACC; i++) {
            mbar_init(smem_u32(&accfull[i]), 1);
            mbar_init(smem_u32(&accempty[i]), tc::NCONS);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    int issued = -1;

    if (tid < tc::NPROD) {
        TcPos cur = first, pf = first;
#pragma unroll
        for (int i = 0; i < tcs::NRAW - 1; i++) {
            if (pf.t < a.ntiles) {
                Dir::prefetch(a, in, pf, smem, i);
                pf = tc_next<Dir>(a, pf);
            }
            cp_async_commit();
        }
        int q = 0;
        while (cur.t < a.ntiles) {
            if (pf.t < a.ntiles) {
                Dir::prefetch(a, in, pf, smem, (q + tcs::NRAW - 1) % tcs::NRAW);
                pf = tc_next<Dir>(a, pf);
            }
            cp_async_commit();
            cp_async_wait<tcs::NRAW - 1>();
            const int s = q % tcs::NSTAGE;
            bool v = true;
            if (tid == 0 && q >= tcs::NSTAGE)
                v = mbar_wait_abort(smem_u32(&empty[s]), (uint32_t)((q / tcs::NSTAGE - 1) & 1), abort);
            if (!producers_and(v)) break;  // also publishes every producer's prefetched data
            float* As = stages + s * tc::STAGE_F;
            float* Bs = As + 4 * tc::ATILE;
            Dir::fill(a, cur, As, Bs, smem, q % tcs::NRAW);
            fence_async_smem();
            producers_sync();
            if (tid == 0) mbar_arrive(smem_u32(&full[s]));
            q++;
            cur = tc_next<Dir>(a, cur);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp == tc::MMA_WARP) {
        // MMA warp: lane 0 issues each staged chunk once the producers filled it
        if (tid == tc::MMA_WARP * 32) {
            TcPos cur = first;
            int q = 0, gq = -1;
            while (cur.t < a.ntiles) {
                const int s = q % tcs::NSTAGE;
                const bool gfirst = cur.kc % a.group == 0;
                const bool glast = cur.kc % a.group == a.group - 1 || cur.kc == cur.nk - 1;
                if (gfirst) gq++;
                const int b = gq % NACC;
                if (!mbar_wait_abort(smem_u32(&full[s]), (uint32_t)((q / tcs::NSTAGE) & 1), abort)) break;
                if (gfirst && gq >= NACC &&
                    !mbar_wait_abort(smem_u32(&accempty[b]), (uint32_t)(((gq - NACC) / NACC) & 1), abort))
                    break;
                tc_fence_after();
                float* As = stages + s * tc::STAGE_F;
                tc_issue_chunk<NC>(As, As + 4 * tc::ATILE, tmem + b * 2 * NC, !gfirst);
                mma_commit(smem_u32(&empty[s]));
                if (glast) mma_commit(smem_u32(&accfull[b]));
                issued = q;
                q++;
                cur = tc_next<Dir>(a, cur);
            }
        }
        __syncwarp();
    } else {
        const int cw = warp - tc::NPROD / 32;
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
                tc_consume<Dir, NC>(a, cur, tmem, b, cw, cur.kc < a.group, cur.kc == cur.nk - 1, out);
                tc_fence_before();
                mbar_arrive(smem_u32(&accempty[b]));
            }
            cur = tc_next<Dir>(a, cur);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort) {
        // let the last issued chunk finish before its tensor memory is freed
        if (tid == tc::MMA_WARP * 32) {
            if (issued >= 0) {
                const uint32_t bar = smem_u32(&empty[issued % tcs::NSTAGE]);
                const uint32_t ph = (uint32_t)((issued / tcs::NSTAGE) & 1);
                const uint64_t t0 = globaltimer();
                while (!mbar_try(bar, ph) && globaltimer() - t0 < tc::WAIT_NS) {
                }
            }
            atomicOr(a.flag, 1);
        }
        __syncthreads();
    }
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, NCOLS);
    }
}

#include "legendre_tcs.cuh"
#include "legendre_tcb.cuh"
#include "legendre_i8.cuh"
#include "legendre_i8b.cuh"

// rows: padded row count (a multiple of 64), slices: z extent
static int encode_map(CUtensorMap* map, float* base, unsigned long long rows, unsigned long long slices) {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* f = nullptr;
        SPH_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
        if (!f || q != cudaDriverEntryPointSuccess) {
            set_error("cuTensorMapEncodeTiled is not available");
            return SPH_ERR_CUDA;
        }
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    // dims (64 rows x 4 floats, row blocks, slices, 2 parts); box 256 x 2 x 4 x 2
    const cuuint64_t dims[4] = {256, rows / 64, slices, 2};
    const cuuint64_t strides[3] = {1024, 16ull * rows, 16ull * rows * slices};
    const cuuint32_t box[4] = {256, 2, 4, 2};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}

static int tcs_tables_build(Handle* h, MixedTables* T) {
    const int tl = T->lmax, nh = h->nh, mm = std::min(tl, h->L);
    const int nhP = tcs_pad64(nh);
    std::vector<long long> so(mm + 2, 0), ao(mm + 2, 0);
    for (int m = 0; m <= mm; m++) {
        so[m + 1] = so[m] + 8LL * tcs_nchunks(tl, m);
        ao[m + 1] = ao[m] + tcs_pad64(tcs_nlp(tl, m, 0)) + tcs_pad64(tcs_nlp(tl, m, 1));
    }
    T->zS = so[mm + 1];
    T->rowsA = ao[mm + 1];
    T->zA = (nh + 3) / 4;
    const size_t bs = sizeof(float) * 2 * (size_t)T->zS * nhP * 4, ba = sizeof(float) * 2 * (size_t)T->zA * T->rowsA * 4;
    SPH_CUDA_TRY(cudaMalloc(&T->S, bs));
    SPH_CUDA_TRY(cudaMalloc(&T->A, ba));
    SPH_CUDA_TRY(cudaMemset(T->S, 0, bs));
    SPH_CUDA_TRY(cudaMemset(T->A, 0, ba));
    SPH_CUDA_TRY(cudaMalloc(&T->soff, sizeof(long long) * (mm + 2)));
    SPH_CUDA_TRY(cudaMalloc(&T->aoff, sizeof(long long) * (mm + 2)));
    SPH_CUDA_TRY(cudaMemcpy(T->soff, so.data(), sizeof(long long) * (mm + 2), cudaMemcpyHostToDevice));
    SPH_CUDA_TRY(cudaMemcpy(T->aoff, ao.data(), sizeof(long long) * (mm + 2), cudaMemcpyHostToDevice));
    k_tcs_tables<<<dim3((nh + 127) / 128, mm + 1), 128>>>(nh, nhP, tl, mm, h->mu, T->soff, T->aoff, T->zS, T->rowsA,
                                                          T->zA, T->S, T->A);
    SPH_CUDA_TRY(cudaGetLastError());
    if (int rc = encode_map(&T->mapS, T->S, (unsigned long long)nhP, (unsigned long long)T->zS)) return rc;
    if (int rc = encode_map(&T->mapA, T->A, (unsigned long long)T->rowsA, (unsigned long long)T->zA)) return rc;
    T->streamed = true;
    return SPH_OK;
}

// tensor map of an int8 digit table seen as 32-bit words: dims (64 rows x 16 B,
// row blocks, z, 4 digit planes), box {256, 2, 2, 4} = 128 rows x 32 K x 4 planes
static int encode_map_i8(CUtensorMap* map, unsigned char* base, unsigned long long rows, unsigned long long zext) {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* f = nullptr;
        SPH_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
        if (!f || q != cudaDriverEntryPointSuccess) {
            set_error("cuTensorMapEncodeTiled is not available");
            return SPH_ERR_CUDA;
        }
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    const cuuint64_t dims[4] = {256, rows / 64, zext, 4};
    const cuuint64_t strides[3] = {1024, 16ull * rows, 16ull * rows * zext};
    const cuuint32_t box[4] = {256, 2, 2, 4};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (int8 tables) failed (" + std::to_string((int)r) + ")");
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}

static int i8_tables_build(Handle* h, MixedTables* T) {
    const int tl = T->lmax, nh = h->nh, mm = std::min(tl, h->L);
    const int nhP = tcs_pad64(nh);
    std::vector<long long> zo(mm + 2, 0), ao(mm + 2, 0);
    for (int m = 0; m <= mm; m++) {
        zo[m + 1] = zo[m] + 4LL * i8_nch(tl, m);
        ao[m + 1] = ao[m] + tcs_pad64(i8_nlp(tl, m, 0)) + tcs_pad64(i8_nlp(tl, m, 1));
    }
    T->zSY = zo[mm + 1];
    T->rowsAN = ao[mm + 1];
    T->zAN = 2 * ((nh + li8::KC - 1) / li8::KC);
    const long long nlmT = (long long)(tl + 1) * (tl + 2) / 2;
    const size_t bs = (size_t)4 * T->zSY * nhP * 16, ba = (size_t)4 * T->zAN * T->rowsAN * 16;
    SPH_CUDA_TRY(cudaMalloc(&T->SY, bs));
    SPH_CUDA_TRY(cudaMalloc(&T->AN, ba));
    SPH_CUDA_TRY(cudaMalloc(&T->ANc, ba));
    SPH_CUDA_TRY(cudaMemset(T->SY, 0, bs));
    SPH_CUDA_TRY(cudaMemset(T->AN, 0, ba));
    SPH_CUDA_TRY(cudaMemset(T->ANc, 0, ba));
    SPH_CUDA_TRY(cudaMalloc(&T->esy, sizeof(int) * (size_t)(mm + 1) * nh));
    SPH_CUDA_TRY(cudaMalloc(&T->ean, sizeof(int) * (size_t)nlmT));
    SPH_CUDA_TRY(cudaMemset(T->ean, 0, sizeof(int) * (size_t)nlmT));
    SPH_CUDA_TRY(cudaMalloc(&T->eanc, sizeof(int) * (size_t)nlmT));
    SPH_CUDA_TRY(cudaMemset(T->eanc, 0, sizeof(int) * (size_t)nlmT));
    SPH_CUDA_TRY(cudaMalloc(&T->i8zoff, sizeof(long long) * (mm + 2)));
    SPH_CUDA_TRY(cudaMalloc(&T->i8aoff, sizeof(long long) * (mm + 2)));
    SPH_CUDA_TRY(cudaMemcpy(T->i8zoff, zo.data(), sizeof(long long) * (mm + 2), cudaMemcpyHostToDevice));
    SPH_CUDA_TRY(cudaMemcpy(T->i8aoff, ao.data(), sizeof(long long) * (mm + 2), cudaMemcpyHostToDevice));
    unsigned long long* amax = nullptr;
    SPH_CUDA_TRY(cudaMalloc(&amax, sizeof(unsigned long long) * (size_t)nlmT));
    cudaError_t e = cudaMemset(amax, 0, sizeof(unsigned long long) * (size_t)nlmT);
    const dim3 grid((nh + 127) / 128, mm + 1);
    if (e == cudaSuccess) {
        // weights w: synthesis rows and the analysis table AN
        k_i8_rowmax<<<grid, 128>>>(nh, tl, mm, h->mu, h->w, T->esy, amax);
        k_i8_anexp<<<(unsigned)((nlmT + 255) / 256), 256>>>(nlmT, amax, T->ean);
        k_i8_tables<<<grid, 128>>>(nh, nhP, tl, mm, h->mu, h->w, T->esy, T->ean, T->i8zoff, T->i8aoff, T->zSY,
                                   T->rowsAN, T->zAN, T->SY, T->AN);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * (size_t)nlmT);
    if (e == cudaSuccess) {
        // weights w / cos(phi): the analysis table ANc only
        k_i8_rowmax<<<grid, 128>>>(nh, tl, mm, h->mu, h->wc, nullptr, amax);
        k_i8_anexp<<<(unsigned)((nlmT + 255) / 256), 256>>>(nlmT, amax, T->eanc);
        k_i8_tables<<<grid, 128>>>(nh, nhP, tl, mm, h->mu, h->wc, T->esy, T->eanc, T->i8zoff, T->i8aoff, T->zSY,
                                   T->rowsAN, T->zAN, nullptr, T->ANc);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    cudaFree(amax);
    if (e != cudaSuccess) {
        set_error(std::string("int8 Legendre tables: ") + cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    if (int rc = encode_map_i8(&T->mapSY, T->SY, (unsigned long long)nhP, (unsigned long long)T->zSY)) return rc;
    if (int rc = encode_map_i8(&T->mapAN, T->AN, (unsigned long long)T->rowsAN, (unsigned long long)T->zAN)) return rc;
    if (int rc = encode_map_i8(&T->mapANc, T->ANc, (unsigned long long)T->rowsAN, (unsigned long long)T->zAN))
        return rc;
    T->i8 = true;
    return SPH_OK;
}

template <int NC>
static int tc_attr() {
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_tcb<SynB<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, tsb::BYTES));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_tcb<AnaB<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, tsb::BYTES));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_tcs<SynS<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, tss::BYTES));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_tcs<AnaS<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, tss::BYTES));
    const int bytes = (int)tc_smem_bytes();
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_tc<SynDir<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_tc<AnaDir<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_i8<SynI8<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, li8::BYTES));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_i8<AnaI8<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, li8::BYTES));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_i8b<SynI8<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, li8b::bytes<NC>()));
    SPH_CUDA_TRY(cudaFuncSetAttribute((const void*)k_legendre_i8b<AnaI8<NC>, NC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, li8b::bytes<NC>()));
    cudaFuncAttributes fa;  // load the preparation kernels now (lazy module loading)
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_i8b_prep<SynI8<NC>, NC>));
    SPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_i8b_prep<AnaI8<NC>, NC>));
    return SPH_OK;
}

static int g_tc_sms = 0;
static int g_tc_group = 1;

int tc_kernels_init() {
    int dev = 0;
    SPH_CUDA_TRY(cudaGetDevice(&dev));
    SPH_CUDA_TRY(cudaDeviceGetAttribute(&g_tc_sms, cudaDevAttrMultiProcessorCount, dev));
    // chunks per FP32 accumulation group: 1 (default, each 16-term chunk folded into FP64) or 2
    if (const char* e = getenv("SPH_TC_GROUP")) g_tc_group = atoi(e) == 2 ? 2 : 1;
    // P_l^m operand: streamed from split-TF32 tables by TMA (default) or
    // regenerated from recurrence checkpoints (SPH_TC_STREAM=0)
    if (const char* e = getenv("SPH_TC_STREAM")) g_tc_stream = atoi(e) != 0;
    // int8 integer-split kernels (default) or only the split-TF32 ones (SPH_TC_I8=0)
    if (const char* e = getenv("SPH_TC_I8")) g_tc_i8 = atoi(e) != 0;
    if (int rc = tc_attr<16>()) return rc;
    if (int rc = tc_attr<32>()) return rc;
    return tc_attr<64>();
}

static TcArgs make_args(const Handle* h, const MixedTables* T, int lmax, int batch, long long ld_spec, long long ldF) {
    TcArgs a;
    a.ab = T->ab;
    a.ck = T->ck;
    a.ckx = T->ckx;
    a.mu = h->mu;
    a.w = h->w;
    a.tlmax = T->lmax;
    a.lmax = lmax;
    a.nh = h->nh;
    a.nhp = T->nhp;
    a.nlat = h->nlat;
    a.batch = batch;
    a.nct = a.nrt = a.ntiles = 0;
    a.group = g_tc_group;
    a.ld_spec = ld_spec;
    a.ldF = ldF;
    a.flag = T->flag;
    return a;
}

static int check_tables(const MixedTables* T, int lmax) {
    if (!T || lmax > T->lmax) {
        set_error("mixed-precision tables are not built for this degree");
        return SPH_ERR_ARG;
    }
    return SPH_OK;
}

// columns per CTA from the batch: 8, 16 or 32 fields
static int tc_cols(int batch) { return batch <= 8 ? 16 : (batch <= 16 ? 32 : 64); }

// column tile of an autotuned variant (bits 0-1: 0 rule, 1: 16, 2: 32, 3: 64)
static int tc_cols_v(int batch, int var) {
    const int c = var & 3;
    return c == 0 ? tc_cols(batch) : (8 << c);
}


template <template <int> class Dir>
static int tc_launch(TcArgs& a, int nrt, int nm, const double2* in, double2* out, int var, cudaStream_t s) {
    const int nc = tc_cols_v(a.batch, var);
    a.nct = (2 * a.batch + nc - 1) / nc;
    a.nrt = nrt;
    a.ntiles = a.nct * nrt * nm;
    const int grid = std::max(1, std::min(a.ntiles, g_tc_sms > 0 ? g_tc_sms : 148));
    const size_t sm = tc_smem_bytes();
    if (nc == 16) k_legendre_tc<Dir<16>, 16><<<grid, tc::NT, sm, s>>>(a, in, out);
    else if (nc == 32) k_legendre_tc<Dir<32>, 32><<<grid, tc::NT, sm, s>>>(a, in, out);
    else k_legendre_tc<Dir<64>, 64><<<grid, tc::NT, sm, s>>>(a, in, out);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

static TsArgs make_sargs(const Handle* h, const MixedTables* T, int lmax, int batch, long long ld_spec, long long ldF) {
    TsArgs a;
    a.soff = T->soff;
    a.aoff = T->aoff;
    a.w = h->w;
    a.tlmax = T->lmax;
    a.lmax = lmax;
    a.nh = h->nh;
    a.nlat = h->nlat;
    a.batch = batch;
    a.nct = a.nrt = a.ntiles = 0;
    a.group = g_tc_group;
    a.ld_spec = ld_spec;
    a.ldF = ldF;
    a.flag = T->flag;
    return a;
}

template <template <int> class Dir>
static int tcs_launch(const CUtensorMap& map, TsArgs& a, int nrt, int nm, const double2* in, double2* out, int var,
                      cudaStream_t s) {
    const int nc = tc_cols_v(a.batch, var);
    a.nct = (2 * a.batch + nc - 1) / nc;
    a.nrt = nrt;
    a.ntiles = a.nct * nrt * nm;
    const int grid = std::max(1, std::min(a.ntiles, g_tc_sms > 0 ? g_tc_sms : 148));
    if (nc == 16) k_legendre_tcs<Dir<16>, 16><<<grid, tss::NT, tss::BYTES, s>>>(map, a, in, out);
    else if (nc == 32) k_legendre_tcs<Dir<32>, 32><<<grid, tss::NT, tss::BYTES, s>>>(map, a, in, out);
    else k_legendre_tcs<Dir<64>, 64><<<grid, tss::NT, tss::BYTES, s>>>(map, a, in, out);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// bytes of prepared B stages for `cols` real columns (a multiple of the tile width)
static size_t tcb_bytes(const Handle* h, bool syn, int lmax, int cols) {
    const int nm = std::min(lmax, h->L) + 1;
    const long long chunks = syn ? tcb_syn_coff(lmax, nm) : (long long)nm * ((h->nh + tc::KC - 1) / tc::KC);
    return (size_t)chunks * (size_t)cols * tc::KC * 4 * sizeof(float);
}

// bytes of the prepared B chunks and column exponents of an int8 call
static size_t i8b_bytes(const Handle* h, bool syn, int lmax, int nct, int nc) {
    const int nm = std::min(lmax, h->L) + 1;
    const long long cpt = syn ? i8b_syn_coff(lmax, nm) : (long long)nm * i8b_ana_nch(h->nh);
    return (size_t)nct * (size_t)cpt * i8b_chunk(nc) + (size_t)nct * nm * nc * sizeof(int);
}

// grow the B buffer; inside a stream capture it must already be large enough
static int tcb_ensure(MixedTables* T, size_t bytes, cudaStream_t s) {
    if (bytes <= T->Bcap) return SPH_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    SPH_CUDA_TRY(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
        set_error("tensor-core Legendre stage: operand workspace not reserved before stream capture");
        return SPH_ERR_ARG;
    }
    // the old buffer is retired, not freed: work in flight and graphs captured
    // earlier may still use it
    float* nb = nullptr;
    SPH_CUDA_TRY(cudaMalloc(&nb, bytes));
    if (T->Bbuf) T->retired.push_back(T->Bbuf);
    T->Bbuf = nb;
    T->Bcap = bytes;
    return SPH_OK;
}

// true if a synthesis of `batch` fields up to degree lmax would grow the
// prepared-B buffer (the loader-only variant chosen by the autotuner for this
// batch, and the buffer not yet large enough)
bool tc_synthesis_needs_alloc(const Handle* h, int lmax, int batch) {
    const MixedTables* T = static_cast<const MixedTables*>(h->mixed);
    if (!T || !T->streamed || batch <= 0) return false;
    const int var = tune_get(h, TUNE_TC_SYNTHESIS, batch, 0);
    if ((var & 16) || (var & 4) || !(var & 8)) return false;
    const int nc = tc_cols_v(batch, var);
    const int nct = (2 * batch + nc - 1) / nc;
    return tcb_bytes(h, true, lmax, nct * nc) > T->Bcap;
}

int tc_reserve(const Handle* h, int batch) {
    MixedTables* T = static_cast<MixedTables*>(h->mixed);
    if (!T || batch <= 0) return SPH_OK;
    const int cols = (2 * batch + 63) / 64 * 64;  // covers every column tile width
    size_t need = 0;
    // the int8 kernels with both operands by TMA (the default) prepare B in the buffer
    if (T->i8) {
        for (int nc : {16, 32, 64}) {
            const int nct = (2 * batch + nc - 1) / nc;
            need = std::max(need, std::max(i8b_bytes(h, true, T->lmax, nct, nc), i8b_bytes(h, false, T->lmax, nct, nc)));
        }
    }
    // so does the split-TF32 loader-only variant (autotuned in)
    bool used = false;
    for (const auto& kv : h->tune) {
        const int kind = (int)(kv.first >> 32), var = kv.second;
        if (kind <= TUNE_TC_ANALYSIS && (var & 8) && !(var & 4)) used = true;
    }
    if (used && T->streamed)
        need = std::max(need, std::max(tcb_bytes(h, true, T->lmax, cols), tcb_bytes(h, false, T->lmax, cols)));
    return need ? tcb_ensure(T, need, nullptr) : SPH_OK;
}

template <int NC>
static int tcb_launch_nc(const Handle* h, MixedTables* T, bool syn, TbArgs& a, const double2* in, long long ld_in,
                         double2* out, const double* wts, cudaStream_t s) {
    constexpr int PART = NC * tc::KC;
    const dim3 pb((PART + 255) / 256);
    if (syn) {
        if (a.csyn > 65535) { set_error("tensor-core Legendre stage: too many chunks"); return SPH_ERR_ARG; }
        k_tcb_prep_syn<NC><<<dim3(pb.x, (unsigned)a.csyn, a.nct), 256, 0, s>>>(in, ld_in, a.lmax, a.batch, a.csyn,
                                                                              T->Bbuf);
    } else {
        if ((long long)a.nm * a.nkA > 65535) { set_error("tensor-core Legendre stage: too many chunks"); return SPH_ERR_ARG; }
        k_tcb_prep_ana<NC><<<dim3(pb.x, a.nm * a.nkA, a.nct), 256, 0, s>>>(in, ld_in, a.nlat, a.nh, a.nm, a.nkA, wts,
                                                                          a.batch, T->Bbuf);
    }
    SPH_CUDA_TRY(cudaGetLastError());
    const int grid = std::max(1, std::min(a.ntiles, g_tc_sms > 0 ? g_tc_sms : 148));
    if (syn) k_legendre_tcb<SynB<NC>, NC><<<grid, tsb::NT, tsb::BYTES, s>>>(T->mapS, a, out);
    else k_legendre_tcb<AnaB<NC>, NC><<<grid, tsb::NT, tsb::BYTES, s>>>(T->mapA, a, out);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// loader-only kernel: prepare B, then run the contraction (in: spectra for
// synthesis, Fourier data for analysis)
static int tcb_launch(const Handle* h, const MixedTables* Tc, bool syn, int lmax, int batch, int nrt, int nm,
                      const double2* in, long long ld_in, double2* out, long long ld_out, int var, cudaStream_t s,
                      const double* wts = nullptr) {
    if (!wts) wts = h->w;
    MixedTables* T = const_cast<MixedTables*>(Tc);
    const int nc = tc_cols_v(batch, var);
    TbArgs a;
    a.soff = T->soff;
    a.aoff = T->aoff;
    a.tlmax = T->lmax;
    a.lmax = lmax;
    a.nh = h->nh;
    a.nlat = h->nlat;
    a.batch = batch;
    a.nct = (2 * batch + nc - 1) / nc;
    a.nrt = nrt;
    a.nm = nm;
    a.ntiles = a.nct * nrt * nm;
    a.group = g_tc_group;
    a.nkA = (h->nh + tc::KC - 1) / tc::KC;
    a.csyn = tcb_syn_coff(lmax, nm);
    a.ld_spec = syn ? ld_in : ld_out;
    a.ldF = syn ? ld_out : ld_in;
    a.flag = T->flag;
    if (int rc = tcb_ensure(T, tcb_bytes(h, syn, lmax, a.nct * nc), s)) return rc;
    a.B = T->Bbuf;
    if (nc == 16) return tcb_launch_nc<16>(h, T, syn, a, in, ld_in, out, wts, s);
    if (nc == 32) return tcb_launch_nc<32>(h, T, syn, a, in, ld_in, out, wts, s);
    return tcb_launch_nc<64>(h, T, syn, a, in, ld_in, out, wts, s);
}

// Variants of the tensor-core Legendre stages (the autotuner's numbers):
//   bits 0-1  column tile: 0 the built-in rule, 1: 16, 2: 32, 3: 64 real columns
//   none of 4, 8, 16, 32   int8 integer-split kernels: both operands by TMA
//             after a B preparation kernel (legendre_i8b.cuh), or with bit 128
//             B staged by producer warps inside the kernel (legendre_i8.cuh);
//             bit 64: m order paired with its complement instead of ascending
//   32        split-TF32, P streamed by TMA, B staged by producer warps
//   8         split-TF32, both operands by TMA (B prepared once per call)
//   4         split-TF32, P regenerated from recurrence checkpoints
//   16        the FP64 tensor-core kernels of the plain form (legendre.cu)
static bool use_i8(const MixedTables* T, int var) { return T->i8 && !(var & (4 | 8 | 16 | 32)); }


// columns per CTA of the int8 kernels: 16 (8 fields) for small batches, else 32
static int i8_cols_v(int batch, int var) {
    const int c = var & 3;
    return c == 0 ? (batch <= 8 ? 16 : 32) : (8 << c);
}

static I8Args make_i8args(const Handle* h, const MixedTables* T, bool syn, int lmax, int batch, long long ld_spec,
                          long long ldF, int var) {
    I8Args a;
    a.erow = syn ? T->esy : T->ean;
    a.zoff = T->i8zoff;
    a.aoff = T->i8aoff;
    a.tlmax = T->lmax;
    a.lmax = lmax;
    a.nh = h->nh;
    a.nlat = h->nlat;
    a.batch = batch;
    a.nm = std::min(lmax, h->L) + 1;
    a.order = (var & 64) ? 1 : 0;
    a.ld_spec = ld_spec;
    a.ldF = ldF;
    a.flag = T->flag;
    a.nct = a.nrt = a.ntiles = 0;
    return a;
}

// the int8 kernels with both operands by TMA: B preparation, then the contraction
template <template <int> class Dir>
static int i8b_launch(const Handle* h, const MixedTables* Tc, bool syn, const CUtensorMap& map, I8Args& a, int nrt,
                      const double2* in, double2* out, int nc, cudaStream_t s) {
    MixedTables* T = const_cast<MixedTables*>(Tc);
    a.nct = (2 * a.batch + nc - 1) / nc;
    a.nrt = nrt;
    a.ntiles = a.nct * nrt * a.nm;
    a.cpt = syn ? i8b_syn_coff(a.lmax, a.nm) : (long long)a.nm * i8b_ana_nch(a.nh);
    if (a.nct > 65535) { set_error("tensor-core Legendre stage: too many column tiles"); return SPH_ERR_ARG; }
    const size_t bbytes = (size_t)a.nct * (size_t)a.cpt * i8b_chunk(nc);
    if (int rc = tcb_ensure(T, i8b_bytes(h, syn, a.lmax, a.nct, nc), s)) return rc;
    a.B = reinterpret_cast<unsigned char*>(T->Bbuf);
    a.ecol = reinterpret_cast<int*>(a.B + bbytes);
    const dim3 pg((unsigned)a.nm, (unsigned)a.nct);
    const int grid = std::max(1, std::min(a.ntiles, g_tc_sms > 0 ? g_tc_sms : 148));
    if (nc == 16) {
        k_i8b_prep<Dir<16>, 16><<<pg, li8b::PREP_NT, 0, s>>>(a, in);
        k_legendre_i8b<Dir<16>, 16><<<grid, li8b::NT, li8b::bytes<16>(), s>>>(map, a, out);
    } else if (nc == 32) {
        k_i8b_prep<Dir<32>, 32><<<pg, li8b::PREP_NT, 0, s>>>(a, in);
        k_legendre_i8b<Dir<32>, 32><<<grid, li8b::NT, li8b::bytes<32>(), s>>>(map, a, out);
    } else {
        k_i8b_prep<Dir<64>, 64><<<pg, li8b::PREP_NT, 0, s>>>(a, in);
        k_legendre_i8b<Dir<64>, 64><<<grid, li8b::NT, li8b::bytes<64>(), s>>>(map, a, out);
    }
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

template <template <int> class Dir>
static int i8_launch(const CUtensorMap& map, I8Args& a, int nrt, const double2* in, double2* out, int nc,
                     cudaStream_t s) {
    a.nct = (2 * a.batch + nc - 1) / nc;
    a.nrt = nrt;
    a.ntiles = a.nct * nrt * a.nm;
    const int grid = std::max(1, std::min(a.ntiles, g_tc_sms > 0 ? g_tc_sms : 148));
    if (nc == 16) k_legendre_i8<Dir<16>, 16><<<grid, li8::NT, li8::BYTES, s>>>(map, a, in, out);
    else if (nc == 32) k_legendre_i8<Dir<32>, 32><<<grid, li8::NT, li8::BYTES, s>>>(map, a, in, out);
    else k_legendre_i8<Dir<64>, 64><<<grid, li8::NT, li8::BYTES, s>>>(map, a, in, out);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

int legendre_synthesis_tc(const Handle* h, const double2* spec, long long ld_spec, int lmax, double2* F, long long ldF,
                          int batch, cudaStream_t s, int nobuf) {
    const MixedTables* T = static_cast<const MixedTables*>(h->mixed);
    if (int rc = check_tables(T, lmax)) return rc;
    if (batch <= 0) return SPH_OK;
    const int nrt = (h->nh + tc::M - 1) / tc::M, nm = std::min(lmax, h->L) + 1;
    const int var = tune_get(h, TUNE_TC_SYNTHESIS, batch, 0);
    if (use_i8(T, var)) {
        I8Args a = make_i8args(h, T, true, lmax, batch, ld_spec, ldF, var);
        const int nrt8 = (h->nh + li8::M - 1) / li8::M;
        if (!(var & 128) && !nobuf)
            return i8b_launch<SynI8>(h, T, true, T->mapSY, a, nrt8, spec, F, i8_cols_v(batch, var), s);
        return i8_launch<SynI8>(T->mapSY, a, nrt8, spec, F, i8_cols_v(batch, var), s);
    }
    if (T->streamed && !(var & 4) && (var & 8))
        return tcb_launch(h, T, true, lmax, batch, nrt, nm, spec, ld_spec, F, ldF, var, s);
    if (T->streamed && !(var & 4)) {
        TsArgs a = make_sargs(h, T, lmax, batch, ld_spec, ldF);
        return tcs_launch<SynS>(T->mapS, a, nrt, nm, spec, F, var, s);
    }
    TcArgs a = make_args(h, T, lmax, batch, ld_spec, ldF);
    return tc_launch<SynDir>(a, nrt, nm, spec, F, var, s);
}

int legendre_analysis_tc(const Handle* h, const double2* F, long long ldF, double2* spec, long long ld_spec, int lmax,
                         int batch, cudaStream_t s, int wmode) {
    const MixedTables* T = static_cast<const MixedTables*>(h->mixed);
    if (int rc = check_tables(T, lmax)) return rc;
    if (batch <= 0) return SPH_OK;
    const int nrt = lmax / (2 * tc::M) + 1, nm = std::min(lmax, h->L) + 1;
    const int var = tune_get(h, TUNE_TC_ANALYSIS, batch, 0);
    const double* wts = wmode ? h->wc : h->w;
    if (use_i8(T, var)) {
        I8Args a = make_i8args(h, T, false, lmax, batch, ld_spec, ldF, var);
        if (wmode) a.erow = T->eanc;
        const CUtensorMap& map = wmode ? T->mapANc : T->mapAN;
        const int nrt8 = (i8_nlp(lmax, 0, 0) + li8::M - 1) / li8::M;
        if (!(var & 128)) return i8b_launch<AnaI8>(h, T, false, map, a, nrt8, F, spec, i8_cols_v(batch, var), s);
        return i8_launch<AnaI8>(map, a, nrt8, F, spec, i8_cols_v(batch, var), s);
    }
    if (T->streamed && !(var & 4) && (var & 8))
        return tcb_launch(h, T, false, lmax, batch, nrt, nm, F, ldF, spec, ld_spec, var, s, wts);
    if (T->streamed && !(var & 4)) {
        TsArgs a = make_sargs(h, T, lmax, batch, ld_spec, ldF);
        a.w = wts;
        return tcs_launch<AnaS>(T->mapA, a, nrt, nm, F, spec, var, s);
    }
    TcArgs a = make_args(h, T, lmax, batch, ld_spec, ldF);
    a.w = wts;
    return tc_launch<AnaDir>(a, nrt, nm, F, spec, var, s);
}

int tc_check(const Handle* h) {
    const MixedTables* T = static_cast<const MixedTables*>(h->mixed);
    if (!T) return SPH_OK;
    int flag = 0;
    SPH_CUDA_TRY(cudaMemcpy(&flag, T->flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        // reported once: the flag is cleared so that the handle stays usable
        SPH_CUDA_TRY(cudaMemset(T->flag, 0, sizeof(int)));
        set_error("tensor-core Legendre stage: a bounded wait gave up");
        return SPH_ERR_TIMEOUT;
    }
    return SPH_OK;
}

int tc_wait_selftest(const Handle* h, double seconds, cudaStream_t s) {
    const MixedTables* T = static_cast<const MixedTables*>(h->mixed);
    if (!T) {
        set_error("sph_wait_selftest: the bounded waits belong to the tensor-core kernels of a mixed handle");
        return SPH_ERR_ARG;
    }
    if (!(seconds > 0.0 && seconds <= 10.0)) {
        set_error("sph_wait_selftest: the limit must lie in (0, 10] seconds");
        return SPH_ERR_ARG;
    }
    k_wait_selftest<<<1, 32, 0, s>>>((unsigned long long)(seconds * 1e9), T->flag);
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

}  // namespace sphgpu
