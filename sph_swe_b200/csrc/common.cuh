// Shared definitions of the sm_100a spectral shallow-water library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <map>
#include <string>
#include <vector>

#include "../../include/sph_gpu.h"

namespace sphgpu {

constexpr double kPi = 3.14159265358979323846264338327950288;

#define SPH_CUDA_TRY(expr)                                                    \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) {                                              \
            set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));    \
            return SPH_ERR_CUDA;                                              \
        }                                                                     \
    } while (0)

void set_error(const std::string& msg);
const char* get_error();

// packed real layout for degree lmax: m-major, n contiguous from n = m
__host__ __device__ inline int pidx(int lmax, int n, int m) { return ((m * (2 * lmax - m + 1)) >> 1) + n; }
// complex layout n*n + n + m
__host__ __device__ inline int cidx(int n, int m) { return n * n + n + m; }

// FFT plan for one ring length (device twiddles exp(-2 pi i t / n))
struct FFTPlan {
    int n = 0;
    int nrad = 0;
    int rad[16] = {0};
    double2* tw = nullptr;  // device, n entries
};

// Per-handle state.  All arrays are device-resident.
struct Handle {
    int L = 0, nlat = 0, nphi = 0, nh = 0, nlm = 0, ncplx = 0, nspat = 0;
    int flags = 0;
    int device = 0;
    double* mu = nullptr;       // nlat
    double* w = nullptr;        // nlat
    double* wc = nullptr;       // nlat: w / cos(phi)
    double* cosphi = nullptr;   // nlat
    double* lat = nullptr;      // nlat
    // P_l^m(mu_j), j < nh, m = 0..L+1, l = m..L+1 at plm[poff[m] + (l-m)*nh + j]
    double* plm = nullptr;
    std::vector<long long> poff_h;
    long long* poff = nullptr;  // device copy, L+3 entries
    FFTPlan fft;
    // mixed-precision Legendre state (legendre_tc.cu): recurrence checkpoints, error flag
    void* mixed = nullptr;
    // RK4 buffers and captured step graph (swe.cu)
    void* rk = nullptr;
    // autotuned kernel variants: key (kind << 32 | batch) -> variant (tune.cu)
    std::map<long long, int> tune;
    // workspace (Fourier-space buffer and grids)
    void* ws = nullptr;
    size_t ws_bytes = 0;
    cudaStream_t last_stream = nullptr;
    // host copies of the grid
    std::vector<double> mu_h, w_h, cosphi_h, lat_h;
};

int ensure_workspace(Handle* h, size_t bytes);
// device address of the fixed scratch array of sph_SH_to_spat_noalloc on
// device dev (the current device); the first call per device loads the
// array's module, which reserves its memory (noalloc.cu)
int noalloc_scratch(int dev, void** out);

// kernel variants chosen by the autotuner (tune.cu); 0 = the built-in rule
enum TuneKind { TUNE_TC_SYNTHESIS = 0, TUNE_TC_ANALYSIS = 1, TUNE_RING_ANALYSIS = 2, TUNE_RING_SYNTHESIS = 3 };
inline int tune_get(const Handle* h, int kind, int batch, int dflt) {
    if (h->tune.empty()) return dflt;
    const auto it = h->tune.find(((long long)kind << 32) | (unsigned)batch);
    return it == h->tune.end() ? dflt : it->second;
}
void rk_free(Handle* h);        // swe.cu
void rk_invalidate(Handle* h);  // swe.cu: the next RK4 call re-captures its step graph

// ---- kernels launched by the C-ABI layer (stream-ordered)
int setup_tables(Handle* h);
int fft_kernels_init();
int fft_plan_init(FFTPlan* p, int n);
void fft_plan_free(FFTPlan* p);

// Fourier buffer layout: F[f][m][j] complex, m = 0..mF-1 (real) or
// (m+L) for m = -L..L (complex), j = 0..nlat-1; per-field stride ldF complex.

// grid (real) -> Fourier, m = 0..mF-1 kept (m > L zero)
int ring_analysis_real(const Handle* h, const double* spat, long long ld_spat, double2* F, long long ldF, int mF,
                       int batch, cudaStream_t s);
// Fourier -> grid (real).  Optional output map (HOST arrays of length
// period <= 16, batch a multiple of period): output k of member k/period reads
// Fourier field (k/period)*src_stride + src[k%period], modified by mod[k%period]
// (0 plain, 1 multiply by i*m, i.e. d/dlambda).  src = NULL: output k reads field k.
// rowdiv (optional): ring j of every output is multiplied by 1 / rowdiv[j]
// after the transform (the 1 / cos phi of velocities from U = u cos phi).
int ring_synthesis_real(const Handle* h, const double2* F, long long ldF, int mF, double* spat, long long ld_spat,
                        int batch, const int* src, const int* mod, int period, int src_stride, cudaStream_t s,
                        const double* rowdiv = nullptr);
int ring_analysis_cplx(const Handle* h, const double2* spat, long long ld_spat, double2* F, long long ldF, int batch,
                       cudaStream_t s);
int ring_synthesis_cplx(const Handle* h, const double2* F, long long ldF, double2* spat, long long ld_spat, int batch,
                        cudaStream_t s);

// Legendre stage (FP64).  Real: spectral packed for degree lmax (L or L+1),
// m = 0..min(lmax, L).  Complex: m = -L..L, layout n*n+n+m.
int legendre_kernels_init();  // loads the FP64 Legendre kernels (lazy module loading)
// exact_m0 != 0 (mixed handles): the orders m = 0 and 1 in FP64 after the
// tensor-core stage.  For spectra of Robert velocities U = u cos(phi): near the
// poles their m = 0 part vanishes like cos(phi)^2 while each term P_l^0 does
// not, and their m = 1 part is O(cos(phi)) while the largest term of a row
// grows like l^1.5 cos(phi); the mixed form's error, relative to the terms,
// would become a large relative error of u = U / cos(phi) at the polar rings.
// Orders m >= 2 keep the mixed form's accuracy.
// nobuf != 0: no kernel variant that needs the handle's prepared-operand
// buffer (which a call may grow): the int8 kernel that stages B itself
int legendre_synthesis_real(const Handle* h, const double2* spec, long long ld_spec, int lmax, double2* F,
                            long long ldF, int batch, cudaStream_t s, int exact_m0 = 0, int nobuf = 0);
// wmode 0: Gauss weights; 1: Gauss weights / cos(phi) -- the input then holds
// cos(phi) times the integrand (e.g. u / cos(phi) analysed from u), which keeps
// it bounded at the polar rings, where the mixed form's per-column scales would
// otherwise be set by a 1/cos(phi) growth; on mixed handles these analyses of
// velocity-derived fields also take the orders m = 0, 1 in FP64
int legendre_analysis_real(const Handle* h, const double2* F, long long ldF, double2* spec, long long ld_spec,
                           int lmax, int batch, cudaStream_t s, int wmode = 0);
int legendre_synthesis_cplx(const Handle* h, const double2* spec, long long ld_spec, double2* F, long long ldF,
                            int batch, cudaStream_t s);
int legendre_analysis_cplx(const Handle* h, const double2* F, long long ldF, double2* spec, long long ld_spec,
                           int batch, cudaStream_t s);

// Legendre stage of the mixed-precision form on tcgen05 (legendre_tc.cu), real layout only
int tc_kernels_init();
int tc_tables_build(Handle* h, int lmax);
void tc_tables_free(Handle* h);
int tc_check(const Handle* h);
int tc_wait_selftest(const Handle* h, double seconds, cudaStream_t s);
// reserve the tensor-core operand workspace for calls of up to `batch` fields
// (before a stream capture, which cannot allocate)
int tc_reserve(const Handle* h, int batch);
bool tc_synthesis_needs_alloc(const Handle* h, int lmax, int batch);
int legendre_synthesis_tc(const Handle* h, const double2* spec, long long ld_spec, int lmax, double2* F, long long ldF,
                          int batch, cudaStream_t s, int nobuf = 0);
int legendre_analysis_tc(const Handle* h, const double2* F, long long ldF, double2* spec, long long ld_spec, int lmax,
                         int batch, cudaStream_t s, int wmode = 0);

// spectral operators (packed real or complex layout)
int spec_copy_modes(const Handle* hs, const double2* src, long long lds, const Handle* hd, double2* dst,
                    long long ldd, int batch, cudaStream_t s);
int spec_op(const Handle* h, int op, const double2* in, long long ld_in, double2* out, long long ld_out, double2 a,
            double2 b, int batch, int cplx, cudaStream_t s);

}  // namespace sphgpu
