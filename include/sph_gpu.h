/*
 * sph_gpu.h — C ABI of the B200 (sm_100a) spectral shallow-water library
 * (libsphgpu.so).
 *
 * Drop-in boundary for the hot path of schreiberx/sph_swe.  Every entry point
 * replaces one call the reference makes into SHTNS 2.6.6 (spherical-harmonic
 * transforms), LAPACK 3.6.1 (zgbsv) or one of its own spectral-space loops;
 * the replaced interface is cited beside each declaration (paths relative to
 * the reference's src/ directory).
 *
 * Conventions (identical to the reference):
 *   grid            double[nphi*nlat], index i_lon*nlat + j_lat, j = 0 nearest
 *                   the north pole, mu_j = sin(latitude) decreasing
 *                   (SHT_THETA_CONTIGUOUS, SPHConfig.hpp:344,390);
 *                   longitude lambda_i = 2*pi*i/nphi.
 *   real spectral   complex (double2) packed m-major, n contiguous:
 *                   index (m*(2L-m+1))/2 + n, m = 0..L, n = m..L
 *                   (SPHConfig::getArrayIndexByModes, SPHConfig.hpp:106-116).
 *   complex spectral index n*n + n + m, m = -n..n
 *                   (getArrayIndexByModes_Complex, SPHConfig.hpp:120-130).
 *   normalisation   orthonormal spherical harmonics with Condon-Shortley
 *                   phase (sht_orthonormal, SPHConfig.hpp:338); real fields
 *                   f = sum_l Q_l0 Y_l0 + 2 Re sum_{m>0} Q_lm Y_lm; complex
 *                   fields use Y_l^{-m} = (-1)^m conj(Y_l^m).
 *
 * All pointers passed to compute entry points are DEVICE pointers; all work
 * is ordered on the given stream (cudaStream_t passed as void*; NULL = the
 * legacy default stream).  Every function returns SPH_OK (0) or an error
 * code; sph_last_error() describes the last failure of the calling process.
 * Handles are not thread safe: use one handle per host thread.
 * The library has no CPU fallback: if no sm_100 device is present, every
 * compute entry point fails with SPH_ERR_CUDA.
 */
#ifndef SPH_GPU_H_
#define SPH_GPU_H_

#ifdef __cplusplus
extern "C" {
#endif

enum sph_status {
    SPH_OK = 0,
    SPH_ERR_ARG = 1,       /* invalid argument (sizes, layouts, null pointers) */
    SPH_ERR_CUDA = 2,      /* CUDA runtime error or no usable device           */
    SPH_ERR_SINGULAR = 3,  /* zero pivot in a banded solve (zgbsv INFO > 0)    */
    SPH_ERR_NAN = 4,       /* non-finite value detected in the state           */
    SPH_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up               */
    SPH_ERR_NOMEM = 6      /* device allocation failed                         */
};

/* precision forms (flags of sph_create) */
enum sph_precision {
    SPH_PREC_FP64 = 0,     /* plain method: FP64 everywhere                      */
    SPH_PREC_MIXED = 1     /* Legendre GEMMs on tcgen05 (split-TF32, FP32 chunk
                              sums added in FP64); everything else FP64         */
};

typedef struct sph_handle sph_handle;
typedef struct sph_rexi sph_rexi;
typedef struct sph_ensemble sph_ensemble;

/* ---------------------------------------------------------------- setup */

/* Create a transform handle for triangular truncation lmax == mmax on an
 * nlat x nphi Gauss-Legendre grid.  nlat <= 0 or nphi <= 0 chooses the grid by
 * the quadratic (3/2) rule: nphi = smallest 7-smooth integer >= 3*mmax+1,
 * nlat = 3*lmax/2+1 rounded up to even.  Gauss nodes, weights and the P_l^m
 * table are computed on the device in FP64.
 * Replaces shtns_create + shtns_set_grid (SPHConfig::setup, SPHConfig.hpp:324-352)
 * and shtns_set_grid_auto (SPHConfig::setupAutoPhysicalSpace, SPHConfig.hpp:366-399). */
int sph_create(int lmax, int mmax, int nlat, int nphi, int flags, sph_handle** out);

/* Release a handle (shtns_destroy, SPHConfig::shutdown, SPHConfig.hpp:421-446). */
int sph_destroy(sph_handle* h);

/* Sizes: lmax, nlat, nphi, nlm = (L+1)(L+2)/2, ncplx = (L+1)^2 (any may be NULL).
 * Replaces the shtns_cfg fields read in SPHConfig::setup_data (SPHConfig.hpp:160-168). */
int sph_info(const sph_handle* h, int* lmax, int* nlat, int* nphi, int* nlm, int* ncplx);

/* Host copies of mu_j (sin latitude, = SHTNS ct), cos(latitude) (= SHTNS st),
 * Gauss weights and latitude angles, nlat each (any may be NULL).
 * Replaces lat_gaussian / lat_cogaussian / lat (SPHConfig.hpp:303-319). */
int sph_grid(const sph_handle* h, double* mu, double* cosphi, double* w, double* lat);

/* ---------------------------------------------------------------- transforms */

/* Real analysis, batch fields: spat[b*ld_spat + .] -> spec[b*ld_spec + .]
 * (strides in doubles / double2; <= 0 means dense).
 * Replaces spat_to_SH(shtns, double* Vr, cplx* Qlm) (SPHData.hpp:201,509,527). */
int sph_spat_to_SH(sph_handle* h, const double* spat, double* spec, int batch, long long ld_spat,
                   long long ld_spec, void* stream);

/* Real synthesis.  Replaces SH_to_spat(shtns, cplx* Qlm, double* Vr)
 * (SPHData.hpp:221,510,526). */
int sph_SH_to_spat(sph_handle* h, const double* spec, double* spat, int batch, long long ld_spec,
                   long long ld_spat, void* stream);

/* Real synthesis that performs no device allocation.  No counterpart in the
 * reference: it exists for callers that cannot have cudaMalloc called once
 * they are running (their own allocator has reserved the device memory, or a
 * cudaMalloc/cudaFree synchronisation would break their latency budget).
 * Same result as sph_SH_to_spat on dense arrays (spec: batch*nlm complex,
 * spat: batch*nphi*nlat doubles).  The Fourier intermediate lives in a fixed
 * 8 MiB device array inside the library, shared by all calls: batch is
 * limited to 8 MiB / ((L+1)*nlat*16 bytes) fields (5 at T255, 85 at T63) and
 * larger batches fail with SPH_ERR_ARG.  The array is reserved on a device,
 * and its device address looked up, when the first handle is created on that
 * device (sph_create, where allocating is still allowed); the device keeps it
 * until the process exits, and this entry point only reuses it.
 * Calls that overlap on the GPU (other streams, other host threads) race on
 * the shared array: serialise them.  A mixed handle whose autotuned synthesis
 * variant for this batch is the loader-only tensor-core kernel needs a
 * per-handle operand buffer that only an allocating call grows: until one
 * sph_SH_to_spat with this batch has run, the call fails with SPH_ERR_ARG
 * rather than allocate. */
int sph_SH_to_spat_noalloc(sph_handle* h, const double* spec, double* spat, int batch, void* stream);

/* Complex analysis / synthesis on complex grids (double2[nphi*nlat]) and
 * (L+1)^2 complex coefficients.  Replace spat_cplx_to_SH / SH_to_spat_cplx
 * (SPHDataComplex.hpp:190,210,469-470,486-487). */
int sph_cplx_spat_to_SH(sph_handle* h, const double* spat, double* spec, int batch, long long ld_spat,
                        long long ld_spec, void* stream);
int sph_cplx_SH_to_spat(sph_handle* h, const double* spec, double* spat, int batch, long long ld_spec,
                        long long ld_spat, void* stream);

/* Vector pair: vorticity/divergence spectra (real layout, unit sphere)
 * -> velocity grids u (eastward), v (northward):
 *   psi = lap^-1 vort, chi = lap^-1 div,
 *   u*cos(phi) = d chi/d lambda - (1-mu^2) d psi/d mu,
 *   v*cos(phi) = d psi/d lambda + (1-mu^2) d chi/d mu,
 * with the exact (degree L+1 retained) meridional derivative.  robert != 0
 * returns (u cos phi, v cos phi).  The reference has no inverse vector
 * transform; the forward direction replaces SPHOperators::vort/div
 * (SPHOperators.hpp:507-529) applied to (u, v). */
int sph_vec_SH_to_spat(sph_handle* h, const double* vort, const double* div, double* u, double* v, int batch,
                       int robert, void* stream);
int sph_vec_spat_to_SH(sph_handle* h, const double* u, const double* v, double* vort, double* div, int batch,
                       int robert, void* stream);

/* Legendre stage alone (per-m contraction with P_l^m at the Gauss nodes), for
 * callers that run their own longitude stage or profile the stages apart.
 * Fourier buffer four: double2[batch][L+1][nlat], F_m(mu_j) at
 * four[b*(L+1)*nlat + m*nlat + j], with the analysis convention
 * F_m = (2 pi / nphi) sum_i f(lambda_i) e^{-i m lambda_i}; the synthesis writes
 * F_m without that factor, so that f = sum_m (2 - delta_m0) Re(F_m e^{i m lambda}).
 * These are the Legendre halves of SHTNS spat_to_SH / SH_to_spat
 * (SPHData.hpp:201,221). */
int sph_legendre_synthesis(sph_handle* h, const double* spec, double* four, int batch, void* stream);
int sph_legendre_analysis(sph_handle* h, const double* four, double* spec, int batch, void* stream);

/* Copy batch real packed spectra of handle hs (truncation Ls) into the layout
 * of handle hd (truncation Ld): coefficients with n <= min(Ls, Ld) are
 * copied, the rest of dst is zero.  Dense batches (nlm of each handle per
 * field).  Replaces SPHData::spec_copyToDifferentModes (SPHData.hpp:108-187),
 * which the REXI extended-modes option (sh_example X<k>, AppSWE.hpp:338-350,
 * 434-445, 524-535) uses to run the REXI step at truncation L+k. */
int sph_spec_copy_modes(const sph_handle* hs, const double* src, const sph_handle* hd, double* dst, int batch,
                        void* stream);

/* ---------------------------------------------------------------- spectral operators */

enum sph_spec_op_id {
    SPH_OP_DIFF_LON = 0,   /* x i m                          SPHOperators::diff_lon (SPHOperators.hpp:30-54) */
    SPH_OP_D1MU2 = 1,      /* truncated (1-mu^2) d/dmu       spec_one_minus_mu_squared_diff_lat_mu (:234-260) */
    SPH_OP_MU = 2,         /* mu x (Galerkin)                SPHOperators::mu (:268-297)          */
    SPH_OP_MU2 = 3,        /* mu^2 x (Galerkin)              SPHOperators::mu2 (:303-333)         */
    SPH_OP_LAPLACE = 4,    /* -n(n+1) x                      SPHOperators::laplace (:482-498)     */
    SPH_OP_HELMHOLTZ = 5,  /* x / (a - b n(n+1)), b = b_ref / r^2  spec_solve_helmholtz (SPHData.hpp:475-497) */
    SPH_OP_SCALE = 6,      /* a x                            SPHData operator*(double/complex)    */
    SPH_OP_AXPY = 7        /* out = out + a x                SPHData operator+= with scaling      */
};

/* Apply a spectral-space operator to batch fields.  cplx = 0: real packed
 * layout (nlm entries), cplx = 1: complex layout ((L+1)^2 entries).
 * a = (a_re, a_im), b = (b_re, b_im) are operator arguments: SCALE/AXPY use a;
 * HELMHOLTZ computes x / (a - b*n(n+1)) (the caller folds r^2 into b), as
 * SPHData::spec_solve_helmholtz (SPHData.hpp:475-497) and
 * SPHDataComplex::spec_solve_helmholtz (SPHDataComplex.hpp:523-545).
 * in == out is allowed for the pointwise operators (DIFF_LON, LAPLACE,
 * HELMHOLTZ, SCALE, AXPY) but not for the recurrences (D1MU2, MU, MU2). */
int sph_spec_op(sph_handle* h, int op, const double* in, double* out, double a_re, double a_im, double b_re,
                double b_im, int batch, int cplx, void* stream);

/* ---------------------------------------------------------------- SWE */

typedef struct sph_swe_params {
    double radius;     /* a     (SimVars::earth_radius)     */
    double gravity;    /* g     (SimVars::gravitation)      */
    double omega;      /* Omega (SimVars::coriolis_omega)   */
    double h0;         /* mean depth (SimVars::h0)          */
    double viscosity;  /* nu    (SimVars::viscosity2)       */
    double dt;         /* time step (current_timestep_size) */
    int nonlinear;     /* SimVars::use_nonlinear_equations: 0 linear, 1 the
                          reference's nonlinear advective form (robert is then
                          ignored, as AppSWE.hpp:622-650 does), 2 the full
                          nonlinear equations in vorticity-divergence form
                          with Robert velocities on the grid (new form; the
                          state is then [h | vorticity | divergence])        */
    int robert;        /* SimVars::use_robert_functions     */
} sph_swe_params;

/* One SWE tendency evaluation: state = [h | u | v] spectral (3*nlm complex,
 * contiguous) -> tend = [h_t | u_t | v_t].  Follows the projection points of
 * AppSWE::p_run_euler_timestep_update (AppSWE.hpp:574-659). */
int sph_swe_tendency(sph_handle* h, const sph_swe_params* p, const double* state, double* tend, void* stream);

/* nsteps classical RK4 steps in place on state = [h | u | v] (3*nlm complex;
 * [h | vorticity | divergence] with nonlinear = 2),
 * as TimesteppingRK::run_rk_timestep order 4 (TimesteppingRK.hpp:310-392)
 * driven by AppSWE::run (AppSWE.hpp:293-336).  The step is captured once in a
 * CUDA graph and replayed.  Returns SPH_ERR_NAN if h became non-finite
 * (AppSWE.hpp:322-327). */
int sph_swe_rk4(sph_handle* h, const sph_swe_params* p, double* state, int nsteps, void* stream);

/* kernel launches in one replay of the handle's captured RK4 step graph (0
 * before the first sph_swe_rk4 / sph_swe_rk4_batched call) */
int sph_swe_rk4_launches(const sph_handle* h);

/* Batched ensemble: nmem independent members, state of member k at
 * state + 3*nlm*k (complex), all with the same handle and parameters except
 * dt_k = dts[k] (host array, may be NULL = p->dt). */
int sph_swe_rk4_batched(sph_handle* h, const sph_swe_params* p, const double* dts, double* state, int nmem,
                        int nsteps, void* stream);

/* Ensemble of uneven truncations advanced by one CUDA graph.  Group g holds
 * nmem[g] members of truncation handles[g]; member k of group g has its state
 * [h | u | v] (3*nlm complex) at states[g] + 6*nlm*k doubles and its own
 * dt = dts[g][k] (dts or dts[g] may be NULL: params[g].dt).  The step of every
 * group is captured once, each group on its own graph branch; one replay
 * advances all members by one RK4 step.  The reference runs one AppSWE::run
 * (AppSWE.hpp:293-336) per member; the member arithmetic is that of
 * sph_swe_rk4_batched.  The state pointers are bound at creation. */
int sph_ensemble_create(int ngroups, sph_handle* const* handles, const sph_swe_params* params, double* const* states,
                        const int* nmem, const double* const* dts, sph_ensemble** out);
/* nsteps graph replays on stream; SPH_ERR_NAN names the groups whose h became
 * non-finite. */
int sph_ensemble_step(sph_ensemble* e, int nsteps, void* stream);
/* kernel launches in one replay of the step graph */
int sph_ensemble_launches(const sph_ensemble* e);
int sph_ensemble_destroy(sph_ensemble* e);

/* ---------------------------------------------------------------- REXI */

typedef struct sph_rexi_params {
    double radius, gravity, omega, h0, viscosity, tau;
    int robert;        /* SWERexiSPHRobert (1) or SWERexiSPH (0)            */
    int coriolis;      /* include_coriolis_effect                           */
    int fix_z5robert;  /* 0: reproduce SPHSolverComplex.hpp:305-309 as written */
    int precision;     /* SPH_PREC_FP64 direct, SPH_PREC_MIXED (complex FP32
                          factor/solve + FP64 iterative refinement)          */
    int factor_each_step; /* 1: never keep the factors of the banded systems
                          (FP64 form) but factor them in every step, as the
                          reference does; for plans of one or a few poles,
                          whose stored factors would cost more memory than
                          their steps cost time.  0 (zero-initialised): keep
                          them when they fit (see sph_rexi_create)          */
} sph_rexi_params;

/* Prepare a REXI integrator for npoles poles alpha[k], beta[k] (host arrays of
 * interleaved complex).  Replaces the per-pole SWERexiSPH[Robert]::setup loop
 * (AppSWE.hpp:381-412, SWERexiSPH.hpp:68-130, SWERexiSPHRobert.hpp:68-132).
 * p->robert = 0 selects the non-Robert form (state [h | u | v]); it keeps, per
 * pole, phi and the spectra of its two grid-valued gradients plus their
 * Fourier buffer (about 16 * npoles * ((L+1)^2 * 3 + 2 (2L+1) nlat) bytes:
 * 1.1 GB at T127 with 535 poles).  With SPH_PREC_FP64 and
 * the Coriolis term, every banded system (pole x m x parity) is factored here
 * once and its factors are kept on the device (178 bytes per block row and
 * pole: 1.6 GB at T127 with 535 poles) if they fit in half the free device
 * memory; each sph_rexi_step then only substitutes.  A zero pivot met while
 * factoring is reported by the first sph_rexi_step (SPH_ERR_SINGULAR), as when
 * factoring per step.  Environment SPH_REXI_STORE=0: factor every step. */
int sph_rexi_create(sph_handle* h, const double* alpha, const double* beta, int npoles, const sph_rexi_params* p,
                    sph_rexi** out);
int sph_rexi_destroy(sph_rexi* r);

/* REXI coefficients (host computation, no device needed): poles alpha and the
 * weights beta_re / beta_im of e^{ix} ~ sum_n beta_n / (ix + alpha_n), from the
 * L = 11 Gaussian approximation with step h and M terms (N = M + 11 poles each
 * side; half != 0 keeps n = -N..0 with doubled weights).  alpha, beta_re and
 * beta_im are interleaved complex arrays of capacity cap; *npoles receives the
 * pole count (cap = 0 and NULL arrays: size query).
 * Replaces REXI::setup (rexi/REXI.hpp:52-131). */
int sph_rexi_coefficients(double h, int M, int half, int cap, double* alpha, double* beta_re, double* beta_im,
                          int* npoles);

/* nsteps REXI steps in place on state = [h | u | v] (3*nlm complex): all poles
 * x all m x both l-parities are solved in one launch per step (the non-Robert
 * form: one launch for phi, one batched transform pair for its gradients, one
 * launch for the velocities); replaces the serial pole loop of AppSWE::run
 * (AppSWE.hpp:414-566) with SWERexiSPH[Robert]::solve (SWERexiSPH.hpp:137-244,
 * SWERexiSPHRobert.hpp:139-258) and
 * SPHSolverComplex::solve -> zgbsv (SPHSolverComplex.hpp:462-511,
 * BandedMatrixSolver.hpp:416-427). */
int sph_rexi_step(sph_rexi* r, double* state, int nsteps, void* stream);

/* ---------------------------------------------------------------- grid arithmetic */

/* elementwise grid operations of sph_spat_op */
enum sph_spat_op_kind {
    SPH_SPAT_MUL = 0,        /* out = alpha * x * y                              */
    SPH_SPAT_AXPBY = 1,      /* out = alpha * x + beta * y   (y may be NULL)     */
    SPH_SPAT_FILL = 2,       /* out = alpha                                      */
    SPH_SPAT_ADD_CONST = 3,  /* out = x + alpha                                  */
    SPH_SPAT_CMUL = 4        /* complex: out = alpha * x * y, n complex elements */
};

/* n elements (doubles; complex elements for SPH_SPAT_CMUL) on the stream; in
 * place allowed.  The grid arithmetic of SPHData / SPHDataComplex: the grid
 * product operator* (SPHData.hpp:334-353, SPHDataComplex.hpp:321-340) and the
 * scalar grid updates spat_set_value / spat_set_zero (SPHData.hpp:768-798). */
int sph_spat_op(sph_handle* h, int op, const double* x, const double* y, double* out, double alpha, double beta,
                long long n, void* stream);

/* ---------------------------------------------------------------- autotuner */

/* Time the kernel variants of the handle for `batch` fields per launch on
 * `stream` and keep the fastest for every later call with that batch: the
 * column tile (8, 16 or 32 fields per CTA) and P_l^m source (streamed table
 * or regenerated) of the tensor-core Legendre stages of a mixed handle, or
 * the FP64 Legendre kernel in their place where that is faster (variant 16),
 * and the rings per CTA of the fixed-length ring FFTs.  json (optional, capacity
 * cap bytes) receives the table with every candidate's time.  Variants are
 * exact alternatives (no change of arithmetic beyond the last bits of
 * P_l^m).  A captured RK4 graph of the handle is re-captured on its next
 * call; ensembles take the variants in force at sph_ensemble_create.  No
 * counterpart in the reference (SHTNS picks its own algorithm at
 * shtns_set_grid, SPHConfig.hpp:324-352). */
int sph_autotune(sph_handle* h, int batch, char* json, int cap, void* stream);
/* Kernel families of sph_autotune_ex (bit mask).  sph_autotune takes
 * SPH_TUNE_INT8 | SPH_TUNE_FP64: the families whose transforms of
 * velocity-derived fields stay within the mixed form's relL2 <= 1e-6; the
 * split-TF32 family (~3e-7 per transform) meets it for scalar fields only. */
enum sph_tune_family { SPH_TUNE_INT8 = 1, SPH_TUNE_TF32 = 2, SPH_TUNE_FP64 = 4 };
/* sph_autotune over the given kernel families of the tensor-core Legendre
 * stages (the ring-FFT tile widths are always timed). */
int sph_autotune_ex(sph_handle* h, int batch, int families, char* json, int cap, void* stream);
/* Re-apply a table written by sph_autotune (same truncation, grid, precision). */
int sph_tune_load(sph_handle* h, const char* json);
/* Back to the built-in rules. */
int sph_tune_clear(sph_handle* h);

/* ---------------------------------------------------------------- errors */

/* Wait for the stream and report device-side failures of the handle's kernels
 * (a bounded wait inside a tensor-core kernel that gave up: SPH_ERR_TIMEOUT).
 * No counterpart in the reference, whose CPU path has no asynchronous errors. */
int sph_sync(sph_handle* h, void* stream);

/* Diagnostic of the failure path of the bounded device-side waits (mixed
 * handles only): launches one block that waits, with the same bounded wait as
 * the tensor-core Legendre kernels, for a barrier that nothing completes.  The
 * wait gives up after `seconds` (0 < seconds <= 10) and records the failure
 * in the handle exactly as a timed-out kernel would, so the next sph_sync
 * returns SPH_ERR_TIMEOUT (once: the record is then cleared) and the CUDA
 * context stays usable.  No counterpart in the reference. */
int sph_wait_selftest(sph_handle* h, double seconds, void* stream);

/* Copy the message of the last error into buf (NUL terminated); returns its length. */
int sph_last_error(char* buf, int n);

#ifdef __cplusplus
}
#endif

#endif /* SPH_GPU_H_ */
