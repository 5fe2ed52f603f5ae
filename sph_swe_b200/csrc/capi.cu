// C ABI of libsphgpu.so (declarations and the replaced reference interfaces
// are in include/sph_gpu.h).
#include "common.cuh"

#include <cstdio>
#include <cstring>
#include <mutex>

struct sph_handle : public sphgpu::Handle {};

namespace sphgpu {

static std::mutex g_err_mu;
static std::string g_err;

void set_error(const std::string& msg) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
}
const char* get_error() { return g_err.c_str(); }

int ensure_workspace(Handle* h, size_t bytes) {
    if (bytes <= h->ws_bytes) return SPH_OK;
    if (h->ws) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            set_error(std::string("workspace sync: ") + cudaGetErrorString(e));
            return SPH_ERR_CUDA;
        }
        cudaFree(h->ws);
        h->ws = nullptr;
        h->ws_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&h->ws, bytes);
    if (e != cudaSuccess) {
        set_error(std::string("workspace allocation: ") + cudaGetErrorString(e));
        return SPH_ERR_NOMEM;
    }
    h->ws_bytes = bytes;
    return SPH_OK;
}

static bool smooth7(int n) {
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}

}  // namespace sphgpu

using namespace sphgpu;

static inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

int sph_last_error(char* buf, int n) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    const int len = (int)g_err.size();
    if (buf && n > 0) {
        const int c = len < n - 1 ? len : n - 1;
        std::memcpy(buf, g_err.data(), c);
        buf[c] = 0;
    }
    return len;
}

int sph_create(int lmax, int mmax, int nlat, int nphi, int flags, sph_handle** out) {
    if (!out) { set_error("sph_create: out is NULL"); return SPH_ERR_ARG; }
    *out = nullptr;
    if (lmax < 1 || mmax != lmax) {
        set_error("sph_create: only lmax == mmax >= 1 (triangular truncation) is supported");
        return SPH_ERR_ARG;
    }
    if (nlat <= 0 || nphi <= 0) {
        int np = 3 * mmax + 1;
        while (!smooth7(np)) np++;
        int nl = (3 * lmax) / 2 + 1;
        if (nl & 1) nl++;
        nlat = nl;
        nphi = np;
    }
    if ((nlat & 1) || nlat < lmax + 2 || nphi < 2 * mmax + 2) {
        set_error("sph_create: need even nlat >= lmax+2 and nphi >= 2*mmax+2");
        return SPH_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { set_error(std::string("sph_create: no CUDA device: ") + cudaGetErrorString(e)); return SPH_ERR_CUDA; }
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) { set_error(std::string("sph_create: ") + cudaGetErrorString(e)); return SPH_ERR_CUDA; }
    if (prop.major != 10) {
        set_error("sph_create: this library is built for sm_100a (B200); device is sm_" + std::to_string(prop.major) +
                  std::to_string(prop.minor));
        return SPH_ERR_CUDA;
    }
    sph_handle* h = new sph_handle();
    h->L = lmax;
    h->nlat = nlat;
    h->nphi = nphi;
    h->nh = nlat / 2;
    h->nlm = (lmax + 1) * (lmax + 2) / 2;
    h->ncplx = (lmax + 1) * (lmax + 1);
    h->nspat = nlat * nphi;
    h->flags = flags;
    h->device = dev;
    int rc = fft_kernels_init();
    if (rc == SPH_OK) rc = legendre_kernels_init();
    if (rc == SPH_OK) rc = fft_plan_init(&h->fft, nphi);
    if (rc == SPH_OK) rc = setup_tables(h);
    if (rc == SPH_OK && (flags & SPH_PREC_MIXED)) {
        rc = tc_kernels_init();
        if (rc == SPH_OK) rc = tc_tables_build(h, lmax + 1);
    }
    // reserve the fixed scratch of sph_SH_to_spat_noalloc on this device now,
    // so that the no-allocation entry point never triggers the reservation
    void* scratch = nullptr;
    if (rc == SPH_OK) rc = noalloc_scratch(dev, &scratch);
    if (rc != SPH_OK) {
        sph_destroy(h);
        return rc;
    }
    *out = h;
    return SPH_OK;
}

int sph_destroy(sph_handle* h) {
    if (!h) return SPH_OK;
    cudaDeviceSynchronize();
    rk_free(h);
    tc_tables_free(h);
    if (h->mu) cudaFree(h->mu);
    if (h->w) cudaFree(h->w);
    if (h->wc) cudaFree(h->wc);
    if (h->cosphi) cudaFree(h->cosphi);
    if (h->lat) cudaFree(h->lat);
    if (h->plm) cudaFree(h->plm);
    if (h->poff) cudaFree(h->poff);
    if (h->ws) cudaFree(h->ws);
    fft_plan_free(&h->fft);
    delete h;
    return SPH_OK;
}

int sph_info(const sph_handle* h, int* lmax, int* nlat, int* nphi, int* nlm, int* ncplx) {
    if (!h) { set_error("sph_info: NULL handle"); return SPH_ERR_ARG; }
    if (lmax) *lmax = h->L;
    if (nlat) *nlat = h->nlat;
    if (nphi) *nphi = h->nphi;
    if (nlm) *nlm = h->nlm;
    if (ncplx) *ncplx = h->ncplx;
    return SPH_OK;
}

int sph_grid(const sph_handle* h, double* mu, double* cosphi, double* w, double* lat) {
    if (!h) { set_error("sph_grid: NULL handle"); return SPH_ERR_ARG; }
    const size_t b = sizeof(double) * h->nlat;
    if (mu) std::memcpy(mu, h->mu_h.data(), b);
    if (cosphi) std::memcpy(cosphi, h->cosphi_h.data(), b);
    if (w) std::memcpy(w, h->w_h.data(), b);
    if (lat) std::memcpy(lat, h->lat_h.data(), b);
    return SPH_OK;
}

#define CHECK_H(fn)                                                  \
    if (!h) { set_error(std::string(fn) + ": NULL handle"); return SPH_ERR_ARG; }

int sph_sync(sph_handle* h, void* stream) {
    CHECK_H("sph_sync");
    SPH_CUDA_TRY(cudaStreamSynchronize(S(stream)));
    return tc_check(h);
}

int sph_wait_selftest(sph_handle* h, double seconds, void* stream) {
    CHECK_H("sph_wait_selftest");
    return tc_wait_selftest(h, seconds, S(stream));
}

int sph_spat_to_SH(sph_handle* h, const double* spat, double* spec, int batch, long long ld_spat, long long ld_spec,
                   void* stream) {
    CHECK_H("sph_spat_to_SH");
    if (batch < 0 || (batch > 0 && (!spat || !spec))) { set_error("sph_spat_to_SH: bad arguments"); return SPH_ERR_ARG; }
    if (batch == 0) return SPH_OK;
    if (ld_spat <= 0) ld_spat = h->nspat;
    if (ld_spec <= 0) ld_spec = h->nlm;
    const int mF = h->L + 1;
    const long long ldF = (long long)mF * h->nlat;
    if (int rc = ensure_workspace(h, sizeof(double2) * ldF * batch)) return rc;
    double2* F = static_cast<double2*>(h->ws);
    if (int rc = ring_analysis_real(h, spat, ld_spat, F, ldF, mF, batch, S(stream))) return rc;
    return legendre_analysis_real(h, F, ldF, reinterpret_cast<double2*>(spec), ld_spec, h->L, batch, S(stream));
}

int sph_SH_to_spat(sph_handle* h, const double* spec, double* spat, int batch, long long ld_spec, long long ld_spat,
                   void* stream) {
    CHECK_H("sph_SH_to_spat");
    if (batch < 0 || (batch > 0 && (!spat || !spec))) { set_error("sph_SH_to_spat: bad arguments"); return SPH_ERR_ARG; }
    if (batch == 0) return SPH_OK;
    if (ld_spat <= 0) ld_spat = h->nspat;
    if (ld_spec <= 0) ld_spec = h->nlm;
    const int mF = h->L + 1;
    const long long ldF = (long long)mF * h->nlat;
    if (int rc = ensure_workspace(h, sizeof(double2) * ldF * batch)) return rc;
    double2* F = static_cast<double2*>(h->ws);
    if (int rc = legendre_synthesis_real(h, reinterpret_cast<const double2*>(spec), ld_spec, h->L, F, ldF, batch, S(stream)))
        return rc;
    return ring_synthesis_real(h, F, ldF, mF, spat, ld_spat, batch, nullptr, nullptr, 0, 0, S(stream));
}

int sph_cplx_spat_to_SH(sph_handle* h, const double* spat, double* spec, int batch, long long ld_spat,
                        long long ld_spec, void* stream) {
    CHECK_H("sph_cplx_spat_to_SH");
    if (batch < 0 || (batch > 0 && (!spat || !spec))) { set_error("sph_cplx_spat_to_SH: bad arguments"); return SPH_ERR_ARG; }
    if (batch == 0) return SPH_OK;
    if (ld_spat <= 0) ld_spat = h->nspat;
    if (ld_spec <= 0) ld_spec = h->ncplx;
    const long long ldF = (long long)(2 * h->L + 1) * h->nlat;
    if (int rc = ensure_workspace(h, sizeof(double2) * ldF * batch)) return rc;
    double2* F = static_cast<double2*>(h->ws);
    if (int rc = ring_analysis_cplx(h, reinterpret_cast<const double2*>(spat), ld_spat, F, ldF, batch, S(stream))) return rc;
    return legendre_analysis_cplx(h, F, ldF, reinterpret_cast<double2*>(spec), ld_spec, batch, S(stream));
}

int sph_cplx_SH_to_spat(sph_handle* h, const double* spec, double* spat, int batch, long long ld_spec,
                        long long ld_spat, void* stream) {
    CHECK_H("sph_cplx_SH_to_spat");
    if (batch < 0 || (batch > 0 && (!spat || !spec))) { set_error("sph_cplx_SH_to_spat: bad arguments"); return SPH_ERR_ARG; }
    if (batch == 0) return SPH_OK;
    if (ld_spat <= 0) ld_spat = h->nspat;
    if (ld_spec <= 0) ld_spec = h->ncplx;
    const long long ldF = (long long)(2 * h->L + 1) * h->nlat;
    if (int rc = ensure_workspace(h, sizeof(double2) * ldF * batch)) return rc;
    double2* F = static_cast<double2*>(h->ws);
    if (int rc = legendre_synthesis_cplx(h, reinterpret_cast<const double2*>(spec), ld_spec, F, ldF, batch, S(stream)))
        return rc;
    return ring_synthesis_cplx(h, F, ldF, reinterpret_cast<double2*>(spat), ld_spat, batch, S(stream));
}

int sph_legendre_synthesis(sph_handle* h, const double* spec, double* four, int batch, void* stream) {
    CHECK_H("sph_legendre_synthesis");
    if (batch < 0 || (batch > 0 && (!spec || !four))) { set_error("sph_legendre_synthesis: bad arguments"); return SPH_ERR_ARG; }
    const long long ldF = (long long)(h->L + 1) * h->nlat;
    return legendre_synthesis_real(h, reinterpret_cast<const double2*>(spec), h->nlm, h->L,
                                   reinterpret_cast<double2*>(four), ldF, batch, S(stream));
}

int sph_legendre_analysis(sph_handle* h, const double* four, double* spec, int batch, void* stream) {
    CHECK_H("sph_legendre_analysis");
    if (batch < 0 || (batch > 0 && (!spec || !four))) { set_error("sph_legendre_analysis: bad arguments"); return SPH_ERR_ARG; }
    const long long ldF = (long long)(h->L + 1) * h->nlat;
    return legendre_analysis_real(h, reinterpret_cast<const double2*>(four), ldF, reinterpret_cast<double2*>(spec), h->nlm,
                                  h->L, batch, S(stream));
}

int sph_spec_op(sph_handle* h, int op, const double* in, double* out, double a_re, double a_im, double b_re,
                double b_im, int batch, int cplx, void* stream) {
    CHECK_H("sph_spec_op");
    if (!in || !out || batch < 0) { set_error("sph_spec_op: bad arguments"); return SPH_ERR_ARG; }
    if (in == out && (op == SPH_OP_D1MU2 || op == SPH_OP_MU || op == SPH_OP_MU2)) {
        set_error("sph_spec_op: recurrence operators cannot run in place");
        return SPH_ERR_ARG;
    }
    const long long ld = cplx ? h->ncplx : h->nlm;
    return spec_op(h, op, reinterpret_cast<const double2*>(in), ld, reinterpret_cast<double2*>(out), ld,
                   make_double2(a_re, a_im), make_double2(b_re, b_im), batch, cplx ? 1 : 0, S(stream));
}

int sph_spec_copy_modes(const sph_handle* hs, const double* src, const sph_handle* hd, double* dst, int batch,
                        void* stream) {
    if (!hs || !hd || batch < 0 || (batch > 0 && (!src || !dst))) {
        set_error("sph_spec_copy_modes: bad arguments");
        return SPH_ERR_ARG;
    }
    if (hs->device != hd->device) {
        set_error("sph_spec_copy_modes: the two handles are on different devices");
        return SPH_ERR_ARG;
    }
    if (batch > 0) {
        // blocks of the copy kernel read src while others write dst, so the
        // two arrays must not share any byte
        const char* s0 = reinterpret_cast<const char*>(src);
        const char* s1 = s0 + sizeof(double2) * (size_t)hs->nlm * (size_t)batch;
        const char* d0 = reinterpret_cast<const char*>(dst);
        const char* d1 = d0 + sizeof(double2) * (size_t)hd->nlm * (size_t)batch;
        if (s0 < d1 && d0 < s1) {
            set_error("sph_spec_copy_modes: source and destination arrays overlap");
            return SPH_ERR_ARG;
        }
    }
    int dev = 0;
    SPH_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != hs->device) {
        set_error("sph_spec_copy_modes: the current device is not the handles' device");
        return SPH_ERR_ARG;
    }
    return spec_copy_modes(hs, reinterpret_cast<const double2*>(src), hs->nlm, hd, reinterpret_cast<double2*>(dst),
                           hd->nlm, batch, S(stream));
}

}  // extern "C"
