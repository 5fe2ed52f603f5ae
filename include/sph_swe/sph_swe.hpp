// C++ class surface of the spectral shallow-water path on top of the C ABI of
// libsphgpu.so (sph_gpu.h): SPHConfig, SPHData, SPHDataComplex, SPHOperators,
// REXI and the RK4 / REXI time steppers, with the names, argument meanings and
// lazy dual (spectral / physical) representation of the reference classes
// (sph/SPHConfig.hpp, sph/SPHData.hpp, sph/SPHDataComplex.hpp,
// sph/SPHOperators.hpp, rexi/REXI.hpp, AppSWE.hpp).
//
// Data live on the device: data_spec (packed complex, nlm or (L+1)^2
// elements) and data_spat (theta-contiguous grid, nphi * nlat doubles,
// index lon * nlat + lat).  Each object owns its two buffers (from a per-size
// cache, so that the value-semantics temporaries of the operators do not
// call cudaMalloc each time); a request_data_* call transforms on demand,
// exactly like the reference's validity flags.  All device work is ordered
// on SPHConfig::stream.  Functions that take host lambdas (the *_update_lambda
// family) evaluate them on the host and upload the result, as the reference
// evaluates them on its CPU grid.  Errors throw std::runtime_error with the
// library's message (the reference asserts and exits).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../sph_gpu.h"

namespace sph_swe {

using cplx = std::complex<double>;

inline void check(int rc, const char* what) {
    if (rc != SPH_OK) {
        char buf[1024];
        sph_last_error(buf, (int)sizeof(buf));
        throw std::runtime_error(std::string(what) + ": " + buf);
    }
}
inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Device buffers by size, reused across SPHData temporaries (the role of the
// reference's MemBlockAlloc).
class DeviceCache {
  public:
    static void* get(size_t bytes) {
        std::lock_guard<std::mutex> lk(mu());
        auto& v = pool()[bytes];
        if (!v.empty()) {
            void* p = v.back();
            v.pop_back();
            return p;
        }
        void* p = nullptr;
        cuda_check(cudaMalloc(&p, bytes), "cudaMalloc");
        return p;
    }
    static void put(void* p, size_t bytes) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu());
        pool()[bytes].push_back(p);
    }

  private:
    static std::mutex& mu() {
        static std::mutex m;
        return m;
    }
    static std::map<size_t, std::vector<void*>>& pool() {
        static std::map<size_t, std::vector<void*>> p;
        return p;
    }
};

// ------------------------------------------------------------------ SPHConfig
// Replaces SPHConfig (SPHConfig.hpp): the shtns_cfg becomes an sph_handle.
class SPHConfig {
  public:
    int spat_num_lon = -1;
    int spat_num_lat = -1;
    int spat_num_elems = -1;
    int spec_n_max = -1;
    int spec_m_max = -1;
    int spec_num_elems = -1;
    int cplx_spec_num_elems = -1;
    // host arrays of nlat entries: latitude phi, mu = sin(phi) (Gauss nodes), cos(phi)
    double* lat = nullptr;
    double* lat_gaussian = nullptr;
    double* lat_cogaussian = nullptr;
    cudaStream_t stream = nullptr;

    SPHConfig() = default;
    SPHConfig(const SPHConfig&) = delete;
    SPHConfig& operator=(const SPHConfig&) = delete;
    ~SPHConfig() { shutdown(); }

    // SPHConfig::setup (SPHConfig.hpp:324-352): explicit grid
    void setup(int mmax, int nmax, int nphi, int nlat, int precision = SPH_PREC_FP64) {
        create(mmax, nmax, nlat, nphi, precision);
    }

    // SPHConfig::setupAutoPhysicalSpace (SPHConfig.hpp:366-399): quadratic-rule grid
    void setupAutoPhysicalSpace(int mmax, int nmax, int* o_nphi, int* o_nlat, int precision = SPH_PREC_FP64) {
        create(mmax, nmax, 0, 0, precision);
        if (o_nphi) *o_nphi = spat_num_lon;
        if (o_nlat) *o_nlat = spat_num_lat;
    }

    // SPHConfig::setupAdditionalModes (SPHConfig.hpp:403-417): the
    // quadratic-rule grid of base's truncation plus the added modes (the
    // REXI extended-modes option); one truncation for n and m, as sph_create
    void setupAdditionalModes(const SPHConfig* base, int added_lon, int added_lat, int precision = SPH_PREC_FP64) {
        if (added_lon != added_lat)
            throw std::runtime_error("setupAdditionalModes: the same number of modes in longitude and latitude");
        create(base->spec_m_max + added_lon, base->spec_n_max + added_lat, 0, 0, precision);
    }

    void shutdown() {
        free_grids();
        if (h_) sph_destroy(h_);
        h_ = nullptr;
    }

    // packed real layout (SPHConfig.hpp:106-116)
    std::size_t getArrayIndexByModes(int n, int m) const { return ((m * (2 * spec_n_max - m + 1)) >> 1) + n; }
    // complex layout (SPHConfig.hpp:120-130)
    std::size_t getArrayIndexByModes_Complex(int n, int m) const { return (std::size_t)(n * n + n + m); }

    sph_handle* handle() const {
        if (!h_) throw std::runtime_error("SPHConfig: not set up");
        return h_;
    }
    void* s() const { return reinterpret_cast<void*>(stream); }

    // device grids of cos(phi)^-1 and cos(phi)^-2 for the grid-valued operators (built on first use)
    const double* inv_cos() const {
        grids();
        return inv_cos_;
    }
    const double* inv_cos2() const {
        grids();
        return inv_cos2_;
    }
    const double* cos_grid() const {
        grids();
        return cos_;
    }
    // the same weights with every value twice, for complex grids (re, im)
    const double* inv_cos_c() const {
        grids();
        return inv_cos_c_;
    }
    const double* inv_cos2_c() const {
        grids();
        return inv_cos2_c_;
    }
    const double* cos_grid_c() const {
        grids();
        return cos_c_;
    }

  private:
    sph_handle* h_ = nullptr;
    std::vector<double> lat_v_, mu_v_, cos_v_;
    mutable double* inv_cos_ = nullptr;
    mutable double* inv_cos2_ = nullptr;
    mutable double* cos_ = nullptr;
    mutable double* inv_cos_c_ = nullptr;
    mutable double* inv_cos2_c_ = nullptr;
    mutable double* cos_c_ = nullptr;

    void create(int mmax, int nmax, int nlat, int nphi, int precision) {
        shutdown();
        check(sph_create(nmax, mmax, nlat, nphi, precision, &h_), "sph_create");
        int L, nl, np, nlm, nc;
        check(sph_info(h_, &L, &nl, &np, &nlm, &nc), "sph_info");
        spec_n_max = spec_m_max = L;
        spat_num_lat = nl;
        spat_num_lon = np;
        spat_num_elems = nl * np;
        spec_num_elems = nlm;
        cplx_spec_num_elems = nc;
        lat_v_.resize(nl);
        mu_v_.resize(nl);
        cos_v_.resize(nl);
        check(sph_grid(h_, mu_v_.data(), cos_v_.data(), nullptr, lat_v_.data()), "sph_grid");
        lat = lat_v_.data();
        lat_gaussian = mu_v_.data();
        lat_cogaussian = cos_v_.data();
    }
    void grids() const {
        if (inv_cos_) return;
        const size_t n = (size_t)spat_num_elems;
        std::vector<double> a(n), b(n), c(n);
        for (int i = 0; i < spat_num_lon; i++)
            for (int j = 0; j < spat_num_lat; j++) {
                const double cj = cos_v_[j];
                a[(size_t)i * spat_num_lat + j] = 1.0 / cj;
                b[(size_t)i * spat_num_lat + j] = 1.0 / (cj * cj);
                c[(size_t)i * spat_num_lat + j] = cj;
            }
        cuda_check(cudaMalloc(&inv_cos_, n * 8), "cudaMalloc");
        cuda_check(cudaMalloc(&inv_cos2_, n * 8), "cudaMalloc");
        cuda_check(cudaMalloc(&cos_, n * 8), "cudaMalloc");
        cuda_check(cudaMemcpy(inv_cos_, a.data(), n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
        cuda_check(cudaMemcpy(inv_cos2_, b.data(), n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
        cuda_check(cudaMemcpy(cos_, c.data(), n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
        std::vector<double> a2(2 * n), b2(2 * n), c2(2 * n);
        for (size_t k = 0; k < n; k++) {
            a2[2 * k] = a2[2 * k + 1] = a[k];
            b2[2 * k] = b2[2 * k + 1] = b[k];
            c2[2 * k] = c2[2 * k + 1] = c[k];
        }
        cuda_check(cudaMalloc(&inv_cos_c_, 2 * n * 8), "cudaMalloc");
        cuda_check(cudaMalloc(&inv_cos2_c_, 2 * n * 8), "cudaMalloc");
        cuda_check(cudaMalloc(&cos_c_, 2 * n * 8), "cudaMalloc");
        cuda_check(cudaMemcpy(inv_cos_c_, a2.data(), 2 * n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
        cuda_check(cudaMemcpy(inv_cos2_c_, b2.data(), 2 * n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
        cuda_check(cudaMemcpy(cos_c_, c2.data(), 2 * n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    void free_grids() {
        for (double** p : {&inv_cos_, &inv_cos2_, &cos_, &inv_cos_c_, &inv_cos2_c_, &cos_c_})
            if (*p) {
                cudaFree(*p);
                *p = nullptr;
            }
    }
};

// ------------------------------------------------------------------ SPHData
// Replaces SPHData (SPHData.hpp): real field with lazy spectral / physical representation.
class SPHData {
  public:
    SPHConfig* sphConfig = nullptr;
    cplx* data_spec = nullptr;   // device, spec_num_elems
    double* data_spat = nullptr; // device, spat_num_elems
    mutable bool data_spec_valid = false;
    mutable bool data_spat_valid = false;

    explicit SPHData(SPHConfig* cfg = nullptr) {
        if (cfg) setup(cfg);
    }
    SPHData(const SPHData& o) { *this = o; }
    SPHData(SPHData&& o) noexcept { swap(o); }
    ~SPHData() { release(); }

    // copies only the valid representations (SPHData.hpp:57-103)
    SPHData& operator=(const SPHData& o) {
        if (this == &o) return *this;
        if (sphConfig != o.sphConfig) setup(o.sphConfig);
        if (o.data_spec_valid)
            cuda_check(cudaMemcpyAsync(data_spec, o.data_spec, spec_bytes(), cudaMemcpyDeviceToDevice, sphConfig->stream),
                       "copy");
        if (o.data_spat_valid)
            cuda_check(cudaMemcpyAsync(data_spat, o.data_spat, spat_bytes(), cudaMemcpyDeviceToDevice, sphConfig->stream),
                       "copy");
        data_spec_valid = o.data_spec_valid;
        data_spat_valid = o.data_spat_valid;
        return *this;
    }
    SPHData& operator=(SPHData&& o) noexcept {
        swap(o);
        return *this;
    }

    void setup(SPHConfig* cfg) {
        release();
        sphConfig = cfg;
        data_spec = static_cast<cplx*>(DeviceCache::get(spec_bytes()));
        data_spat = static_cast<double*>(DeviceCache::get(spat_bytes()));
        data_spec_valid = data_spat_valid = false;
    }

    // SPHData.hpp:190-207
    void request_data_spectral() const {
        if (data_spec_valid) return;
        if (!data_spat_valid) throw std::runtime_error("SPHData: no valid representation");
        check(sph_spat_to_SH(h(), data_spat, reinterpret_cast<double*>(data_spec), 1, 0, 0, sphConfig->s()),
              "sph_spat_to_SH");
        data_spec_valid = true;
    }
    // SPHData.hpp:210-227
    void request_data_physical() const {
        if (data_spat_valid) return;
        if (!data_spec_valid) throw std::runtime_error("SPHData: no valid representation");
        check(sph_SH_to_spat(h(), reinterpret_cast<const double*>(data_spec), data_spat, 1, 0, 0, sphConfig->s()),
              "sph_SH_to_spat");
        data_spat_valid = true;
    }

    // spectral arithmetic (SPHData.hpp:231-330, 410-443)
    SPHData operator+(const SPHData& b) const { return spec_axpby(1.0, *this, 1.0, b); }
    SPHData operator-(const SPHData& b) const { return spec_axpby(1.0, *this, -1.0, b); }
    SPHData operator-() const { return spec_axpby(-1.0, *this, 0.0, *this); }
    SPHData operator*(double v) const { return spec_axpby(v, *this, 0.0, *this); }
    SPHData operator/(double v) const { return spec_axpby(1.0 / v, *this, 0.0, *this); }
    SPHData& operator+=(const SPHData& b) { return *this = *this + b; }
    SPHData& operator-=(const SPHData& b) { return *this = *this - b; }
    SPHData& operator*=(double v) { return *this = *this * v; }
    // adds v to the field: sqrt(4 pi) v on the (0,0) coefficient (SPHData.hpp:429-443)
    SPHData operator+(double v) const {
        request_data_spectral();
        SPHData out(sphConfig);
        copy_spec_to(out);
        check(sph_spat_op(h(), SPH_SPAT_ADD_CONST, reinterpret_cast<const double*>(out.data_spec), nullptr,
                          reinterpret_cast<double*>(out.data_spec), v * std::sqrt(4.0 * M_PI), 0.0, 1, sphConfig->s()),
              "sph_spat_op");
        out.data_spec_valid = true;
        return out;
    }
    SPHData operator-(double v) const { return *this + (-v); }

    // product of two fields on the grid (SPHData.hpp:334-353)
    SPHData operator*(const SPHData& b) const {
        request_data_physical();
        b.request_data_physical();
        SPHData out(sphConfig);
        check(sph_spat_op(h(), SPH_SPAT_MUL, data_spat, b.data_spat, out.data_spat, 1.0, 0.0, sphConfig->spat_num_elems,
                          sphConfig->s()),
              "sph_spat_op");
        out.data_spat_valid = true;
        return out;
    }
    SPHData& operator*=(const SPHData& b) { return *this = *this * b; }

    // x / (a - b l(l+1) / r^2)  (SPHData.hpp:475-497)
    SPHData spec_solve_helmholtz(double a, double b, double r) const {
        request_data_spectral();
        SPHData out(sphConfig);
        check(sph_spec_op(h(), SPH_OP_HELMHOLTZ, reinterpret_cast<const double*>(data_spec),
                          reinterpret_cast<double*>(out.data_spec), a, 0.0, b / (r * r), 0.0, 1, 0, sphConfig->s()),
              "sph_spec_op");
        out.data_spec_valid = true;
        return out;
    }

    // SPHData::spec_copyToDifferentModes (SPHData.hpp:108-187): this field's
    // spectrum in o's truncation (shared modes copied, the others zero)
    const SPHData& spec_copyToDifferentModes(SPHData& o) const {
        if (o.sphConfig == sphConfig) throw std::runtime_error("spec_copyToDifferentModes: same configuration");
        request_data_spectral();
        if (sphConfig->stream != o.sphConfig->stream) cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        check(sph_spec_copy_modes(h(), reinterpret_cast<const double*>(data_spec), o.h(),
                                  reinterpret_cast<double*>(o.data_spec), 1, o.sphConfig->s()),
              "sph_spec_copy_modes");
        o.data_spec_valid = true;
        o.data_spat_valid = false;
        return *this;
    }

    void spec_set_zero() {
        cuda_check(cudaMemsetAsync(data_spec, 0, spec_bytes(), sphConfig->stream), "memset");
        data_spec_valid = true;
        data_spat_valid = false;
    }
    void spat_set_zero() { spat_set_value(0.0); }
    void spat_set_value(double v) {
        check(sph_spat_op(h(), SPH_SPAT_FILL, nullptr, nullptr, data_spat, v, 0.0, sphConfig->spat_num_elems,
                          sphConfig->s()),
              "sph_spat_op");
        data_spat_valid = true;
        data_spec_valid = false;
    }

    // host lambdas on the grid (SPHData.hpp:645-766): (lon, phi), (lon, mu), (lon, cos phi)
    void spat_update_lambda(const std::function<void(double, double, double&)>& f) {
        grid_lambda(f, sphConfig->lat);
    }
    void spat_update_lambda_gaussian_grid(const std::function<void(double, double, double&)>& f) {
        grid_lambda(f, sphConfig->lat_gaussian);
    }
    void spat_update_lambda_cogaussian_grid(const std::function<void(double, double, double&)>& f) {
        grid_lambda(f, sphConfig->lat_cogaussian);
    }
    // host lambda on the coefficients (SPHData.hpp:536-558)
    void spec_update_lambda(const std::function<void(int, int, cplx&)>& f) {
        std::vector<cplx> host((size_t)sphConfig->spec_num_elems);
        for (int m = 0; m <= sphConfig->spec_m_max; m++)
            for (int n = m; n <= sphConfig->spec_n_max; n++) f(n, m, host[sphConfig->getArrayIndexByModes(n, m)]);
        cuda_check(cudaMemcpyAsync(data_spec, host.data(), spec_bytes(), cudaMemcpyHostToDevice, sphConfig->stream),
                   "upload");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        data_spec_valid = true;
        data_spat_valid = false;
    }

    // host grid (nphi x nlat, theta-contiguous) -> this field's grid
    void spat_from_host(const std::vector<double>& v) {
        if (v.size() != (size_t)sphConfig->spat_num_elems) throw std::runtime_error("spat_from_host: wrong size");
        cuda_check(cudaMemcpyAsync(data_spat, v.data(), spat_bytes(), cudaMemcpyHostToDevice, sphConfig->stream), "ul");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        data_spat_valid = true;
        data_spec_valid = false;
    }
    // host spectrum (packed layout) -> this field's spectrum
    void spec_from_host(const std::vector<cplx>& v) {
        if (v.size() != (size_t)sphConfig->spec_num_elems) throw std::runtime_error("spec_from_host: wrong size");
        cuda_check(cudaMemcpyAsync(data_spec, v.data(), spec_bytes(), cudaMemcpyHostToDevice, sphConfig->stream), "ul");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        data_spec_valid = true;
        data_spat_valid = false;
    }
    // the spectral array was written directly (by a C-ABI call on data_spec)
    void mark_spectral() {
        data_spec_valid = true;
        data_spat_valid = false;
    }

    std::vector<cplx> spec_to_host() const {
        request_data_spectral();
        std::vector<cplx> v((size_t)sphConfig->spec_num_elems);
        cuda_check(cudaMemcpyAsync(v.data(), data_spec, spec_bytes(), cudaMemcpyDeviceToHost, sphConfig->stream), "dl");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        return v;
    }
    std::vector<double> spat_to_host() const {
        request_data_physical();
        std::vector<double> v((size_t)sphConfig->spat_num_elems);
        cuda_check(cudaMemcpyAsync(v.data(), data_spat, spat_bytes(), cudaMemcpyDeviceToHost, sphConfig->stream), "dl");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        return v;
    }

    // grid as a tab-separated table in the reference's CSV layout (SPHData.hpp:935-1037):
    // "#TI title", "#TX Longitude", "#TY Latitude", then "0" and the longitudes in
    // degrees, then one row per latitude ring j = nlat-1 .. 0 (south to north)
    // with the latitude in degrees first; `shifted` moves longitude 0 to the
    // middle (spat_write_file_lon_pi_shifted)
    void spat_write_file(const char* filename, const char* title = "", int precision = 8, bool shifted = false) const {
        const auto v = spat_to_host();
        const int nlon = sphConfig->spat_num_lon, nlat = sphConfig->spat_num_lat;
        std::ofstream f(filename, std::ios_base::trunc);
        if (!f) throw std::runtime_error(std::string("cannot write ") + filename);
        f << std::setprecision(precision);
        f << "#TI " << title << "\n#TX Longitude\n#TY Latitude\n0\t";
        for (int i = 0; i < nlon; i++) {
            const double lon = (double)i / nlon * 2.0 * M_PI;
            f << ((shifted ? lon - M_PI : lon) / M_PI * 180.0);
            if (i < nlon - 1) f << "\t";
        }
        f << "\n";
        for (int j = nlat - 1; j >= 0; j--) {
            f << sphConfig->lat[j] / M_PI * 180.0 << "\t";
            for (int i = 0; i < nlon; i++) {
                int ia = shifted ? i + nlon / 2 : i;
                if (ia >= nlon) ia -= nlon;
                f << v[(size_t)ia * nlat + j];
                if (i < nlon - 1) f << "\t";
            }
            f << "\n";
        }
    }
    void spat_write_file_lon_pi_shifted(const char* filename, const char* title = "", int precision = 8) const {
        spat_write_file(filename, title, precision, true);
    }

    // reductions on the grid (SPHData.hpp:800-876) and the NaN check (SPHData.hpp:560-569,
    // here on a requested grid)
    double spat_reduce_abs_max() const {
        double r = 0;
        for (double x : spat_to_host()) r = std::max(r, std::fabs(x));
        return r;
    }
    double spat_reduce_max() const {
        const auto v = spat_to_host();
        double r = v[0];
        for (double x : v) r = std::max(r, x);
        return r;
    }
    double spat_reduce_min() const {
        const auto v = spat_to_host();
        double r = v[0];
        for (double x : v) r = std::min(r, x);
        return r;
    }
    double spat_reduce_error_max(const SPHData& o) const {
        const auto a = spat_to_host(), b = o.spat_to_host();
        double r = 0;
        for (size_t i = 0; i < a.size(); i++) r = std::max(r, std::fabs(a[i] - b[i]));
        return r;
    }
    bool isAnyNaNorInf() const {
        for (double x : spat_to_host())
            if (!std::isfinite(x)) return true;
        return false;
    }

    sph_handle* h() const { return sphConfig->handle(); }
    size_t spec_bytes() const { return sizeof(cplx) * (size_t)sphConfig->spec_num_elems; }
    size_t spat_bytes() const { return sizeof(double) * (size_t)sphConfig->spat_num_elems; }

    // out = a x + b y in spectral space
    static SPHData spec_axpby(double a, const SPHData& x, double b, const SPHData& y) {
        x.request_data_spectral();
        y.request_data_spectral();
        SPHData out(x.sphConfig);
        check(sph_spat_op(x.h(), SPH_SPAT_AXPBY, reinterpret_cast<const double*>(x.data_spec),
                          reinterpret_cast<const double*>(y.data_spec), reinterpret_cast<double*>(out.data_spec), a, b,
                          2LL * x.sphConfig->spec_num_elems, x.sphConfig->s()),
              "sph_spat_op");
        out.data_spec_valid = true;
        return out;
    }

  private:
    void release() {
        if (sphConfig) {
            DeviceCache::put(data_spec, spec_bytes());
            DeviceCache::put(data_spat, spat_bytes());
        }
        data_spec = nullptr;
        data_spat = nullptr;
        data_spec_valid = data_spat_valid = false;
    }
    void swap(SPHData& o) noexcept {
        std::swap(sphConfig, o.sphConfig);
        std::swap(data_spec, o.data_spec);
        std::swap(data_spat, o.data_spat);
        std::swap(data_spec_valid, o.data_spec_valid);
        std::swap(data_spat_valid, o.data_spat_valid);
    }
    void copy_spec_to(SPHData& out) const {
        cuda_check(cudaMemcpyAsync(out.data_spec, data_spec, spec_bytes(), cudaMemcpyDeviceToDevice, sphConfig->stream),
                   "copy");
    }
    void grid_lambda(const std::function<void(double, double, double&)>& f, const double* latv) {
        const int nlon = sphConfig->spat_num_lon, nlat = sphConfig->spat_num_lat;
        std::vector<double> host((size_t)nlon * nlat);
        for (int i = 0; i < nlon; i++) {
            const double lon = 2.0 * M_PI * i / nlon;
            for (int j = 0; j < nlat; j++) f(lon, latv[j], host[(size_t)i * nlat + j]);
        }
        cuda_check(cudaMemcpyAsync(data_spat, host.data(), spat_bytes(), cudaMemcpyHostToDevice, sphConfig->stream),
                   "upload");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        data_spat_valid = true;
        data_spec_valid = false;
    }
};

inline SPHData operator*(double v, const SPHData& x) { return x * v; }
inline SPHData operator+(double v, const SPHData& x) { return x + v; }
inline SPHData operator-(double v, const SPHData& x) { return (-x) + v; }

// ------------------------------------------------------------------ SPHDataComplex
// Replaces SPHDataComplex (SPHDataComplex.hpp): complex field, layout n*n+n+m.
class SPHDataComplex {
  public:
    SPHConfig* sphConfig = nullptr;
    cplx* data_spec = nullptr;  // device, (L+1)^2
    cplx* data_spat = nullptr;  // device, nphi * nlat complex
    mutable bool data_spec_valid = false;
    mutable bool data_spat_valid = false;

    explicit SPHDataComplex(SPHConfig* cfg = nullptr) {
        if (cfg) setup(cfg);
    }
    SPHDataComplex(const SPHDataComplex& o) { *this = o; }
    ~SPHDataComplex() { release(); }
    SPHDataComplex& operator=(const SPHDataComplex& o) {
        if (this == &o) return *this;
        if (sphConfig != o.sphConfig) setup(o.sphConfig);
        if (o.data_spec_valid)
            cuda_check(cudaMemcpyAsync(data_spec, o.data_spec, spec_bytes(), cudaMemcpyDeviceToDevice, sphConfig->stream),
                       "copy");
        if (o.data_spat_valid)
            cuda_check(cudaMemcpyAsync(data_spat, o.data_spat, spat_bytes(), cudaMemcpyDeviceToDevice, sphConfig->stream),
                       "copy");
        data_spec_valid = o.data_spec_valid;
        data_spat_valid = o.data_spat_valid;
        return *this;
    }
    // complex field from a real one through the grid (SPHDataComplex.hpp:67-77)
    explicit SPHDataComplex(const SPHData& r) : SPHDataComplex(r.sphConfig) { spat_fromSPHData(r); }
    // SPHDataComplex.hpp:93-104: assignment from a real field goes through the grid
    SPHDataComplex& operator=(const SPHData& r) {
        if (sphConfig != r.sphConfig) setup(r.sphConfig);
        spat_fromSPHData(r);
        return *this;
    }
    // grid of the real field as the real part, imaginary part zero; only the
    // grid is valid afterwards (SPHDataComplex.hpp:162-175)
    void spat_fromSPHData(const SPHData& r) {
        if (r.sphConfig != sphConfig) throw std::runtime_error("spat_fromSPHData: fields of different configurations");
        r.request_data_physical();
        check(sph_spat_op(h(), SPH_SPAT_FILL, nullptr, nullptr, reinterpret_cast<double*>(data_spat), 0.0, 0.0,
                          2LL * sphConfig->spat_num_elems, sphConfig->s()),
              "sph_spat_op");
        cuda_check(cudaMemcpy2DAsync(data_spat, sizeof(cplx), r.data_spat, sizeof(double), sizeof(double),
                                     (size_t)sphConfig->spat_num_elems, cudaMemcpyDeviceToDevice, sphConfig->stream),
                   "copy");
        data_spec_valid = false;
        data_spat_valid = true;
    }
    // real part of this field's grid into o's grid; o becomes grid-valid only
    // (SPHDataComplex.hpp:129-142)
    void spat_RealToSPHData(SPHData& o) const { part_to(o, 0); }
    // imaginary part likewise (SPHDataComplex.hpp:145-158)
    void spat_ImagToSPHData(SPHData& o) const { part_to(o, 1); }

    void setup(SPHConfig* cfg) {
        release();
        sphConfig = cfg;
        data_spec = static_cast<cplx*>(DeviceCache::get(spec_bytes()));
        data_spat = static_cast<cplx*>(DeviceCache::get(spat_bytes()));
    }
    void request_data_spectral() const {
        if (data_spec_valid) return;
        if (!data_spat_valid) throw std::runtime_error("SPHDataComplex: no valid representation");
        check(sph_cplx_spat_to_SH(h(), reinterpret_cast<const double*>(data_spat), reinterpret_cast<double*>(data_spec),
                                  1, 0, 0, sphConfig->s()),
              "sph_cplx_spat_to_SH");
        data_spec_valid = true;
    }
    void request_data_physical() const {
        if (data_spat_valid) return;
        if (!data_spec_valid) throw std::runtime_error("SPHDataComplex: no valid representation");
        check(sph_cplx_SH_to_spat(h(), reinterpret_cast<const double*>(data_spec), reinterpret_cast<double*>(data_spat),
                                  1, 0, 0, sphConfig->s()),
              "sph_cplx_SH_to_spat");
        data_spat_valid = true;
    }
    // product on the full grid (SPHDataComplex.hpp:321-340; the reference stops its loop at (L+1)^2)
    SPHDataComplex operator*(const SPHDataComplex& b) const {
        request_data_physical();
        b.request_data_physical();
        SPHDataComplex out(sphConfig);
        check(sph_spat_op(h(), SPH_SPAT_CMUL, reinterpret_cast<const double*>(data_spat),
                          reinterpret_cast<const double*>(b.data_spat), reinterpret_cast<double*>(out.data_spat), 1.0,
                          0.0, sphConfig->spat_num_elems, sphConfig->s()),
              "sph_spat_op");
        out.data_spat_valid = true;
        return out;
    }
    SPHDataComplex operator+(const SPHDataComplex& b) const { return axpby(1.0, *this, 1.0, b); }
    SPHDataComplex operator-(const SPHDataComplex& b) const { return axpby(1.0, *this, -1.0, b); }
    SPHDataComplex operator*(double v) const { return axpby(v, *this, 0.0, *this); }

    // host spectrum (layout n*n+n+m) -> this field's spectrum
    void spec_from_host(const std::vector<cplx>& v) {
        if (v.size() != (size_t)sphConfig->cplx_spec_num_elems) throw std::runtime_error("spec_from_host: wrong size");
        cuda_check(cudaMemcpyAsync(data_spec, v.data(), spec_bytes(), cudaMemcpyHostToDevice, sphConfig->stream), "ul");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        data_spec_valid = true;
        data_spat_valid = false;
    }
    std::vector<cplx> spat_to_host() const {
        request_data_physical();
        std::vector<cplx> v((size_t)sphConfig->spat_num_elems);
        cuda_check(cudaMemcpyAsync(v.data(), data_spat, spat_bytes(), cudaMemcpyDeviceToHost, sphConfig->stream), "dl");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        return v;
    }
    // x / (a - (b / r^2) n(n+1)) (SPHDataComplex.hpp:523-545)
    SPHDataComplex spec_solve_helmholtz(cplx a, cplx b, double r) const {
        request_data_spectral();
        SPHDataComplex out(sphConfig);
        const cplx br = b / (r * r);
        check(sph_spec_op(h(), SPH_OP_HELMHOLTZ, reinterpret_cast<const double*>(data_spec),
                          reinterpret_cast<double*>(out.data_spec), a.real(), a.imag(), br.real(), br.imag(), 1, 1,
                          sphConfig->s()),
              "sph_spec_op");
        out.data_spec_valid = true;
        return out;
    }

    std::vector<cplx> spec_to_host() const {
        request_data_spectral();
        std::vector<cplx> v((size_t)sphConfig->cplx_spec_num_elems);
        cuda_check(cudaMemcpyAsync(v.data(), data_spec, spec_bytes(), cudaMemcpyDeviceToHost, sphConfig->stream), "dl");
        cuda_check(cudaStreamSynchronize(sphConfig->stream), "sync");
        return v;
    }

    sph_handle* h() const { return sphConfig->handle(); }
    size_t spec_bytes() const { return sizeof(cplx) * (size_t)sphConfig->cplx_spec_num_elems; }
    size_t spat_bytes() const { return sizeof(cplx) * (size_t)sphConfig->spat_num_elems; }

    static SPHDataComplex axpby(double a, const SPHDataComplex& x, double b, const SPHDataComplex& y) {
        x.request_data_spectral();
        y.request_data_spectral();
        SPHDataComplex out(x.sphConfig);
        check(sph_spat_op(x.h(), SPH_SPAT_AXPBY, reinterpret_cast<const double*>(x.data_spec),
                          reinterpret_cast<const double*>(y.data_spec), reinterpret_cast<double*>(out.data_spec), a, b,
                          2LL * x.sphConfig->cplx_spec_num_elems, x.sphConfig->s()),
              "sph_spat_op");
        out.data_spec_valid = true;
        return out;
    }

  private:
    void part_to(SPHData& o, int part) const {
        if (o.sphConfig != sphConfig) throw std::runtime_error("SPHDataComplex: fields of different configurations");
        request_data_physical();
        cuda_check(cudaMemcpy2DAsync(o.data_spat, sizeof(double), reinterpret_cast<const double*>(data_spat) + part,
                                     sizeof(cplx), sizeof(double), (size_t)sphConfig->spat_num_elems,
                                     cudaMemcpyDeviceToDevice, sphConfig->stream),
                   "copy");
        o.data_spec_valid = false;
        o.data_spat_valid = true;
    }
    void release() {
        if (sphConfig) {
            DeviceCache::put(data_spec, spec_bytes());
            DeviceCache::put(data_spat, spat_bytes());
        }
        data_spec = nullptr;
        data_spat = nullptr;
        data_spec_valid = data_spat_valid = false;
    }
};

// ------------------------------------------------------------------ SPHOperators
// Replaces SPHOperators (SPHOperators.hpp).  Spectral operators return spectral
// fields; the grid-valued ones (grad_*, div_*, vort, div) return physical fields
// with the reference's projection points: a spectral operator, one synthesis,
// then the division by cos(phi) or cos(phi)^2 on the grid.
class SPHOperators {
  public:
    // x i m (SPHOperators.hpp:30-54)
    static SPHData diff_lon(const SPHData& x) { return spec(SPH_OP_DIFF_LON, x); }
    // truncated (1 - mu^2) d/dmu (SPHOperators.hpp:234-260)
    static SPHData spec_one_minus_mu_squared_diff_lat_mu(const SPHData& x) { return spec(SPH_OP_D1MU2, x); }
    // mu x, mu^2 x (SPHOperators.hpp:268-333)
    static SPHData mu(const SPHData& x) { return spec(SPH_OP_MU, x); }
    static SPHData mu2(const SPHData& x) { return spec(SPH_OP_MU2, x); }
    // -l(l+1) x (SPHOperators.hpp:482-498)
    static SPHData laplace(const SPHData& x) { return spec(SPH_OP_LAPLACE, x); }

    // I(i m x) / cos(phi) (SPHOperators.hpp:100-119); div_lon is the same operator (:397-402)
    static SPHData grad_lon(const SPHData& x) { return grid_div(diff_lon(x), x.sphConfig->inv_cos()); }
    static SPHData div_lon(const SPHData& x) { return grad_lon(x); }
    // I(D x) / cos(phi) (SPHOperators.hpp:339-388)
    static SPHData grad_lat(const SPHData& x) {
        return grid_div(spec_one_minus_mu_squared_diff_lat_mu(x), x.sphConfig->inv_cos());
    }
    // I(D F(cos(phi) x)) / cos(phi)^2 (SPHOperators.hpp:411-439)
    static SPHData div_lat(const SPHData& x) {
        x.request_data_physical();
        SPHData cx(x.sphConfig);
        check(sph_spat_op(x.h(), SPH_SPAT_MUL, x.data_spat, x.sphConfig->cos_grid(), cx.data_spat, 1.0, 0.0,
                          x.sphConfig->spat_num_elems, x.sphConfig->s()),
              "sph_spat_op");
        cx.data_spat_valid = true;
        return grid_div(spec_one_minus_mu_squared_diff_lat_mu(cx), x.sphConfig->inv_cos2());
    }
    // d/dmu: I(D x) / (1 - mu^2) (SPHOperators.hpp:63-78); d/dphi is grad_lat (:86-91)
    static SPHData diff_lat_mu(const SPHData& x) {
        return grid_div(spec_one_minus_mu_squared_diff_lat_mu(x), x.sphConfig->inv_cos2());
    }
    static SPHData diff_lat_phi(const SPHData& x) { return grad_lat(x); }
    // the truncated (1 - mu^2) d/dmu under its other two names (SPHOperators.hpp:224-230)
    static SPHData spec_cosphi_squared_diff_lat_mu(const SPHData& x) { return spec_one_minus_mu_squared_diff_lat_mu(x); }
    static SPHData spec_one_minus_sinphi_squared_diff_lat_mu(const SPHData& x) {
        return spec_one_minus_mu_squared_diff_lat_mu(x);
    }
    // Robert-variable operators, U = u cos(phi) (SPHOperators.hpp:129-210):
    // I(i m U) / cos^2, I(D V) / cos^2, i m Phi and D Phi (spectral)
    static SPHData robert_div_lon(const SPHData& x) { return grid_div(diff_lon(x), x.sphConfig->inv_cos2()); }
    static SPHData robert_div_lat(const SPHData& x) {
        return grid_div(spec_cosphi_squared_diff_lat_mu(x), x.sphConfig->inv_cos2());
    }
    static SPHData robert_grad_lon(const SPHData& x) { return diff_lon(x); }
    static SPHData robert_grad_lat(const SPHData& x) { return spec_one_minus_mu_squared_diff_lat_mu(x); }

    // vorticity grad_lon(v) - grad_lat(u) and divergence div_lon(u) + div_lat(v)
    // (SPHOperators.hpp:507-529); the sums are spectral, as SPHData's operators are
    static SPHData vort(const SPHData& u, const SPHData& v) { return grad_lon(v) - grad_lat(u); }
    static SPHData div(const SPHData& u, const SPHData& v) { return div_lon(u) + div_lat(v); }

  private:
    static SPHData spec(int op, const SPHData& x) {
        x.request_data_spectral();
        SPHData out(x.sphConfig);
        check(sph_spec_op(x.h(), op, reinterpret_cast<const double*>(x.data_spec), reinterpret_cast<double*>(out.data_spec),
                          0.0, 0.0, 0.0, 0.0, 1, 0, x.sphConfig->s()),
              "sph_spec_op");
        out.data_spec_valid = true;
        return out;
    }
    static SPHData grid_div(const SPHData& y, const double* w) {
        y.request_data_physical();
        SPHData out(y.sphConfig);
        check(sph_spat_op(y.h(), SPH_SPAT_MUL, y.data_spat, w, out.data_spat, 1.0, 0.0, y.sphConfig->spat_num_elems,
                          y.sphConfig->s()),
              "sph_spat_op");
        out.data_spat_valid = true;
        return out;
    }
};

// ------------------------------------------------------------------ SPHOperatorsComplex
// Replaces SPHOperatorsComplex (SPHOperatorsComplex.hpp): the same operators on
// complex fields (m = -L..L); grid-valued ones divide on the grid after one
// complex synthesis, as the reference does.
class SPHOperatorsComplex {
  public:
    // x i m, truncated (1 - mu^2) d/dmu under its three names, mu x, mu^2 x,
    // -n(n+1) x (SPHOperatorsComplex.hpp:27-50, 119-222, 430-470)
    static SPHDataComplex diff_lon(const SPHDataComplex& x) { return spec(SPH_OP_DIFF_LON, x); }
    static SPHDataComplex spec_one_minus_mu_squared_diff_lat_mu(const SPHDataComplex& x) { return spec(SPH_OP_D1MU2, x); }
    static SPHDataComplex spec_cosphi_squared_diff_lat_mu(const SPHDataComplex& x) { return spec(SPH_OP_D1MU2, x); }
    static SPHDataComplex spec_one_minus_sinphi_squared_diff_lat_mu(const SPHDataComplex& x) {
        return spec(SPH_OP_D1MU2, x);
    }
    static SPHDataComplex mu(const SPHDataComplex& x) { return spec(SPH_OP_MU, x); }
    static SPHDataComplex mu2(const SPHDataComplex& x) { return spec(SPH_OP_MU2, x); }
    static SPHDataComplex laplace(const SPHDataComplex& x) { return spec(SPH_OP_LAPLACE, x); }

    // I(i m x) / cos, I(D x) / cos, I(D x) / cos^2 (SPHOperatorsComplex.hpp:62-116, 224-282)
    static SPHDataComplex grad_lon(const SPHDataComplex& x) { return grid_mul(diff_lon(x), x.sphConfig->inv_cos_c()); }
    static SPHDataComplex grad_lat(const SPHDataComplex& x) {
        return grid_mul(spec_one_minus_mu_squared_diff_lat_mu(x), x.sphConfig->inv_cos_c());
    }
    static SPHDataComplex diff_lat_mu(const SPHDataComplex& x) {
        return grid_mul(spec_one_minus_mu_squared_diff_lat_mu(x), x.sphConfig->inv_cos2_c());
    }
    static SPHDataComplex diff_lat_phi(const SPHDataComplex& x) { return grad_lat(x); }
    // div_lon = grad_lon; div_lat = I(D F(cos x)) / cos^2 (SPHOperatorsComplex.hpp:284-344)
    static SPHDataComplex div_lon(const SPHDataComplex& x) { return grad_lon(x); }
    static SPHDataComplex div_lat(const SPHDataComplex& x) {
        const SPHDataComplex cx = grid_mul(x, x.sphConfig->cos_grid_c());
        return grid_mul(spec_one_minus_mu_squared_diff_lat_mu(cx), x.sphConfig->inv_cos2_c());
    }
    // Robert-variable operators (SPHOperatorsComplex.hpp:347-428)
    static SPHDataComplex robert_div_lon(const SPHDataComplex& x) {
        return grid_mul(diff_lon(x), x.sphConfig->inv_cos2_c());
    }
    static SPHDataComplex robert_div_lat(const SPHDataComplex& x) {
        return grid_mul(spec_cosphi_squared_diff_lat_mu(x), x.sphConfig->inv_cos2_c());
    }
    static SPHDataComplex robert_grad_lon(const SPHDataComplex& x) { return diff_lon(x); }
    static SPHDataComplex robert_grad_lat(const SPHDataComplex& x) { return spec_cosphi_squared_diff_lat_mu(x); }

    // vorticity and divergence (SPHOperatorsComplex.hpp:480-550); sums are spectral
    static SPHDataComplex vort(const SPHDataComplex& lon, const SPHDataComplex& lat) {
        return grad_lon(lat) - grad_lat(lon);
    }
    static SPHDataComplex robert_vort(const SPHDataComplex& lon, const SPHDataComplex& lat) {
        return robert_grad_lon(lat) - robert_grad_lat(lon);
    }
    static SPHDataComplex div(const SPHDataComplex& lon, const SPHDataComplex& lat) {
        return div_lon(lon) + div_lat(lat);
    }
    // one division: I(i m U + D V) / cos^2
    static SPHDataComplex robert_div(const SPHDataComplex& lon, const SPHDataComplex& lat) {
        return grid_mul(diff_lon(lon) + spec_cosphi_squared_diff_lat_mu(lat), lon.sphConfig->inv_cos2_c());
    }

  private:
    static SPHDataComplex spec(int op, const SPHDataComplex& x) {
        x.request_data_spectral();
        SPHDataComplex out(x.sphConfig);
        check(sph_spec_op(x.h(), op, reinterpret_cast<const double*>(x.data_spec),
                          reinterpret_cast<double*>(out.data_spec), 0.0, 0.0, 0.0, 0.0, 1, 1, x.sphConfig->s()),
              "sph_spec_op");
        out.data_spec_valid = true;
        return out;
    }
    // y times a real weight per grid point (w: the doubled grids of SPHConfig)
    static SPHDataComplex grid_mul(const SPHDataComplex& y, const double* w) {
        y.request_data_physical();
        SPHDataComplex out(y.sphConfig);
        check(sph_spat_op(y.h(), SPH_SPAT_MUL, reinterpret_cast<const double*>(y.data_spat), w,
                          reinterpret_cast<double*>(out.data_spat), 1.0, 0.0, 2LL * y.sphConfig->spat_num_elems,
                          y.sphConfig->s()),
              "sph_spat_op");
        out.data_spat_valid = true;
        return out;
    }
};

// ------------------------------------------------------------------ REXI
// Replaces REXI::setup (rexi/REXI.hpp:52-131): poles and weights of
// e^{ix} ~ sum_n beta_n / (ix + alpha_n).
class REXI {
  public:
    std::vector<cplx> alpha, beta_re, beta_im;
    void setup(double h, int M, int L = 0, bool half = true) {
        if (L != 0 && L != 11) throw std::runtime_error("REXI: only the L = 11 Gaussian approximation is available");
        int n = 0;
        check(sph_rexi_coefficients(h, M, half ? 1 : 0, 0, nullptr, nullptr, nullptr, &n), "sph_rexi_coefficients");
        alpha.assign(n, 0.0);
        beta_re.assign(n, 0.0);
        beta_im.assign(n, 0.0);
        check(sph_rexi_coefficients(h, M, half ? 1 : 0, n, reinterpret_cast<double*>(alpha.data()),
                                    reinterpret_cast<double*>(beta_re.data()), reinterpret_cast<double*>(beta_im.data()),
                                    &n),
              "sph_rexi_coefficients");
    }
};

// ------------------------------------------------------------------ time steppers
// The prognostic state of AppSWE: h, u, v (or U, V = u cos(phi), v cos(phi) with
// Robert functions) as spectral fields.
struct SWEParameters {
    double earth_radius = 6.37122e6;
    double gravitation = 9.80616;
    double coriolis_omega = 7.292e-5;
    double h0 = 10000.0;
    double viscosity2 = 1e5;
    bool use_nonlinear_equations = true;
    bool use_robert_functions = false;
    // full nonlinear equations in vorticity-divergence form with Robert
    // velocities on the grid (a form the reference does not have); the stepper's
    // prognostic fields are then h, vorticity, divergence
    bool use_vort_div_form = false;
};

// nonlinear / linear RK4 of AppSWE::run (AppSWE.hpp:293-336, TimesteppingRK.hpp:310-392):
// the three fields are packed into one device state and stepped by sph_swe_rk4.
class SWERK4 {
  public:
    SWERK4(SPHConfig* cfg, const SWEParameters& p) : cfg_(cfg), p_(p) {
        cuda_check(cudaMalloc(&state_, 3 * sizeof(cplx) * (size_t)cfg->spec_num_elems), "cudaMalloc");
    }
    ~SWERK4() { cudaFree(state_); }
    SWERK4(const SWERK4&) = delete;
    SWERK4& operator=(const SWERK4&) = delete;

    // advance (h, u, v) by nsteps steps of dt
    void run(SPHData& h, SPHData& u, SPHData& v, double dt, int nsteps) {
        pack(h, u, v);
        sph_swe_params sp = {p_.earth_radius, p_.gravitation, p_.coriolis_omega, p_.h0, p_.viscosity2, dt,
                             p_.use_vort_div_form ? 2 : (p_.use_nonlinear_equations ? 1 : 0),
                             p_.use_robert_functions ? 1 : 0};
        check(sph_swe_rk4(cfg_->handle(), &sp, reinterpret_cast<double*>(state_), nsteps, cfg_->s()), "sph_swe_rk4");
        unpack(h, u, v);
    }

  protected:
    SPHConfig* cfg_;
    SWEParameters p_;
    cplx* state_ = nullptr;

    void pack(const SPHData& h, const SPHData& u, const SPHData& v) {
        const size_t n = (size_t)cfg_->spec_num_elems;
        const SPHData* f[3] = {&h, &u, &v};
        for (int k = 0; k < 3; k++) {
            f[k]->request_data_spectral();
            cuda_check(cudaMemcpyAsync(state_ + k * n, f[k]->data_spec, n * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                       cfg_->stream),
                       "pack");
        }
    }
    void unpack(SPHData& h, SPHData& u, SPHData& v) {
        const size_t n = (size_t)cfg_->spec_num_elems;
        SPHData* f[3] = {&h, &u, &v};
        for (int k = 0; k < 3; k++) {
            cuda_check(cudaMemcpyAsync(f[k]->data_spec, state_ + k * n, n * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                       cfg_->stream),
                       "unpack");
            f[k]->data_spec_valid = true;
            f[k]->data_spat_valid = false;
        }
    }
};

// REXI time stepping of AppSWE::run (AppSWE.hpp:337-568) with the Robert
// formulation: the serial pole loop over SWERexiSPHRobert::setup/solve
// (SWERexiSPHRobert.hpp:68-258) is one sph_rexi_step over all poles.
// All poles of a REXI step in one launch per step: the pole loop of
// AppSWE::run (AppSWE.hpp:368-566) over SWERexiSPH (robert = false,
// SWERexiSPH.hpp) or SWERexiSPHRobert (robert = true, SWERexiSPHRobert.hpp);
// the state is (h, u, v), with the Robert velocities u cos(phi), v cos(phi) in
// the Robert form.
class SWERexi : public SWERK4 {
  public:
    SWERexi(SPHConfig* cfg, const SWEParameters& p, const REXI& rexi, double tau, bool robert,
            bool fix_z5robert = false, int precision = SPH_PREC_FP64)
        : SWERK4(cfg, p) {
        sph_rexi_params rp = {p.earth_radius, p.gravitation,          p.coriolis_omega, p.h0, p.viscosity2, tau,
                              robert ? 1 : 0, p.coriolis_omega != 0.0 ? 1 : 0, fix_z5robert ? 1 : 0, precision};
        check(sph_rexi_create(cfg->handle(), reinterpret_cast<const double*>(rexi.alpha.data()),
                              reinterpret_cast<const double*>(rexi.beta_re.data()), (int)rexi.alpha.size(), &rp, &r_),
              "sph_rexi_create");
    }
    ~SWERexi() {
        if (r_) sph_rexi_destroy(r_);
    }
    // advance (h, u, v) by nsteps steps of tau
    void run(SPHData& h, SPHData& u, SPHData& v, int nsteps) {
        pack(h, u, v);
        check(sph_rexi_step(r_, reinterpret_cast<double*>(state_), nsteps, cfg_->s()), "sph_rexi_step");
        unpack(h, u, v);
    }

  private:
    sph_rexi* r_ = nullptr;
};
class SWERexiRobert : public SWERexi {
  public:
    SWERexiRobert(SPHConfig* cfg, const SWEParameters& p, const REXI& rexi, double tau, bool fix_z5robert = false,
                  int precision = SPH_PREC_FP64)
        : SWERexi(cfg, p, rexi, tau, true, fix_z5robert, precision) {}
};

// One pole of the REXI sum: SWERexiSPH (SWERexiSPH.hpp:68-244) and
// SWERexiSPHRobert (SWERexiSPHRobert.hpp:68-258) share this body.  setup takes
// the pole alpha, weight beta (both divided by the time step here, as there)
// and the physical constants; solve returns this pole's Re(I(beta x)) for the
// geopotential phi0 and the velocities u0, v0 (the Robert velocities
// u cos(phi), v cos(phi) in the Robert form), which the caller sums over the
// poles as AppSWE::run does.  Each object is a one-pole plan of sph_rexi that
// factors its banded systems in every solve
// (sph_rexi_params.factor_each_step); SWERexi runs all poles of a step in one
// launch instead.
class SWERexiSPHPole {
  public:
    explicit SWERexiSPHPole(bool robert) : robert_(robert) {}
    SWERexiSPHPole(const SWERexiSPHPole&) = delete;
    SWERexiSPHPole& operator=(const SWERexiSPHPole&) = delete;
    SWERexiSPHPole(SWERexiSPHPole&& o) noexcept : robert_(o.robert_) { swap(o); }
    SWERexiSPHPole& operator=(SWERexiSPHPole&& o) noexcept {
        std::swap(robert_, o.robert_);
        swap(o);
        return *this;
    }
    ~SWERexiSPHPole() { release(); }

    void setup(SPHConfig* cfg, const cplx& alpha, const cplx& beta, double radius, double coriolis_omega,
               double avg_geopotential, double timestep_size, bool include_coriolis_effect = true) {
        release();
        cfg_ = cfg;
        sph_rexi_params rp{};
        rp.radius = radius;
        rp.gravity = 1.0;  // the state is the geopotential itself
        rp.omega = coriolis_omega;
        rp.h0 = avg_geopotential;
        rp.viscosity = 0.0;  // AppSWE applies viscosity after the pole sum
        rp.tau = timestep_size;
        rp.robert = robert_ ? 1 : 0;
        rp.coriolis = include_coriolis_effect ? 1 : 0;
        rp.fix_z5robert = 0;
        rp.precision = SPH_PREC_FP64;
        rp.factor_each_step = 1;
        const double ab[4] = {alpha.real(), alpha.imag(), beta.real(), beta.imag()};
        check(sph_rexi_create(cfg->handle(), ab, ab + 2, 1, &rp, &r_), "sph_rexi_create");
        cuda_check(cudaMalloc(&state_, 3 * sizeof(cplx) * (size_t)cfg->spec_num_elems), "cudaMalloc");
    }

    void solve(const SPHData& phi0, const SPHData& u0, const SPHData& v0, SPHData& o_phi, SPHData& o_u,
               SPHData& o_v) {
        if (!r_) throw std::runtime_error("SWERexiSPH: solve before setup");
        const size_t n = (size_t)cfg_->spec_num_elems;
        const SPHData* in[3] = {&phi0, &u0, &v0};
        for (int k = 0; k < 3; k++) {
            in[k]->request_data_spectral();
            cuda_check(cudaMemcpyAsync(state_ + k * n, in[k]->data_spec, n * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                       cfg_->stream),
                       "copy");
        }
        check(sph_rexi_step(r_, reinterpret_cast<double*>(state_), 1, cfg_->s()), "sph_rexi_step");
        SPHData* out[3] = {&o_phi, &o_u, &o_v};
        for (int k = 0; k < 3; k++) {
            if (out[k]->sphConfig != cfg_) *out[k] = SPHData(cfg_);
            cuda_check(cudaMemcpyAsync(out[k]->data_spec, state_ + k * n, n * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                       cfg_->stream),
                       "copy");
            out[k]->mark_spectral();
        }
    }
    // the reference's signature also passes its operator object, which holds no state
    void solve(const SPHData& phi0, const SPHData& u0, const SPHData& v0, SPHData& o_phi, SPHData& o_u, SPHData& o_v,
               const SPHOperatorsComplex&) {
        solve(phi0, u0, v0, o_phi, o_u, o_v);
    }

  private:
    bool robert_;
    SPHConfig* cfg_ = nullptr;
    sph_rexi* r_ = nullptr;
    cplx* state_ = nullptr;
    void swap(SWERexiSPHPole& o) noexcept {
        std::swap(cfg_, o.cfg_);
        std::swap(r_, o.r_);
        std::swap(state_, o.state_);
    }
    void release() {
        if (r_) sph_rexi_destroy(r_);
        if (state_) cudaFree(state_);
        r_ = nullptr;
        state_ = nullptr;
    }
};

// SWERexiSPH: the non-Robert form (velocities u, v; SWERexiSPH.hpp)
class SWERexiSPH : public SWERexiSPHPole {
  public:
    SWERexiSPH() : SWERexiSPHPole(false) {}
};
// SWERexiSPHRobert: the Robert form (velocities u cos(phi), v cos(phi); SWERexiSPHRobert.hpp)
class SWERexiSPHRobert : public SWERexiSPHPole {
  public:
    SWERexiSPHRobert() : SWERexiSPHPole(true) {}
};

}  // namespace sph_swe
