// Real synthesis that allocates nothing (sph_SH_to_spat_noalloc).
//
// sph_SH_to_spat keeps its Fourier-space intermediate in a workspace that the
// handle grows with cudaMalloc on demand.  Some callers cannot call cudaMalloc
// (or let a library call it for them) once they are running: a host program
// whose own allocator has already reserved the device memory, so a late
// cudaMalloc fails or fragments the pool, and code on a latency budget that
// must not stall, since cudaMalloc / cudaFree can synchronise the device.
// This variant keeps the intermediate in a fixed, file-scope device array
// instead.
#include "common.cuh"

#include <mutex>

namespace sphgpu {
namespace {

// 8 MiB of scratch: (L+1)*nlat*16 bytes per field, i.e. at most 5 fields at
// T255 (384 latitudes), 85 at T63, 1 at T511.  The library is built without
// relocatable device code, so this array sits in a device module of its own,
// and with lazy module loading (the CUDA default) the driver reserves its
// 8 MiB only when the module is first touched.  sph_create touches it (through
// noalloc_scratch) on the handle's device, while allocating is still allowed;
// from then on the device holds the array until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
__device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double2)];

// Device address of the array, looked up once per device with that device
// current (the symbol's name in host code is only a host-side stand-in and
// must not reach a kernel).
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

}  // namespace

int noalloc_scratch(int dev, void** out) {
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("sph_SH_to_spat_noalloc: device index out of range");
        return SPH_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("sph_SH_to_spat_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return SPH_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return SPH_OK;
}

}  // namespace sphgpu

using namespace sphgpu;

extern "C" int sph_SH_to_spat_noalloc(sph_handle* hh, const double* spec, double* spat, int batch, void* stream) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || batch < 0 || (batch > 0 && (!spec || !spat))) {
        set_error("sph_SH_to_spat_noalloc: bad arguments");
        return SPH_ERR_ARG;
    }
    if (batch == 0) return SPH_OK;
    const int mF = h->L + 1;
    const long long ldF = (long long)mF * h->nlat;
    const size_t need = sizeof(double2) * (size_t)ldF * (size_t)batch;
    if (need > kNoAllocScratchBytes) {
        const size_t per = sizeof(double2) * (size_t)ldF;
        set_error("sph_SH_to_spat_noalloc: " + std::to_string(batch) + " fields need " + std::to_string(need) +
                  " bytes of scratch; the fixed scratch holds " + std::to_string(kNoAllocScratchBytes) +
                  " bytes, i.e. at most " + std::to_string(kNoAllocScratchBytes / per) +
                  " fields per call at this truncation");
        return SPH_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("sph_SH_to_spat_noalloc: ") + cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    if (dev != h->device) {
        set_error("sph_SH_to_spat_noalloc: the current device is not the handle's device");
        return SPH_ERR_ARG;
    }
    // a mixed handle whose autotuned synthesis variant for this batch is the
    // loader-only kernel needs the handle's prepared-operand buffer; if that
    // buffer has not been grown yet (by an allocating call with this batch),
    // using the variant here would allocate, so refuse instead
    if ((h->flags & SPH_PREC_MIXED) && tc_synthesis_needs_alloc(h, h->L, batch)) {
        set_error("sph_SH_to_spat_noalloc: the autotuned tensor-core variant for " + std::to_string(batch) +
                  " fields needs a workspace this handle has not reserved; make one allocating call "
                  "(sph_SH_to_spat) with this batch first, or clear the tuning (sph_tune_clear)");
        return SPH_ERR_ARG;
    }
    void* scratch = nullptr;
    if (int rc = noalloc_scratch(dev, &scratch)) return rc;
    double2* F = static_cast<double2*>(scratch);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the Legendre stage writes every (m <= L, j) entry of each field's slice
    // before the longitude stage reads it, so no part of the scratch has to
    // start at zero
    if (int rc = legendre_synthesis_real(h, reinterpret_cast<const double2*>(spec), h->nlm, h->L, F, ldF, batch, s, 0,
                                         1))
        return rc;
    return ring_synthesis_real(h, F, ldF, mF, spat, h->nspat, batch, nullptr, nullptr, 0, 0, s);
}
