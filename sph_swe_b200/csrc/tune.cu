// Autotuner for the kernel variants of a handle.
//
// For a batch size it times every candidate of
//   - the tensor-core Legendre synthesis and analysis (mixed handles): column
//     tile of 16, 32 or 64 real columns per CTA (8, 16, 32 fields) x kernel:
//     the int8 integer-split kernels (B prepared by a separate kernel and
//     loaded by the TMA unit, or staged by producer warps inside the kernel)
//     with the orders m ascending or paired with their complements (the
//     m-to-CTA schedule), the split-TF32 kernels with P
//     loaded by the TMA unit and B staged by producer warps, with both
//     operands loaded by the TMA unit (B prepared once per call), or with P
//     regenerated from recurrence checkpoints; and the FP64 tensor-core kernels
//     of the plain form (variant 16);
//   - the fixed-length ring FFTs (automatic grids): 2P rings per CTA with the
//     default P, twice or half of it (fewer or more CTAs per SM);
// with CUDA events on the caller's stream (one warm-up launch, then the mean
// of three), keeps the fastest in the handle (later calls with that batch
// use it) and writes the table as JSON.  sph_tune_load re-applies a table.
// Within a kernel family the variants are exact alternatives: neither the
// column tile nor the m order changes any arithmetic, the two P sources of the
// split-TF32 form differ in the last bits of P_l^m only.  Across families the
// results differ by the families' rounding (int8 ~1e-8, split TF32 ~3e-7
// relative).  sph_autotune takes the int8 and FP64 families, which keep every
// transform of velocity-derived fields within the mixed form's relL2 <= 1e-6;
// sph_autotune_ex chooses the families (the split-TF32 family meets 1e-6 for
// scalar fields only).
#include "common.cuh"

#include <cstdio>
#include <cstring>

namespace sphgpu {

namespace {

struct Scratch {
    void* p = nullptr;
    ~Scratch() {
        if (p) cudaFree(p);
    }
};

const char* kind_name(int k) {
    switch (k) {
        case TUNE_TC_SYNTHESIS: return "legendre_synthesis_tc";
        case TUNE_TC_ANALYSIS: return "legendre_analysis_tc";
        case TUNE_RING_ANALYSIS: return "ring_analysis";
        default: return "ring_synthesis";
    }
}

bool fixed_ring(int nphi) {
    return nphi == 96 || nphi == 192 || nphi == 384 || nphi == 768 || nphi == 1536 || nphi == 3072;
}

}  // namespace

// mean time (us) of `reps` launches of fn after one warm-up
template <class F>
static int time_us(cudaStream_t s, F&& fn, float* us) {
    cudaEvent_t e0, e1;
    SPH_CUDA_TRY(cudaEventCreate(&e0));
    SPH_CUDA_TRY(cudaEventCreate(&e1));
    int rc = fn();
    const int reps = 3;
    if (!rc) rc = (cudaEventRecord(e0, s) == cudaSuccess) ? SPH_OK : SPH_ERR_CUDA;
    for (int i = 0; i < reps && !rc; i++) rc = fn();
    if (!rc) rc = (cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess) ? SPH_OK
                                                                                                       : SPH_ERR_CUDA;
    float ms = 0.f;
    if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *us = ms * 1000.f / reps;
    if (rc == SPH_ERR_CUDA) set_error("autotune: timing failed");
    return rc;
}

static int autotune(Handle* h, int batch, int families, std::string& json, cudaStream_t s) {
    const int L = h->L, mF = L + 1;
    const long long fou = (long long)mF * h->nlat;
    const size_t bspec = sizeof(double2) * (size_t)h->nlm * batch, bF = sizeof(double2) * (size_t)fou * batch,
                 bgrid = sizeof(double) * (size_t)h->nspat * batch;
    Scratch sc;
    SPH_CUDA_TRY(cudaMalloc(&sc.p, bspec + bF + bgrid));
    SPH_CUDA_TRY(cudaMemsetAsync(sc.p, 0, bspec + bF + bgrid, s));
    double2* spec = static_cast<double2*>(sc.p);
    double2* F = reinterpret_cast<double2*>(static_cast<char*>(sc.p) + bspec);
    double* grid = reinterpret_cast<double*>(static_cast<char*>(sc.p) + bspec + bF);

    char buf[256];
    json = "{\"lmax\": " + std::to_string(L) + ", \"nlat\": " + std::to_string(h->nlat) + ", \"nphi\": " +
           std::to_string(h->nphi) + ", \"precision\": " + std::to_string(h->flags & SPH_PREC_MIXED) +
           ", \"batch\": " + std::to_string(batch) + ", \"kernels\": [";
    bool first_kind = true;
    for (int kind = 0; kind < 4; kind++) {
        std::vector<int> cand;
        if (kind <= TUNE_TC_ANALYSIS) {
            if (!h->mixed) continue;
            // int8 kernels with both operands by TMA (0) or B staged by producer
            // warps (128), in ascending or paired (+64) m order; split TF32 with
            // B staged by producer warps (32), both operands loaded by the TMA unit
            // (8), P regenerated (4)
            if (families & SPH_TUNE_INT8)
                for (int src : {0, 64, 128, 192})
                    for (int c = 1; c <= 3; c++) cand.push_back(src | c);
            if (families & SPH_TUNE_TF32)
                for (int src : {32, 8, 4})
                    for (int c = 1; c <= 3; c++) cand.push_back(src | c);
            if (families & SPH_TUNE_FP64) cand.push_back(16);  // FP64 kernels of the plain form
            if (cand.empty()) continue;
        } else {
            if (!fixed_ring(h->nphi)) continue;
            cand = {0, 1, 2};
        }
        const long long key = ((long long)kind << 32) | (unsigned)batch;
        h->tune.erase(key);
        int best = cand[0];
        float best_us = 1e30f;
        std::string tried;
        for (int v : cand) {
            h->tune[key] = v;
            float us = 0.f;
            auto run = [&]() -> int {
                switch (kind) {
                    case TUNE_TC_SYNTHESIS: return legendre_synthesis_real(h, spec, h->nlm, L, F, fou, batch, s);
                    case TUNE_TC_ANALYSIS: return legendre_analysis_real(h, F, fou, spec, h->nlm, L, batch, s);
                    case TUNE_RING_ANALYSIS: return ring_analysis_real(h, grid, h->nspat, F, fou, mF, batch, s);
                    default: return ring_synthesis_real(h, F, fou, mF, grid, h->nspat, batch, nullptr, nullptr, 0, 0, s);
                }
            };
            if (int rc = time_us(s, run, &us)) {
                h->tune.erase(key);
                return rc;
            }
            std::snprintf(buf, sizeof buf, "%s{\"variant\": %d, \"us\": %.2f}", tried.empty() ? "" : ", ", v, us);
            tried += buf;
            if (us < best_us) {
                best_us = us;
                best = v;
            }
        }
        h->tune[key] = best;
        std::snprintf(buf, sizeof buf, "%s{\"kind\": %d, \"name\": \"%s\", \"batch\": %d, \"variant\": %d, \"us\": %.2f, ",
                      first_kind ? "" : ", ", kind, kind_name(kind), batch, best, best_us);
        json += buf;
        json += "\"candidates\": [" + tried + "]}";
        first_kind = false;
    }
    json += "]}";
    rk_invalidate(h);  // a captured RK4 step graph holds the previous variants
    if (int rc = tc_check(h)) return rc;
    return SPH_OK;
}

// entries "kind": k, ... "batch": b, "variant": v in that order, as autotune writes them
static int tune_load(Handle* h, const char* json) {
    const char* lm = std::strstr(json, "\"lmax\":");
    const char* np = std::strstr(json, "\"nphi\":");
    if (!lm || !np || std::atoi(lm + 7) != h->L || std::atoi(np + 7) != h->nphi) {
        set_error("sph_tune_load: the table is for another truncation or grid");
        return SPH_ERR_ARG;
    }
    const char* p = json;
    int n = 0;
    while ((p = std::strstr(p, "\"kind\":")) != nullptr) {
        int kind = -1, batch = -1, var = -1;
        const char* q = p;
        kind = std::atoi(q + 7);
        const char* b = std::strstr(q, "\"batch\":");
        const char* v = b ? std::strstr(b, "\"variant\":") : nullptr;
        if (!b || !v) break;
        batch = std::atoi(b + 8);
        var = std::atoi(v + 10);
        if (kind < 0 || kind > 3 || batch <= 0 || var < 0 || var > 255) {
            set_error("sph_tune_load: malformed entry");
            return SPH_ERR_ARG;
        }
        h->tune[((long long)kind << 32) | (unsigned)batch] = var;
        n++;
        p = v;
    }
    if (n == 0) {
        set_error("sph_tune_load: no entries");
        return SPH_ERR_ARG;
    }
    rk_invalidate(h);
    return SPH_OK;
}

}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

int sph_autotune_ex(sph_handle* hh, int batch, int families, char* json, int cap, void* stream) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || batch <= 0 || batch > 65535 || (json && cap <= 0) || families <= 0 ||
        (families & ~(SPH_TUNE_INT8 | SPH_TUNE_TF32 | SPH_TUNE_FP64))) {
        set_error("sph_autotune: bad arguments");
        return SPH_ERR_ARG;
    }
    std::string out;
    if (int rc = autotune(h, batch, families, out, reinterpret_cast<cudaStream_t>(stream))) return rc;
    if (json) {
        if ((int)out.size() + 1 > cap) {
            set_error("sph_autotune: json buffer too small (" + std::to_string(out.size() + 1) + " bytes needed)");
            return SPH_ERR_ARG;
        }
        std::memcpy(json, out.c_str(), out.size() + 1);
    }
    return SPH_OK;
}

int sph_autotune(sph_handle* hh, int batch, char* json, int cap, void* stream) {
    return sph_autotune_ex(hh, batch, SPH_TUNE_INT8 | SPH_TUNE_FP64, json, cap, stream);
}

int sph_tune_load(sph_handle* hh, const char* json) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !json) {
        set_error("sph_tune_load: bad arguments");
        return SPH_ERR_ARG;
    }
    return tune_load(h, json);
}

int sph_tune_clear(sph_handle* hh) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) {
        set_error("sph_tune_clear: NULL handle");
        return SPH_ERR_ARG;
    }
    h->tune.clear();
    rk_invalidate(h);
    return SPH_OK;
}

}  // extern "C"
