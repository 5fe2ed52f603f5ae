// REXI integrator (batched banded solves) — entry points.
#include "common.cuh"

using namespace sphgpu;

extern "C" {

int sph_rexi_create(sph_handle*, const double*, const double*, int, const sph_rexi_params*, sph_rexi** out) {
    if (out) *out = nullptr;
    set_error("sph_rexi_create: not available in this build");
    return SPH_ERR_ARG;
}

int sph_rexi_destroy(sph_rexi*) { return SPH_OK; }

int sph_rexi_step(sph_rexi*, double*, int, void*) {
    set_error("sph_rexi_step: not available in this build");
    return SPH_ERR_ARG;
}

}  // extern "C"
