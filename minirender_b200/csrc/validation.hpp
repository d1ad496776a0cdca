// validation.hpp — the reference's settings validation, shared by every entry point that takes
// integrator or render settings.
#pragma once

#include "errors.hpp"
#include "wavefront.cuh"

namespace mr {

// IntegratorSettings::validate (src/render/path_tracer.cpp:55-64).
inline IntegratorParams integrator_params(const mr_integrator_settings* s) {
    IntegratorParams p{MR_SAMPLING_MIS, 8, 1, 3};
    if (s) {
        p = {s->mode, s->maximum_depth, s->russian_roulette ? 1u : 0u, s->roulette_depth};
    }
    require(p.mode <= MR_SAMPLING_MIS, "Sampling mode must be bsdf, light or mis");
    require(p.maximum_depth <= 128 && p.roulette_depth <= 128,
            "Path and roulette depths must not exceed 128");
    return p;
}

// RenderSettings::validate (src/render/path_tracer.cpp:66-71).
inline void validate_render(const mr_render_settings* r) {
    require(r != nullptr, "Render settings are missing");
    if (r->width == 0 || r->height == 0 || r->width > 16384 || r->height > 16384 ||
        r->width * r->height > 64ull * 1024 * 1024 || r->samples_per_pixel == 0) {
        fail(MR_INVALID_ARGUMENT, "Render dimensions or sample count exceed the image budget");
    }
}

}  // namespace mr
