// textures.cuh — texture sampling, normal-map decoding and the environment map on the GPU.
//
// Base-colour and normal textures follow Texture::sample (src/core/texture.cpp:100-139), which
// the reference evaluates in FP32 already: Repeat addressing, nearest or bilinear filtering of
// level 0, the image's origin at the top left and OBJ's UV origin at the bottom left. The path
// tracer samples at lod 0 (src/render/path_tracer.cpp:279-282), where trilinear filtering is
// level 0's bilinear value (the next level enters with weight 0), so no mip levels are stored.
// Products and sums are rounded one by one (no contraction), as the reference writes them.
//
// The environment map follows EnvironmentLight (src/render/light.cpp:61-195) in FP32: a lat-long
// map (+Y north, longitude 0 along +X increasing towards +Z, rotated about +Y), looked up
// bilinearly on level 0 (longitude wraps, latitude clamps, negative texels count as 0), sampled
// with 5% uniform sphere density and 95% by a luminance x solid-angle distribution over a grid of
// at most 1024x512 texels. The distribution is stored as a row marginal CDF and per-row
// conditional CDFs: in exact arithmetic the same texel and remapped offset as the reference's
// single CDF over all grid texels, with FP32 precision per row instead of per map.
#pragma once

#include "device_scene.cuh"

namespace mr {

// The uniform-sphere warp of shading.cuh (defined before this header is included there).
__device__ __forceinline__ f3 sample_sphere(float ux, float uy);

constexpr float kEnvironmentUniformFraction = 0.05f;  // light.cpp:15

__device__ __forceinline__ int wrap_index(int coordinate, int extent) {  // texture.cpp:13-15
    return (coordinate % extent + extent) % extent;
}

// x * (1 - a) + y * a per component, each operation rounded.
__device__ __forceinline__ f3 mix_rn(f3 x, f3 y, float a) {
    const float b = __fsub_rn(1.0f, a);
    return {__fadd_rn(__fmul_rn(x.x, b), __fmul_rn(y.x, a)), __fadd_rn(__fmul_rn(x.y, b), __fmul_rn(y.y, a)),
            __fadd_rn(__fmul_rn(x.z, b), __fmul_rn(y.z, a))};
}

__device__ __forceinline__ f3 texel_at(const DeviceScene& s, const DeviceTexture& t, int x, int y) {
    return xyz(__ldg(s.texels + t.offset + static_cast<size_t>(y) * t.width + x));
}

// Texture::sample at lod 0 (texture.cpp:100-139): nearest, or bilinear on level 0 (also for
// trilinear, whose second level has weight 0 at lod 0).
__device__ __forceinline__ f3 texture_sample(const DeviceScene& s, int texture, float u, float v,
                                             uint32_t filter) {
    const DeviceTexture t = s.textures[texture];
    // image_uv (texture.cpp:17-22): origin moved to the top left, Repeat addressing.
    const float cx = __fsub_rn(u, floorf(u));
    const float cy = __fsub_rn(1.0f, __fsub_rn(v, floorf(v)));
    const int   w = static_cast<int>(t.width), h = static_cast<int>(t.height);
    if (filter == MR_FILTER_NEAREST) {
        const int x = static_cast<int>(floorf(__fmul_rn(cx, static_cast<float>(w))));
        const int y = static_cast<int>(floorf(__fmul_rn(cy, static_cast<float>(h))));
        return texel_at(s, t, wrap_index(x, w), wrap_index(y, h));
    }
    const float x  = __fsub_rn(__fmul_rn(cx, static_cast<float>(w)), 0.5f);
    const float y  = __fsub_rn(__fmul_rn(cy, static_cast<float>(h)), 0.5f);
    const int   ix = static_cast<int>(floorf(x));
    const int   iy = static_cast<int>(floorf(y));
    const float tx = __fsub_rn(x, floorf(x));
    const float ty = __fsub_rn(y, floorf(y));
    const int   x0 = wrap_index(ix, w), x1 = wrap_index(ix + 1, w);
    const int   y0 = wrap_index(iy, h), y1 = wrap_index(iy + 1, h);
    return mix_rn(mix_rn(texel_at(s, t, x0, y0), texel_at(s, t, x1, y0), tx),
                  mix_rn(texel_at(s, t, x0, y1), texel_at(s, t, x1, y1), tx), ty);
}

// uv_tangents (src/geometry/uv_tangents.cpp:12-36) in FP32: the triangle's unit dP/du, dP/dv.
__device__ __forceinline__ bool uv_tangents(f3 p0, f3 p1, f3 p2, float2 c0, float2 c1, float2 c2, f3& u_axis,
                                            f3& v_axis) {
    const f3 a = p1 - p0, b = p2 - p0;
    float    sx = c1.x - c0.x, sy = c1.y - c0.y, tx = c2.x - c0.x, ty = c2.y - c0.y;
    const float scale = fmaxf(fmaxf(fabsf(sx), fabsf(sy)), fmaxf(fabsf(tx), fabsf(ty)));
    if (!isfinite(scale) || scale == 0) {
        return false;
    }
    sx /= scale, sy /= scale, tx /= scale, ty /= scale;
    const float determinant = sx * ty - sy * tx;
    if (!isfinite(determinant) || fabsf(determinant) < 1e-12f) {
        return false;
    }
    const f3    u  = (ty * a - sy * b) / determinant;
    const f3    v  = (-tx * a + sx * b) / determinant;
    const float lu = length(u), lv = length(v);
    if (!isfinite(lu) || !isfinite(lv) || lu == 0 || lv == 0) {
        return false;
    }
    u_axis = u / lu;
    v_axis = v / lv;
    return true;
}

// The normal-map step of SceneBvh::surface_hit (src/render/bvh.cpp:334-358): the texture's
// tangent-space normal in the triangle's UV frame around the interpolated shading normal, kept
// when it stays on the geometric side.
__device__ __forceinline__ f3 apply_normal_map(const DeviceScene& s, const DeviceMaterial& m, f3 shading,
                                               f3 geometric, f3 p0, f3 p1, f3 p2, float2 c0, float2 c1,
                                               float2 c2, float u, float v) {
    f3 axis_u, axis_v;
    if (!uv_tangents(p0, p1, p2, c0, c1, c2, axis_u, axis_v)) {
        return shading;
    }
    const f3 t0 = axis_u - shading * dot(axis_u, shading);
    if (!(dot(t0, t0) > 1e-12f)) {
        return shading;
    }
    const f3 t = normalize(t0);
    f3       b = cross(shading, t);
    if (dot(b, axis_v) < 0) {
        b = -b;
    }
    f3 sample = texture_sample(s, m.normal_texture, u, v, m.filter) * 2.0f - make(1.0f, 1.0f, 1.0f);
    sample.x *= m.normal_scale;
    sample.y *= m.normal_scale * (m.normal_flip_y ? -1.0f : 1.0f);
    const f3 mapped = t * sample.x + b * sample.y + shading * sample.z;
    return dot(mapped, geometric) > 1e-8f ? normalize(mapped) : shading;
}

// EnvironmentLight::coordinates (light.cpp:112-119).
__device__ __forceinline__ float2 environment_coordinates(const DeviceScene& s, f3 direction) {
    const f3 d = normalize(direction);
    float    u = (atan2f(d.z, d.x) + s.env_rotation) * (0.5f * kInvPi);
    u -= floorf(u);
    const float v = atan2f(hypotf(d.x, d.z), d.y) * kInvPi;
    return make_float2(u, v);
}

__device__ __forceinline__ f3 positive3(f3 c) { return {fmaxf(c.x, 0.0f), fmaxf(c.y, 0.0f), fmaxf(c.z, 0.0f)}; }

// EnvironmentLight::lookup (light.cpp:121-138).
__device__ __forceinline__ f3 environment_lookup(const DeviceScene& s, float2 uv) {
    const DeviceTexture t = s.textures[s.env_texture];
    const int   w = static_cast<int>(t.width), h = static_cast<int>(t.height);
    const float x = uv.x * static_cast<float>(w) - 0.5f;
    const float y = uv.y * static_cast<float>(h) - 0.5f;
    const int   ix = static_cast<int>(floorf(x)), iy = static_cast<int>(floorf(y));
    const float tx = x - floorf(x), ty = y - floorf(y);
    const int   x0 = wrap_index(ix, w), x1 = wrap_index(ix + 1, w);
    const int   y0 = min(max(iy, 0), h - 1), y1 = min(max(iy + 1, 0), h - 1);
    const auto  mix = [](f3 a, f3 b, float k) { return a * (1.0f - k) + b * k; };
    return mix(mix(positive3(texel_at(s, t, x0, y0)), positive3(texel_at(s, t, x1, y0)), tx),
               mix(positive3(texel_at(s, t, x0, y1)), positive3(texel_at(s, t, x1, y1)), tx), ty);
}

// EnvironmentLight::evaluate (light.cpp:140-143): the constant plus the map.
__device__ __forceinline__ f3 environment_radiance(const DeviceScene& s, f3 direction) {
    if (s.env_texture < 0) {
        return s.environment;
    }
    return s.environment + s.env_strength * environment_lookup(s, environment_coordinates(s, direction));
}

// EnvironmentLight::pdf (light.cpp:145-157): solid-angle density of sampling `direction`.
__device__ __forceinline__ float environment_density(const DeviceScene& s, f3 direction) {
    if (s.env_uniform) {
        return 1.0f / (4.0f * kPi);
    }
    const float2 uv = environment_coordinates(s, direction);
    const uint32_t x = min(static_cast<uint32_t>(uv.x * static_cast<float>(s.env_w)), s.env_w - 1);
    const uint32_t y = min(static_cast<uint32_t>(uv.y * static_cast<float>(s.env_h)), s.env_h - 1);
    const float*   row = s.env_col_cdf + static_cast<size_t>(y) * (s.env_w + 1);
    const float    p   = (__ldg(s.env_row_cdf + y + 1) - __ldg(s.env_row_cdf + y)) *
                     (__ldg(row + x + 1) - __ldg(row + x));
    return kEnvironmentUniformFraction / (4.0f * kPi) +
           (1.0f - kEnvironmentUniformFraction) * p / __ldg(s.env_solid_angle + y);
}

// upper_bound over cdf[0..n]: the entry i with cdf[i] <= u < cdf[i + 1], its mass and the
// remapped offset (u - cdf[i]) / mass below 1 (DiscreteDistribution::sample, sampling.cpp:129-139).
__device__ __forceinline__ uint32_t sample_cdf(const float* cdf, uint32_t n, float u, float& remapped) {
    uint32_t lo = 0, hi = n + 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) > u) {
            hi = mid;
        } else {
            lo = mid + 1;
        }
    }
    const uint32_t index = min(max(lo, 1u), n) - 1;
    const float    mass  = __ldg(cdf + index + 1) - __ldg(cdf + index);
    remapped             = fminf((u - __ldg(cdf + index)) / mass, 0.99999994039535522461f);
    return index;
}

// EnvironmentLight::sample (light.cpp:159-191): direction, radiance and density.
__device__ __forceinline__ f3 sample_environment(const DeviceScene& s, float ux, float uy, float& density,
                                                 f3& radiance) {
    f3 direction;
    if (s.env_uniform || ux < kEnvironmentUniformFraction) {
        direction = sample_sphere(s.env_uniform ? ux : ux / kEnvironmentUniformFraction, uy);
    } else {
        const float u = (ux - kEnvironmentUniformFraction) / (1.0f - kEnvironmentUniformFraction);
        float       u_row, remapped;
        const uint32_t y = sample_cdf(s.env_row_cdf, s.env_h, u, u_row);
        const uint32_t x = sample_cdf(s.env_col_cdf + static_cast<size_t>(y) * (s.env_w + 1), s.env_w, u_row, remapped);
        const float theta0     = kPi * static_cast<float>(y) / static_cast<float>(s.env_h);
        const float theta1     = kPi * static_cast<float>(y + 1) / static_cast<float>(s.env_h);
        const float difference = 2.0f * sinf((theta0 + theta1) * 0.5f) * sinf((theta1 - theta0) * 0.5f);
        const float v = fminf(fmaxf(uy, kFltEps * 0.5f), 0.99999994039535522461f);
        float cosine, sine;
        if (y < s.env_h / 2) {
            const float h = 1.0f - cosf(theta0) + v * difference;
            cosine        = 1.0f - h;
            sine          = sqrtf(fmaxf(0.0f, h * (2.0f - h)));
        } else {
            const float h = 1.0f + cosf(theta1) + (1.0f - v) * difference;
            cosine        = -1.0f + h;
            sine          = sqrtf(fmaxf(0.0f, h * (2.0f - h)));
        }
        const float phi = 2.0f * kPi * (static_cast<float>(x) + remapped) / static_cast<float>(s.env_w) -
                          s.env_rotation;
        direction = {sine * cosf(phi), cosine, sine * sinf(phi)};
    }
    radiance = environment_radiance(s, direction);
    density  = environment_density(s, direction);
    return direction;
}

}  // namespace mr
