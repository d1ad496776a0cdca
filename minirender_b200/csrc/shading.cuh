// shading.cuh — FP32 restatement of the reference's per-vertex math: warps, camera rays, surface
// hit reconstruction, ray offsetting, BSDFs, light sampling and homogeneous media.
// Each function cites the reference function it follows.
#pragma once

#include "device_scene.cuh"
#include "rng.cuh"
#include "traverse.cuh"

namespace mr {

// ---- warps (src/core/sampling.cpp:67-107) ----

__device__ __forceinline__ void sample_disk(float ux, float uy, float& dx, float& dy) {
    const float sx = 2.0f * ux - 1.0f;
    const float sy = 2.0f * uy - 1.0f;
    if (sx == 0 && sy == 0) {
        dx = dy = 0;
        return;
    }
    const bool  horizontal = fabsf(sx) > fabsf(sy);
    const float radius     = horizontal ? sx : sy;
    const float angle      = horizontal ? (kPi / 4) * (sy / sx) : kPi / 2 - (kPi / 4) * (sx / sy);
    float       s, c;
    sincosf(angle, &s, &c);
    dx = radius * c;
    dy = radius * s;
}

__device__ __forceinline__ f3 sample_sphere(float ux, float uy) {
    const float z      = 1.0f - 2.0f * ux;
    const float radius = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float       s, c;
    sincosf(2.0f * kPi * uy, &s, &c);
    return {radius * c, radius * s, z};
}

}  // namespace mr

#include "textures.cuh"

namespace mr {

__device__ __forceinline__ f3 sample_cosine_hemisphere(float ux, float uy) {
    float dx, dy;
    sample_disk(ux, uy, dx, dy);
    return {dx, dy, sqrtf(fmaxf(0.0f, 1.0f - (dx * dx + dy * dy)))};
}

__device__ __forceinline__ f3 sample_triangle(float ux, float uy) {
    const float root = sqrtf(ux);
    return {1.0f - root, root * (1.0f - uy), root * uy};
}

// ---- camera (src/scene/scene.cpp:171-199, src/render/path_tracer.cpp:368-386) ----

struct CameraRay {
    f3    origin, direction;
    float minimum, maximum;
};

__device__ __forceinline__ CameraRay camera_ray(const CameraBasis& c, float u, float v,
                                                float aspect, float lens_x, float lens_y) {
    const f3 pinhole = normalize(c.forward + ((2.0f * u - 1.0f) * aspect * c.half_height) * c.right +
                                 ((1.0f - 2.0f * v) * c.half_height) * c.up);
    CameraRay r;
    r.origin    = c.position;
    r.direction = pinhole;
    if (c.aperture_radius != 0.0f) {
        float dx, dy;
        sample_disk(lens_x, lens_y, dx, dy);
        dx *= c.aperture_radius;
        dy *= c.aperture_radius;
        const f3 focus  = c.position + pinhole * (c.focus_distance / dot(pinhole, c.forward));
        const f3 origin = c.position + dx * c.right + dy * c.up;
        r.origin        = origin;
        r.direction     = normalize(focus - origin);
    }
    const float cosine = dot(r.direction, c.forward);
    r.minimum          = c.near_plane / cosine;
    r.maximum          = c.far_plane / cosine;
    return r;
}

// ---- surface hit (src/render/bvh.cpp:302-370) ----

struct SurfaceHit {
    f3       position;
    f3       position_error;
    f3       geometric_normal;
    f3       shading_normal;
    float    u, v;  // interpolated corner UVs (0 when the scene has no textures)
    bool     front_face;
    uint32_t instance, triangle, material, prim;
};

// `slot` is the hit's triangle slot (two-level scenes: its flat primitive id). A two-level scene
// (TWO and s.two_level) rebuilds the triangle's world vertices and corner normals from its mesh
// with the flattening's arithmetic, so the hit is the flattened scene's bit for bit.
template <bool TWO = false>
__device__ __forceinline__ SurfaceHit surface_hit(const DeviceScene& s, f3 direction,
                                                  uint32_t slot, float b0, float b1, float b2) {
    f3       v0, v1, v2, m0, m1, m2;
    float2   c0 = make_float2(0, 0), c1 = c0, c2 = c0;  // corner UVs
    uint32_t prim, flags, instance, triangle, material;
    if (TWO && s.two_level) {
        prim                        = slot;
        instance                    = find_instance2(s.instances, s.instance_count, prim);
        const DeviceInstance2& inst = s.instances[instance];
        triangle                    = prim - inst.first_prim;
        material                    = inst.material;
        flags                       = inst.flags;
        const mr_mesh_corner* c     = s.mesh_corners + inst.corner_offset + 3 * static_cast<size_t>(triangle);
        const float*          pos   = s.mesh_positions + 3 * static_cast<size_t>(inst.position_offset);
        const float*          p0    = pos + 3 * static_cast<size_t>(c[0].position);
        const float*          p1    = pos + 3 * static_cast<size_t>(c[1].position);
        const float*          p2    = pos + 3 * static_cast<size_t>(c[2].position);
        v0 = transform_point(inst.to_world, p0[0], p0[1], p0[2]);
        v1 = transform_point(inst.to_world, p1[0], p1[1], p1[2]);
        v2 = transform_point(inst.to_world, p2[0], p2[1], p2[2]);
        m0 = world_normal(inst.normal_to_world, c[0].normal);
        m1 = world_normal(inst.normal_to_world, c[1].normal);
        m2 = world_normal(inst.normal_to_world, c[2].normal);
        if (s.textures) {
            c0 = make_float2(c[0].uv[0], c[0].uv[1]);
            c1 = make_float2(c[1].uv[0], c[1].uv[1]);
            c2 = make_float2(c[2].uv[0], c[2].uv[1]);
        }
    } else {
        const float4* tp = s.tris + 3 * static_cast<size_t>(slot);
        const float4  a4 = __ldg(tp + 0), b4 = __ldg(tp + 1), c4 = __ldg(tp + 2);
        v0    = xyz(a4), v1 = xyz(b4), v2 = xyz(c4);
        prim  = __float_as_uint(a4.w);
        flags = __float_as_uint(b4.w);
        const float4* sp = s.shading + 3 * static_cast<size_t>(prim);
        const float4  n0 = __ldg(sp + 0), n1 = __ldg(sp + 1), n2 = __ldg(sp + 2);
        m0       = xyz(n0), m1 = xyz(n1), m2 = xyz(n2);
        instance = __float_as_uint(n0.w);
        triangle = __float_as_uint(n1.w);
        material = __float_as_uint(n2.w);
        if (s.uvs) {
            c0 = __ldg(s.uvs + 3 * static_cast<size_t>(prim));
            c1 = __ldg(s.uvs + 3 * static_cast<size_t>(prim) + 1);
            c2 = __ldg(s.uvs + 3 * static_cast<size_t>(prim) + 2);
        }
    }
    SurfaceHit h;
    f3 geometric = normalize(cross(v1 - v0, v2 - v0));
    if (flags & kTriMirrored) {
        geometric = -geometric;
    }
    f3 shading = b0 * m0 + b1 * m1 + b2 * m2;
    const f3 t0 = b0 * v0, t1 = b1 * v1, t2 = b2 * v2;
    h.position       = t0 + t1 + t2;
    h.position_error = (fabs3(t0) + fabs3(t1) + fabs3(t2)) * (7.0f * kFltEps);
    if (dot(shading, shading) < 1e-24f) {
        shading = geometric;
    } else {
        shading = normalize(shading);
        if (dot(shading, geometric) < 0) {
            shading = -shading;
        }
    }
    h.u = b0 * c0.x + b1 * c1.x + b2 * c2.x;
    h.v = b0 * c0.y + b1 * c1.y + b2 * c2.y;
    if (s.textures) {
        const DeviceMaterial& m = s.materials[material];
        if (m.normal_texture >= 0 && m.normal_scale > 0) {
            shading = apply_normal_map(s, m, shading, geometric, v0, v1, v2, c0, c1, c2, h.u, h.v);
        }
    }
    h.geometric_normal = geometric;
    h.shading_normal   = shading;
    h.front_face       = dot(direction, geometric) < 0;
    h.instance         = instance;
    h.triangle         = triangle;
    h.material         = material;
    h.prim             = prim;
    return h;
}

// offset_origin (src/render/path_tracer.cpp:87-105) with FP32 error bounds.
__device__ __forceinline__ f3 offset_origin(f3 position, f3 geometric_normal, f3 position_error,
                                            f3 direction) {
    f3 normal = normalize(geometric_normal);
    if (dot(normal, direction) < 0) {
        normal = -normal;
    }
    const float distance = fmaxf(dot(fabs3(normal), position_error), kFltMin);
    f3          origin   = position + distance * normal;
    origin.x = normal.x != 0 ? nextafterf(origin.x, copysignf(INFINITY, normal.x)) : origin.x;
    origin.y = normal.y != 0 ? nextafterf(origin.y, copysignf(INFINITY, normal.y)) : origin.y;
    origin.z = normal.z != 0 ? nextafterf(origin.z, copysignf(INFINITY, normal.z)) : origin.z;
    return origin;
}

// ---- frames and BSDFs (src/render/bsdf.cpp) ----

struct Frame {  // ShadingFrame (bsdf.cpp:89-110)
    f3 t, b, n;
    __device__ __forceinline__ void init(f3 normal) {
        const float maximum = fmaxf(fmaxf(fabsf(normal.x), fabsf(normal.y)), fabsf(normal.z));
        n                   = normalize(normal / maximum);
        const f3 helper     = fabsf(n.z) < 0.999f ? make(0, 0, 1) : make(0, 1, 0);
        t                   = normalize(cross(helper, n));
        b                   = cross(n, t);
    }
    __device__ __forceinline__ f3 to_local(f3 w) const { return {dot(w, t), dot(w, b), dot(w, n)}; }
    __device__ __forceinline__ f3 to_world(f3 l) const { return l.x * t + l.y * b + l.z * n; }
};

__device__ __forceinline__ float ggx_d(f3 m, float alpha) {  // bsdf.cpp:36-41
    const float a2          = alpha * alpha;
    const float denominator = m.x * m.x + m.y * m.y + a2 * m.z * m.z;
    return m.z > 0 ? a2 / (kPi * denominator * denominator) : 0.0f;
}

__device__ __forceinline__ float smith_g1_over_cosine(f3 v, float alpha) {  // bsdf.cpp:43-48
    if (v.z <= 0) {
        return 0.0f;
    }
    return 2.0f / (v.z + sqrtf(v.z * v.z + alpha * alpha * (v.x * v.x + v.y * v.y)));
}

__device__ __forceinline__ float fresnel_from_transmission(float cosine, float sin2, float eta_i,
                                                           float eta_t) {  // bsdf.cpp:51-64
    if (eta_i == eta_t) {
        return 0.0f;
    }
    if (sin2 >= 1) {
        return 1.0f;
    }
    const float tc            = sqrtf(1.0f - sin2);
    const float parallel      = (eta_t * cosine - eta_i * tc) / (eta_t * cosine + eta_i * tc);
    const float perpendicular = (eta_i * cosine - eta_t * tc) / (eta_i * cosine + eta_t * tc);
    return 0.5f * (parallel * parallel + perpendicular * perpendicular);
}

__device__ __forceinline__ f3 schlick(f3 f0, float cosine) {  // bsdf.cpp:66-69
    const float t  = 1.0f - fminf(fmaxf(cosine, 0.0f), 1.0f);
    const float t5 = t * t * t * t * t;
    return f0 + (make(1, 1, 1) - f0) * t5;
}

__device__ __forceinline__ f3 sample_visible_normal(f3 wo, float ux, float uy,
                                                    float alpha) {  // bsdf.cpp:72-85
    const f3    view  = normalize(make(alpha * wo.x, alpha * wo.y, wo.z));
    const float lensq = view.x * view.x + view.y * view.y;
    const f3    t1    = lensq > 0 ? make(-view.y, view.x, 0) / sqrtf(lensq) : make(1, 0, 0);
    const f3    t2    = cross(view, t1);
    const float radius = sqrtf(ux);
    float       s, c;
    sincosf(2.0f * kPi * uy, &s, &c);
    const float x     = radius * c;
    const float blend = 0.5f * (1.0f + view.z);
    const float y     = (1.0f - blend) * sqrtf(fmaxf(0.0f, 1.0f - x * x)) + blend * radius * s;
    const f3 normal   = x * t1 + y * t2 + sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y)) * view;
    return normalize(make(alpha * normal.x, alpha * normal.y, fmaxf(0.0f, normal.z)));
}

struct Bsdf {  // Bsdf (bsdf.cpp:122-277) without cloth, subsurface and energy compensation
    f3       color;
    float    alpha, eta_i, eta_t;
    uint32_t kind;

    // color = base_color * clamp(texture colour, 0, 1) (bsdf.cpp:122-141).
    __device__ __forceinline__ void init(const DeviceMaterial& m, bool front_face,
                                         f3 texture_color = make(1.0f, 1.0f, 1.0f)) {
        color = m.base_color * make(fminf(fmaxf(texture_color.x, 0.0f), 1.0f),
                                    fminf(fmaxf(texture_color.y, 0.0f), 1.0f),
                                    fminf(fmaxf(texture_color.z, 0.0f), 1.0f));
        alpha = m.alpha;
        eta_i = front_face ? 1.0f : m.ior;
        eta_t = front_face ? m.ior : 1.0f;
        kind  = m.kind;
    }
    __device__ __forceinline__ bool is_delta() const {
        return kind == MR_MATERIAL_MIRROR || kind == MR_MATERIAL_DIELECTRIC ||
               (kind == MR_MATERIAL_CONDUCTOR && alpha <= 1e-6f);
    }
    __device__ __forceinline__ f3 evaluate(f3 wo, f3 wi) const {
        if (wo.z <= 0 || wi.z <= 0 || is_delta()) {
            return make(0, 0, 0);
        }
        if (kind == MR_MATERIAL_DIFFUSE) {
            return color * kInvPi;
        }
        const f3 m = normalize(wo + wi);
        return schlick(color, dot(wo, m)) *
               (ggx_d(m, alpha) * smith_g1_over_cosine(wo, alpha) *
                smith_g1_over_cosine(wi, alpha) / 4.0f);
    }
    __device__ __forceinline__ float pdf(f3 wo, f3 wi) const {
        if (wo.z <= 0 || wi.z <= 0 || is_delta()) {
            return 0.0f;
        }
        if (kind == MR_MATERIAL_DIFFUSE) {
            return fmaxf(0.0f, wi.z) * kInvPi;
        }
        const f3 m = normalize(wo + wi);
        return ggx_d(m, alpha) * smith_g1_over_cosine(wo, alpha) / 4.0f;
    }

    struct Sample {
        f3    direction, weight;
        float probability, eta;
        bool  discrete, transmission;
    };

    // Returns false for the reference's std::nullopt (including the GGX null event).
    __device__ __forceinline__ bool sample(f3 wo, float component, float ux, float uy,
                                           Sample& s) const {
        if (wo.z <= 0) {
            return false;
        }
        const f3 reflected = make(-wo.x, -wo.y, wo.z);
        if (kind == MR_MATERIAL_DIELECTRIC) {
            const float ratio = eta_i / eta_t;
            const float sin2  = ratio * ratio * (wo.x * wo.x + wo.y * wo.y);
            const float reflectance =
                fresnel_from_transmission(fminf(fmaxf(wo.z, 0.0f), 1.0f), sin2, eta_i, eta_t);
            s.discrete = true;
            if (component < reflectance) {
                s.direction    = reflected;
                s.weight       = make(1, 1, 1);
                s.probability  = reflectance;
                s.eta          = 1.0f;
                s.transmission = false;
                return true;
            }
            s.direction    = make(-ratio * wo.x, -ratio * wo.y, -sqrtf(fmaxf(0.0f, 1.0f - sin2)));
            s.weight       = color * (ratio * ratio);
            s.probability  = 1.0f - reflectance;
            s.eta          = eta_t / eta_i;
            s.transmission = true;
            return true;
        }
        s.transmission = false;
        s.eta          = 1.0f;
        if (is_delta()) {
            s.direction   = reflected;
            s.weight      = kind == MR_MATERIAL_MIRROR ? color : schlick(color, wo.z);
            s.probability = 1.0f;
            s.discrete    = true;
            return true;
        }
        f3 wi;
        if (kind == MR_MATERIAL_DIFFUSE) {
            wi = sample_cosine_hemisphere(ux, uy);
        } else {
            const f3 m = sample_visible_normal(wo, ux, uy, alpha);
            wi         = normalize(2.0f * dot(wo, m) * m - wo);
        }
        if (wi.z <= 0) {
            return false;
        }
        const f3    evaluated = normalize(wi);
        const float density   = pdf(wo, evaluated);
        s.direction           = wi;
        s.weight              = evaluate(wo, evaluated) * (wi.z / density);
        s.probability         = density;
        s.discrete            = false;
        return true;
    }
};

__device__ __forceinline__ float power_heuristic(float sampled, float other) {  // path_tracer.cpp:73-85
    const float scale = fmaxf(sampled, other);
    if (scale == 0) {
        return 0.0f;
    }
    const float a = sampled / scale;
    const float b = other / scale;
    return a * a / (a * a + b * b);
}

// ---- lights (src/render/light.cpp) ----

__device__ __forceinline__ float area_density(f3 reference, f3 point, f3 normal,
                                              float area) {  // light.cpp:49-57
    const f3    difference       = point - reference;
    const float squared_distance = dot(difference, difference);
    if (squared_distance == 0) {
        return 0.0f;
    }
    const float cosine = fabsf(dot(normal, -difference / sqrtf(squared_distance)));
    return cosine > 0 ? squared_distance / (area * cosine) : 0.0f;
}

struct LightSample {
    f3    direction, radiance;
    float distance, probability;
    bool  discrete;
    f3    position, normal, position_error;
};

// DiscreteDistribution::sample (sampling.cpp:129-139): upper_bound over the CDF.
__device__ __forceinline__ int select_light(const DeviceScene& s, float u, float& mass) {
    int lo = 0, hi = static_cast<int>(s.light_count) + 1;  // first cdf entry > u in [lo, hi)
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(s.light_cdf + mid) > u) {
            hi = mid;
        } else {
            lo = mid + 1;
        }
    }
    const int index = lo - 1;
    mass            = __ldg(s.light_cdf + index + 1) - __ldg(s.light_cdf + index);
    return index;
}

// LightSampler::sample (light.cpp:266-321).
__device__ __forceinline__ bool sample_light(const DeviceScene& s, f3 reference, float light_u,
                                             float ux, float uy, LightSample& out) {
    if (s.light_count == 0) {
        return false;
    }
    float     mass;
    const int index = select_light(s, light_u, mass);
    const DeviceLight& light = s.lights[index];
    if (light.kind == kLightDirectional) {
        out.direction   = light.normal;
        out.radiance    = light.radiance;
        out.distance    = INFINITY;
        out.probability = mass;
        out.discrete    = true;
        return true;
    }
    if (light.kind == kLightEnvironment) {
        float density;
        out.direction   = sample_environment(s, ux, uy, density, out.radiance);
        out.distance    = INFINITY;
        out.probability = mass * density;
        out.discrete    = false;
        return true;
    }
    const f3 bary  = sample_triangle(ux, uy);
    const f3 t0 = bary.x * light.v0, t1 = bary.y * light.v1, t2 = bary.z * light.v2;
    const f3 point = t0 + t1 + t2;
    if (!light.double_sided && dot(light.normal, reference - point) <= 0) {
        return false;
    }
    const float density = area_density(reference, point, light.normal, light.area);
    if (density == 0) {
        return false;
    }
    const f3    direction = point - reference;
    const float distance  = length(direction);
    out.direction         = direction / distance;
    out.radiance          = light.radiance;
    out.distance          = distance;
    out.probability       = mass * density;
    out.discrete          = false;
    out.position          = point;
    out.normal            = light.normal;
    out.position_error    = (fabs3(t0) + fabs3(t1) + fabs3(t2)) * (7.0f * kFltEps);
    return true;
}

// LightSampler::area_pdf (light.cpp:323-334).
__device__ __forceinline__ float area_pdf(const DeviceScene& s, f3 reference, uint32_t prim,
                                          f3 position) {
    const uint32_t choice = __ldg(s.prim_emitter + prim);
    if (choice == kNone) {
        return 0.0f;
    }
    const DeviceLight& light = s.lights[choice];
    if (!light.double_sided && dot(light.normal, reference - position) <= 0) {
        return 0.0f;
    }
    const float mass = __ldg(s.light_cdf + choice + 1) - __ldg(s.light_cdf + choice);
    return mass * area_density(reference, position, light.normal, light.area);
}

__device__ __forceinline__ float environment_pdf(const DeviceScene& s, f3 direction) {  // light.cpp:336-340
    if (s.environment_choice < 0) {
        return 0.0f;
    }
    const float mass = __ldg(s.light_cdf + s.environment_choice + 1) -
                       __ldg(s.light_cdf + s.environment_choice);
    return mass * environment_density(s, direction);
}

// The shadow segment of PathTracer::shadow_transmittance (path_tracer.cpp:126-151): both ends
// offset by their error bounds, the far end pulled in by one ulp and 2^-18 of its length. Returns false when the
// segment has zero length (the reference returns zero transmittance without tracing).
__device__ __forceinline__ bool shadow_segment(f3 origin, const LightSample& light, f3& direction,
                                               float& limit) {
    direction = light.direction;
    limit     = INFINITY;
    if (isfinite(light.distance)) {
        const f3 target     = offset_origin(light.position, light.normal, light.position_error,
                                            -light.direction);
        const f3 difference = target - origin;
        limit               = length(difference);
        if (limit == 0) {
            return false;
        }
        direction = difference / limit;
        // One ulp as in the reference, then 2^-18 of the length: the FP32 distance the triangle
        // test computes for the light's own triangle carries an error of a few ulps of the
        // segment length (not of the light point's coordinates, which set the offset above).
        limit = nextafterf(limit, 0.0f) * 0.99999618530273437500f;  // 1 - 2^-18
    }
    return true;
}

// ---- homogeneous media (src/render/medium.cpp) ----

__device__ __forceinline__ float phase_value(float cosine, float g) {  // medium.cpp:41-46
    const float a           = fabsf(g);
    const float denominator = (1 - a) * (1 - a) + 2 * a * (1 + copysignf(1.0f, g) * cosine);
    return ((1 - g) * (1 + g)) / (4 * kPi * denominator * sqrtf(denominator));
}

__device__ __forceinline__ float henyey_greenstein(f3 wo, f3 wi, float g) {
    return phase_value(fminf(fmaxf(dot(wo, wi), -1.0f), 1.0f), g);
}

__device__ __forceinline__ f3 sample_henyey_greenstein(f3 wo, float g, float ux, float uy,
                                                       float& probability) {  // medium.cpp:96-117
    float c;
    if (g >= 0) {
        const float denominator = (1 - g) + 2 * g * ux;
        c = 1 - 2 * (1 - g) * (1 - g) * (1 - ux) * (1 + g * ux) / (denominator * denominator);
    } else {
        const float denominator = (1 + g) - 2 * g * (1 - ux);
        c = -1 + 2 * (1 + g) * (1 + g) * ux * (1 - g * (1 - ux)) / (denominator * denominator);
    }
    c                = fminf(fmaxf(c, -1.0f), 1.0f);
    const float sine = sqrtf(fmaxf(0.0f, (1 - c) * (1 + c)));
    float       s, co;
    sincosf(2 * kPi * uy, &s, &co);
    Frame frame;
    frame.init(-wo);
    const f3 direction = normalize(frame.to_world(make(sine * co, sine * s, c)));
    probability        = henyey_greenstein(wo, direction, g);
    return direction;
}

__device__ __forceinline__ float optical_depth(float extinction, float distance) {
    return extinction == 0 ? 0.0f : extinction * distance;
}

__device__ __forceinline__ f3 medium_transmittance(const DeviceMedium& m, float distance) {
    return {expf(-optical_depth(m.extinction.x, distance)),
            expf(-optical_depth(m.extinction.y, distance)),
            expf(-optical_depth(m.extinction.z, distance))};
}

// mixture_weight (medium.cpp:53-86) in log space.
__device__ __forceinline__ f3 mixture_weight(const DeviceMedium& m, float distance, bool scattered,
                                             unsigned& error) {
    float ld[3], ln[3];
    for (int c = 0; c < 3; ++c) {
        const float e = comp(m.extinction, c);
        const float attenuation = -optical_depth(e, distance);
        if (!scattered) {
            ld[c] = ln[c] = attenuation;
        } else {
            ld[c] = e > 0 ? logf(e) + attenuation : -INFINITY;
            const float sc = comp(m.scattering, c);
            ln[c] = sc > 0 ? logf(sc) + attenuation : -INFINITY;
        }
    }
    const float largest = fmaxf(fmaxf(ld[0], ld[1]), ld[2]);
    if (!isfinite(largest)) {
        error |= kErrorMedium;
        return make(0, 0, 0);
    }
    const float sum = expf(ld[0] - largest) + expf(ld[1] - largest) + expf(ld[2] - largest);
    const float log_probability = largest + logf(sum / 3.0f);
    return {expf(ln[0] - log_probability), expf(ln[1] - log_probability),
            expf(ln[2] - log_probability)};
}

// Ray-box segment of MediumField::segments (medium.cpp:150-189) for one region.
__device__ __forceinline__ bool medium_segment(const DeviceMedium& m, f3 o, f3 d, float tmin,
                                               float tmax, float& enter, float& leave) {
    enter = tmin;
    leave = tmax;
    for (int a = 0; a < 3; ++a) {
        const float da = comp(d, a), oa = comp(o, a);
        const float lo = comp(m.minimum, a), hi = comp(m.maximum, a);
        if (da == 0) {
            if (oa <= lo || oa >= hi) {
                return false;
            }
            continue;
        }
        float nn = (lo - oa) / da, ff = (hi - oa) / da;
        if (nn > ff) {
            const float t = nn;
            nn            = ff;
            ff            = t;
        }
        enter = fmaxf(enter, nn);
        leave = fminf(leave, ff);
    }
    return leave > enter;
}

// MediumField::transmittance (medium.cpp:191-201).
__device__ __forceinline__ f3 field_transmittance(const DeviceScene& s, f3 o, f3 d, float tmin,
                                                  float tmax) {
    f3 result = make(1, 1, 1);
    for (int i = 0; i < s.medium_count; ++i) {
        const DeviceMedium& m = s.media[i];
        float enter, leave;
        if (m.enabled && medium_segment(m, o, d, tmin, tmax, enter, leave)) {
            result *= medium_transmittance(m, leave - enter);
        }
    }
    return result;
}

// MediumField::sample (medium.cpp:203-229): segments visited in entry order; consumes two
// samples per scattering segment only.
__device__ __forceinline__ f3 field_sample(const DeviceScene& s, f3 o, f3 d, float tmin, float tmax,
                                           Pcg32& rng, bool& scattered, float& scatter_t,
                                           float& anisotropy, unsigned& error) {
    f3 weight = make(1, 1, 1);
    scattered = false;
    float enter[kMaxMedia], leave[kMaxMedia];
    int   order[kMaxMedia];
    int   n = 0;
    for (int i = 0; i < s.medium_count; ++i) {
        const DeviceMedium& m = s.media[i];
        float e, l;
        if (m.enabled && medium_segment(m, o, d, tmin, tmax, e, l)) {
            int k = n++;
            while (k > 0 && enter[k - 1] > e) {  // stable insertion by entry distance
                enter[k] = enter[k - 1];
                leave[k] = leave[k - 1];
                order[k] = order[k - 1];
                --k;
            }
            enter[k] = e;
            leave[k] = l;
            order[k] = i;
        }
    }
    for (int k = 0; k < n; ++k) {
        const DeviceMedium& m      = s.media[order[k]];
        const float         length = leave[k] - enter[k];
        if (!m.scatters) {
            weight *= medium_transmittance(m, length);
            continue;
        }
        const float channel_u  = rng.next_1d();
        const float distance_u = rng.next_1d();
        const int   channel    = min(static_cast<int>(channel_u * 3.0f), 2);
        const float e          = comp(m.extinction, channel);
        const float distance   = e == 0 ? INFINITY : -log1pf(-distance_u) / e;
        const bool  hit        = distance < length;
        const float actual     = hit ? distance : length;
        weight *= mixture_weight(m, actual, hit, error);
        if (hit) {
            scattered  = true;
            scatter_t  = enter[k] + actual;
            anisotropy = m.anisotropy;
            break;
        }
    }
    return weight;
}

}  // namespace mr
