// wavefront.cu — wavefront path tracing on the GPU.
//
// One wave = up to `capacity` camera paths, their state in one 128-byte record per path. Each
// bounce runs two persistent kernels:
//   trace   nearest-hit traversal of the bounce's ray queue, classifying every path into a
//           material bin (miss, diffuse, conductor, mirror, dielectric, medium) with
//           warp-aggregated appends (match_any + popc + one atomic per key per warp), then
//           any-hit traversal of the previous bounce's shadow queue, adding the unoccluded
//           contributions;
//   shade   emission with MIS, next-event estimation, BSDF sampling and Russian roulette,
//           processed bin by bin so warps execute one material's code; appends the shadow
//           queue and the next bounce's ray queue.
// In large waves of non-trivial scenes both queues are then sorted by where each ray starts and
// its direction octant (a counting sort: keys counted in the shading launch, a scan, a scatter),
// so that neighbouring lanes of the next traversal walk the same nodes.
// The per-path logic is PathTracer::trace (src/render/path_tracer.cpp:153-366) in FP32 with the
// reference's RNG stream layout; every path writes only its own state, so images do not depend
// on scheduling. Radiance is kept per path and added to the pixels in sample order after the
// wave (compensated FP32 sums), so a frame is deterministic.
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>

#include "errors.hpp"
#include "shading.cuh"
#include "wavefront.cuh"

namespace mr {

namespace {

struct KernelArgs {
    DeviceScene      scene;
    PathState        st;
    Queues           q;
    IntegratorParams p;
    uint32_t         capacity;
    uint32_t         bounce;
    uint8_t*         occluded_out;  // diagnostics: per-path occlusion of this bounce's shadow ray
    const WaveDesc*  wave;          // multi-job waves: segments (scene, settings, buffers per job)
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// Appends `value` to queue[key] (key == kNone: nothing) with one atomic per distinct key per
// warp and returns its position in that queue (kNone when nothing was appended). Must be called
// by all 32 lanes.
__device__ __forceinline__ uint32_t warp_append(uint32_t key, uint32_t value, uint32_t* counts,
                                                uint32_t* queues, size_t stride) {
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key == kNone) {
        return kNone;
    }
    const int lane   = lane_id();
    const int leader = __ffs(peers) - 1;
    uint32_t  base   = 0;
    if (lane == leader) {
        base = atomicAdd(counts + key, static_cast<uint32_t>(__popc(peers)));
    }
    base               = __shfl_sync(peers, base, leader);
    const uint32_t pos = base + __popc(peers & ((1u << lane) - 1u));
    queues[key * stride + pos] = value;
    return pos;
}

__device__ __forceinline__ void warp_add_stat(unsigned long long* stat, uint32_t value) {
    const uint32_t total = __reduce_add_sync(0xffffffffu, value);
    if (lane_id() == 0 && total) {
        atomicAdd(stat, static_cast<unsigned long long>(total));
    }
}

__device__ __forceinline__ Pcg32 load_rng(const PathState& st, uint32_t path) {
    const ulonglong2 r = st.rng[path];
    return {r.x, r.y};
}

__device__ __forceinline__ void store_rng(const PathState& st, uint32_t path, const Pcg32& r) {
    st.rng[path] = make_ulonglong2(r.state, r.increment);
}

// The scene and integrator settings of a path: the launch's own in a single-job wave, its
// segment's in a multi-job wave.
template <bool BATCH>
__device__ __forceinline__ const WaveSegment* segment_of(const KernelArgs& a, uint32_t path) {
    return BATCH ? a.wave->seg + a.st.segment[path] : nullptr;
}

template <bool BATCH>
__device__ __forceinline__ const DeviceScene& scene_of(const KernelArgs& a, const WaveSegment* g) {
    if constexpr (BATCH) {
        return g->scene;
    } else {
        return a.scene;
    }
}

template <bool BATCH>
__device__ __forceinline__ const IntegratorParams& params_of(const KernelArgs& a, const WaveSegment* g) {
    if constexpr (BATCH) {
        return g->p;
    } else {
        return a.p;
    }
}

// Records a path's error in the wave's word and, in a multi-job wave, in its job's word.
template <bool BATCH>
__device__ __forceinline__ void note_error(const WaveSegment* g, unsigned e, unsigned& error) {
    if (e) {
        if constexpr (BATCH) {
            atomicOr(g->error, e);
        }
        error |= e;
    }
}

__device__ __forceinline__ void init_path(const KernelArgs& a, uint32_t slot, Pcg32 rng, f3 o, f3 d,
                                          float tmin, float tmax) {
    a.st.rng[slot]      = make_ulonglong2(rng.state, rng.increment);
    a.st.ray_o[slot]    = f4(o, tmin);
    a.st.ray_d[slot]    = f4(d, tmax);
    a.st.beta[slot]     = make_float4(1, 1, 1, 1);
    a.st.radiance[slot] = make_float4(0, 0, 0, 0);
    a.st.prev[slot]     = make_float4(0, 0, 0, 0);
    a.st.flags[slot]    = 1u;  // previous_delta = true
    a.q.ext[0][slot]    = slot;
}

// Stream derivation, film jitter and lens sample of one camera sample (PathTracer::sample_pixel,
// src/render/path_tracer.cpp:368-386).
__device__ __forceinline__ CameraRay camera_sample(const CameraBasis& camera, uint32_t x, uint32_t y,
                                                   uint64_t sample, uint32_t width, uint32_t height,
                                                   uint64_t seed, Pcg32& rng) {
    rng               = Pcg32::for_sample(seed, static_cast<uint64_t>(y) * width + x, sample);
    const float fx    = rng.next_1d();
    const float fy    = rng.next_1d();
    const float lx    = rng.next_1d();
    const float ly    = rng.next_1d();
    const float u     = (static_cast<float>(x) + fx) / static_cast<float>(width);
    const float v     = (static_cast<float>(y) + fy) / static_cast<float>(height);
    const float aspect = static_cast<float>(width) / static_cast<float>(height);
    return camera_ray(camera, u, v, aspect, lx, ly);
}

// Camera paths of a pixel rectangle x sample range, or of a pixel/sample list.
__global__ void init_camera_kernel(KernelArgs a, WaveInit w) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = w.count;
    if (i >= n) {
        return;
    }
    uint32_t x, y;
    uint64_t sample;
    if (w.kind == kInitCamera) {
        const uint32_t area = w.w * w.h;
        const uint32_t s    = i / area;
        const uint32_t r    = i - s * area;
        const uint32_t ry   = r / w.w;
        x                   = w.x0 + (r - ry * w.w);
        y                   = w.y0 + ry;
        sample              = w.s0 + s;
    } else {
        x      = w.pixels[2 * i];
        y      = w.pixels[2 * i + 1];
        sample = w.samples[i];
    }
    Pcg32           rng;
    const CameraRay r = camera_sample(a.scene.camera, x, y, sample, w.width, w.height, w.seed, rng);
    init_path(a, i, rng, r.origin, r.direction, r.minimum, r.maximum);
    if (w.camera_rays_out) {
        w.camera_rays_out[2 * i]     = f4(r.origin, r.minimum);
        w.camera_rays_out[2 * i + 1] = f4(r.direction, r.maximum);
    }
    if (i == 0) {
        a.q.counters[0].ext = n;
    }
    if (lane_id() == 0) {
        atomicAdd(a.q.stats + kStatPaths,
                  static_cast<unsigned long long>(min(32u, n - (i & ~31u))));
    }
}

// Segment k of a multi-job wave holding index i: the largest k < segments with first[k] <= i.
__device__ __forceinline__ uint32_t find_segment(const uint32_t* first, uint32_t segments, uint32_t i) {
    uint32_t lo = 0, hi = segments - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(first + mid) <= i) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

// Camera paths of every segment of a multi-job wave (grid-stride, so one grid size serves any
// wave and the launch can be replayed from a graph).
__global__ void __launch_bounds__(256) init_batch_kernel(KernelArgs a) {
    const WaveDesc* w        = a.wave;
    const uint32_t  n        = w->count;
    const uint32_t  segments = w->segments;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t     k     = find_segment(w->first_path, segments, i);
        const WaveSegment& g     = w->seg[k];
        const uint32_t     local = i - g.first_path;
        const uint32_t     area  = g.w * g.h;
        const uint32_t     s     = local / area;
        const uint32_t     r     = local - s * area;
        const uint32_t     ry    = r / g.w;
        Pcg32              rng;
        const CameraRay    ray = camera_sample(g.scene.camera, g.x0 + (r - ry * g.w), g.y0 + ry,
                                               g.s0 + s, g.width, g.height, g.seed, rng);
        init_path(a, i, rng, ray.origin, ray.direction, ray.minimum, ray.maximum);
        a.st.segment[i] = k;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.q.counters[0].ext = n;
        atomicAdd(a.q.stats + kStatPaths, static_cast<unsigned long long>(n));
    }
}

// Paths with caller rays and stream keys (PathTracer::trace).
__global__ void init_rays_kernel(KernelArgs a, WaveInit w) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.count) {
        return;
    }
    const Pcg32  rng = Pcg32::for_sample(w.keys[3 * i], w.keys[3 * i + 1], w.keys[3 * i + 2]);
    const float4 o   = w.rays[2 * i];
    const float4 d   = w.rays[2 * i + 1];
    init_path(a, i, rng, xyz(o), xyz(d), o.w, d.w);
    if (i == 0) {
        a.q.counters[0].ext = w.count;
    }
    if (lane_id() == 0) {
        atomicAdd(a.q.stats + kStatPaths,
                  static_cast<unsigned long long>(min(32u, w.count - (i & ~31u))));
    }
}

// ---- trace: this bounce's nearest-hit queue + the previous bounce's shadow queue ----

// Nearest hit of one extension ray, its material bin (or kNone) and, with media, the
// free-flight sample over the hit interval.
// Nearest hit or occlusion in `s`: the flattened traversal, or (TWO) the two-level one when the
// scene has two levels.
template <bool ANY_HIT, bool TWO>
__device__ __forceinline__ TraceResult trace_scene(const DeviceScene& s, const RayQuery& q, float tmin,
                                                   float tmax, TraceCounters& tc, unsigned& error) {
    if constexpr (TWO) {
        if (s.two_level) {
            return trace2<ANY_HIT>(s, q, tmin, tmax, tc, error);
        }
    }
    return trace<ANY_HIT>(s, q, tmin, tmax, tc, error);
}

template <bool MEDIA, bool TWO>
__device__ __forceinline__ uint32_t extend_item(const KernelArgs& a, const DeviceScene& s, uint32_t path,
                                                bool sorted, TraceCounters& tc, unsigned& error) {
    const float4 o4 = a.st.ray_o[path];
    const float4 d4 = a.st.ray_d[path];
    RayQuery     q;
    q.init(xyz(o4), xyz(d4));
    const TraceResult r    = trace_scene<false, TWO>(s, q, o4.w, d4.w, tc, error);
    uint32_t          kind = 0;
    if (r.slot != kNone) {
        a.st.hit[path] = make_float4(r.t, __fdiv_rn(r.a, r.det), __fdiv_rn(r.b, r.det),
                                     __fdiv_rn(r.c, r.det));
        if (sorted) {
            if (TWO && s.two_level) {
                kind = (r.flags >> 8) & 0xffu;
            } else {
                kind = (__float_as_uint(__ldg(s.tris + 3 * static_cast<size_t>(r.slot) + 1).w) >> 8) & 0xffu;
            }
        }
    }
    a.st.hit_slot[path] = r.slot;
    // Surface bins only group paths by material for the shading launch; unsorted, every
    // surface hit goes to the first.
    uint32_t key        = r.slot == kNone ? kBinMiss : kBinDiffuse + kind;
    if (MEDIA && s.medium_count > 0) {
        // MediumField::sample over [minimum, hit ? distance : maximum]
        // (src/render/path_tracer.cpp:170-177).
        Pcg32  rng   = load_rng(a.st, path);
        float4 beta4 = a.st.beta[path];
        bool   scattered;
        float  scatter_t = 0, g = 0;
        const f3 w = field_sample(s, xyz(o4), xyz(d4), o4.w, r.slot != kNone ? r.t : d4.w, rng,
                                  scattered, scatter_t, g, error);
        f3 beta = xyz(beta4) * w;
        store_rng(a.st, path, rng);
        a.st.beta[path] = f4(beta, beta4.w);
        if (!finite3(beta) || beta.x < 0 || beta.y < 0 || beta.z < 0) {
            error |= kErrorRadiance;
            key = kNone;
        } else if (max3(beta) == 0) {
            key = kNone;
        } else if (scattered) {
            a.st.hit[path] = make_float4(scatter_t, g, 0, 0);
            key            = kBinMedium;
        }
    }
    return key;
}

// Any hit of one shadow segment; adds the contribution (times the media transmittance) when
// the segment is clear.
template <bool MEDIA, bool TWO>
__device__ __forceinline__ void shadow_item(const KernelArgs& a, const DeviceScene& s, uint32_t path,
                                            TraceCounters& tc, unsigned& error) {
    const float4 o4 = a.st.shadow_o[path];
    const float4 d4 = a.st.shadow_d[path];
    RayQuery     q;
    q.init(xyz(o4), xyz(d4));
    const TraceResult r = trace_scene<true, TWO>(s, q, 0.0f, o4.w, tc, error);
    if (a.occluded_out) {
        a.occluded_out[path] = r.slot != kNone ? 1 : 0;
    }
    if (r.slot == kNone) {
        f3 c = xyz(a.st.shadow_c[path]);
        if (MEDIA && s.medium_count > 0) {
            c = c * field_transmittance(s, xyz(o4), xyz(d4), 0.0f, o4.w);
        }
        const float4 L      = a.st.radiance[path];
        a.st.radiance[path] = make_float4(L.x + c.x, L.y + c.y, L.z + c.z, 0);
    }
}

// One persistent launch per bounce traverses both queues: the bounce's extension rays first,
// then the shadow segments the previous bounce's shading queued (their contributions land
// before this bounce's shading adds emission, the reference's accumulation order). Warps fetch
// 32 consecutive items, so only the warp at the boundary mixes the two kinds. 8 resident blocks
// per SM (<= 64 registers): the traversal is latency bound and more warps hide it. In a
// multi-job wave (BATCH) every path finds its scene through its segment. With two-level scenes
// in the launch (TWO) the kernel also carries the two-level traversal and runs 5 blocks per SM
// (<= 102 registers) so that its larger state stays in registers.
template <bool MEDIA, bool BATCH, bool TWO>
__global__ void __launch_bounds__(128, TWO ? 5 : 8) trace_kernel(KernelArgs a) {
    BounceCounters* ctr      = a.q.counters + a.bounce;
    const uint32_t  n_ext    = ctr->ext;
    const uint32_t  n_shadow = a.bounce > 0 ? a.q.counters[a.bounce - 1].shadow : 0;
    const uint32_t  total    = n_ext + n_shadow;
    const bool      sorted   = !BATCH || n_ext >= a.wave->sort_threshold;
    const uint32_t* in       = a.q.ext[a.bounce & 1];
    TraceCounters   tc_ext{0, 0}, tc_shadow{0, 0};
    unsigned        error = 0;
    const int       lane  = lane_id();
    while (true) {
        uint32_t base = 0;
        if (lane == 0) {
            base = atomicAdd(&ctr->work_extend, 32u);
        }
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) {
            break;
        }
        const uint32_t i    = base + lane;
        uint32_t       key  = kNone;
        uint32_t       path = 0;
        if (i < total) {
            path                 = i < n_ext ? in[i] : a.q.shadow[i - n_ext];
            const WaveSegment* g = segment_of<BATCH>(a, path);
            unsigned           e = 0;
            if (i < n_ext) {
                key = extend_item<MEDIA, TWO>(a, scene_of<BATCH>(a, g), path, sorted, tc_ext, e);
            } else {
                shadow_item<MEDIA, TWO>(a, scene_of<BATCH>(a, g), path, tc_shadow, e);
            }
            note_error<BATCH>(g, e, error);
        }
        if (base < n_ext) {
            warp_append(key, path, ctr->bins, a.q.bins, a.capacity);
        }
    }
    warp_add_stat(a.q.stats + kStatExtendBounds, tc_ext.bounds);
    warp_add_stat(a.q.stats + kStatExtendTriangles, tc_ext.triangles);
    warp_add_stat(a.q.stats + kStatShadowBounds, tc_shadow.bounds);
    warp_add_stat(a.q.stats + kStatShadowTriangles, tc_shadow.triangles);
    if (error) {
        atomicOr(a.q.error, error);
    }
}

// ---- shade ----

struct ShadeResult {
    bool     continue_path;
    bool     shadow;
    uint32_t sort_key;         // coherence key of the continuing ray
    uint32_t shadow_sort_key;  // and of the shadow ray
};

// Coherence key of a ray: where it starts, then its direction octant. A ray leaving a surface
// (`slot` its triangle's slot) takes the slot's range in leaf order; a ray leaving a medium vertex
// (`slot` kNone) the Morton code of its origin's cell in the scene's bounds (kSortAxisBits per
// axis). Rays with equal keys start near one another heading the same way, so they visit much of
// the same tree.
__device__ __forceinline__ uint32_t coherence_key(const DeviceScene& s, uint32_t slot, f3 origin,
                                                  f3 direction) {
    uint32_t cell = 0;
    if (slot != kNone && s.slot_count > 0) {
        cell = static_cast<uint32_t>((static_cast<uint64_t>(slot) * kSortCells) / s.slot_count);
        cell = min(cell, kSortCells - 1);
    } else {
        constexpr float cells = static_cast<float>(1u << kSortAxisBits);
        for (int k = 0; k < 3; ++k) {
            const float extent = s.root_hi[k] - s.root_lo[k];
            const float u      = extent > 0 ? (comp(origin, k) - s.root_lo[k]) * (cells / extent) : 0.0f;
            const uint32_t c   = static_cast<uint32_t>(fminf(fmaxf(u, 0.0f), cells - 1.0f));
            for (int bit = 0; bit < kSortAxisBits; ++bit) {
                cell |= ((c >> bit) & 1u) << (3 * bit + k);
            }
        }
    }
    const uint32_t octant = (direction.x < 0 ? 1u : 0u) | (direction.y < 0 ? 2u : 0u) |
                            (direction.z < 0 ? 4u : 0u);
    return cell << 3 | octant;
}

__device__ __forceinline__ float emission_weight(const IntegratorParams& p, uint32_t depth,
                                                 bool previous_delta, float previous_pdf,
                                                 float light_pdf) {
    if (depth == 0 || previous_delta || p.mode == MR_SAMPLING_BSDF) {
        return 1.0f;
    }
    return p.mode == MR_SAMPLING_MIS ? power_heuristic(previous_pdf, light_pdf) : 0.0f;
}

// Russian roulette (src/render/path_tracer.cpp:352-362). Returns false when the path ends.
__device__ __forceinline__ bool roulette(const IntegratorParams& p, uint32_t depth, Pcg32& rng,
                                         f3& beta, float eta_scale, uint32_t& rr_count) {
    const float u = rng.next_1d();
    if (p.russian_roulette && depth + 1 >= p.roulette_depth) {
        const float survival = fminf(fmaxf(max3(beta * eta_scale), 0.05f), 0.95f);
        if (u >= survival) {
            ++rr_count;
            return false;
        }
        beta = beta * (1.0f / survival);
    }
    return true;
}

struct ShadeStats {
    uint32_t shadow_rays = 0, scattering = 0, roulette = 0, medium = 0;
};

template <bool BATCH, bool TWO>
__device__ ShadeResult shade_surface(const KernelArgs& a, uint32_t path, int bin, ShadeStats& stats,
                                     unsigned& error) {
    const WaveSegment*      g     = segment_of<BATCH>(a, path);
    const DeviceScene&      s     = scene_of<BATCH>(a, g);
    const IntegratorParams& p     = params_of<BATCH>(a, g);
    const uint32_t          depth = a.bounce;
    const float4            d4    = a.st.ray_d[path];
    const f3                dir   = xyz(d4);
    const float4            beta4 = a.st.beta[path];
    f3                      beta  = xyz(beta4);
    float                   eta_scale = beta4.w;
    const float4            prev4 = a.st.prev[path];
    const bool              previous_delta = a.st.flags[path] & 1u;
    float4                  L4    = a.st.radiance[path];
    f3                      L     = xyz(L4);
    ShadeResult             out{false, false, 0u, 0u};

    if (bin == kBinMiss) {
        L += beta * environment_radiance(s, dir) *
             emission_weight(p, depth, previous_delta, prev4.w, environment_pdf(s, dir));
        a.st.radiance[path] = f4(L, 0);
        return out;
    }
    Pcg32 rng = load_rng(a.st, path);
    if (bin == kBinMedium) {
        // Medium vertex (src/render/path_tracer.cpp:178-223).
        const float4 h      = a.st.hit[path];
        const float4 o4     = a.st.ray_o[path];
        const f3     vertex = xyz(o4) + h.x * dir;
        const float  g      = h.y;
        if (depth == p.maximum_depth) {
            return out;
        }
        const f3    wo      = -dir;
        const float light_u = rng.next_1d();
        const float lsx     = rng.next_1d();
        const float lsy     = rng.next_1d();
        const float phx     = rng.next_1d();
        const float phy     = rng.next_1d();
        LightSample ls;
        if (sample_light(s, vertex, light_u, lsx, lsy, ls) &&
            (p.mode != MR_SAMPLING_BSDF || ls.discrete)) {
            const float phase = henyey_greenstein(wo, ls.direction, g);
            ++stats.shadow_rays;
            f3    sd;
            float limit;
            if (shadow_segment(vertex, ls, sd, limit)) {
                float weight = 1.0f;
                if (p.mode == MR_SAMPLING_MIS && !ls.discrete) {
                    weight = power_heuristic(ls.probability, phase);
                }
                a.st.shadow_o[path] = f4(vertex, limit);
                a.st.shadow_d[path] = f4(sd, 0);
                a.st.shadow_c[path] = f4(beta * ls.radiance * (phase * weight / ls.probability), 0);
                out.shadow          = true;
                out.shadow_sort_key = a.q.staging ? coherence_key(s, kNone, vertex, sd) : 0u;
            }
        }
        float     pdf;
        const f3  next = sample_henyey_greenstein(wo, g, phx, phy, pdf);
        ++stats.scattering;
        ++stats.medium;
        if (!roulette(p, depth, rng, beta, eta_scale, stats.roulette)) {
            store_rng(a.st, path, rng);
            return out;
        }
        a.st.prev[path]  = f4(vertex, pdf);
        a.st.flags[path] = 0u;
        a.st.ray_o[path] = f4(vertex, 0.0f);
        a.st.ray_d[path] = f4(next, INFINITY);
        a.st.beta[path]  = f4(beta, eta_scale);
        store_rng(a.st, path, rng);
        out.continue_path = true;
        out.sort_key      = a.q.staging ? coherence_key(s, kNone, vertex, next) : 0u;
        return out;
    }

    // Surface vertex (src/render/path_tracer.cpp:224-363).
    const float4     h   = a.st.hit[path];
    const uint32_t   slot = a.st.hit_slot[path];
    const SurfaceHit sh  = surface_hit<TWO>(s, dir, slot, h.y, h.z, h.w);
    const DeviceMaterial m = s.materials[sh.material];
    if (m.emission.x > 0 || m.emission.y > 0 || m.emission.z > 0) {
        L += beta * m.emission *
             emission_weight(p, depth, previous_delta, prev4.w,
                             area_pdf(s, xyz(prev4), sh.prim, sh.position));
        a.st.radiance[path] = f4(L, 0);
    }
    if (depth == p.maximum_depth) {
        return out;
    }
    const f3 wo_world = -dir;
    f3       normal   = m.kind == MR_MATERIAL_DIELECTRIC ? sh.geometric_normal : sh.shading_normal;
    if (dot(normal, wo_world) < 0) {
        normal = -normal;
    }
    Frame frame;
    frame.init(normal);
    const f3 wo = frame.to_local(wo_world);
    Bsdf     bsdf;
    bsdf.init(m, sh.front_face,
              m.base_texture >= 0 ? texture_sample(s, m.base_texture, sh.u, sh.v, m.filter)
                                  : make(1.0f, 1.0f, 1.0f));  // path_tracer.cpp:279-282
    const float light_u   = rng.next_1d();
    const float sux       = rng.next_1d();
    const float suy       = rng.next_1d();
    const float component = rng.next_1d();
    const float dux       = rng.next_1d();
    const float duy       = rng.next_1d();
    if (!bsdf.is_delta()) {
        LightSample ls;
        if (sample_light(s, sh.position, light_u, sux, suy, ls) &&
            (p.mode != MR_SAMPLING_BSDF || ls.discrete)) {
            const f3   wi = frame.to_local(ls.direction);
            const bool reflection_side =
                dot(wo_world, sh.geometric_normal) * dot(ls.direction, sh.geometric_normal) > 0;
            if (wi.z > 0 && reflection_side) {
                ++stats.shadow_rays;
                const f3 origin =
                    offset_origin(sh.position, sh.geometric_normal, sh.position_error, ls.direction);
                LightSample lsn = ls;
                lsn.direction   = normalize(ls.direction);
                f3    sd;
                float limit;
                if (shadow_segment(origin, lsn, sd, limit)) {
                    float weight = 1.0f;
                    if (p.mode == MR_SAMPLING_MIS && !ls.discrete) {
                        weight = power_heuristic(ls.probability, bsdf.pdf(wo, wi));
                    }
                    a.st.shadow_o[path] = f4(origin, limit);
                    a.st.shadow_d[path] = f4(sd, 0);
                    a.st.shadow_c[path] = f4(beta * bsdf.evaluate(wo, wi) * wi.z * ls.radiance *
                                                 (weight / ls.probability),
                                             0);
                    out.shadow = true;
                    out.shadow_sort_key = a.q.staging ? coherence_key(s, slot, origin, sd) : 0u;
                }
            }
        }
    }
    Bsdf::Sample sample;
    if (!bsdf.sample(wo, component, dux, duy, sample) || max3(sample.weight) == 0) {
        store_rng(a.st, path, rng);
        return out;
    }
    const f3    wi_world = normalize(frame.to_world(sample.direction));
    const float sides    = dot(wo_world, sh.geometric_normal) * dot(wi_world, sh.geometric_normal);
    if ((sample.transmission && sides >= 0) || (!sample.transmission && sides <= 0)) {
        store_rng(a.st, path, rng);
        return out;
    }
    beta = beta * sample.weight;
    if (!finite3(beta) || beta.x < 0 || beta.y < 0 || beta.z < 0) {
        error |= kErrorRadiance;
        return out;
    }
    eta_scale *= sample.eta * sample.eta;
    ++stats.scattering;
    const f3 origin = offset_origin(sh.position, sh.geometric_normal, sh.position_error, wi_world);
    const f3 next   = normalize(wi_world);
    if (!roulette(p, depth, rng, beta, eta_scale, stats.roulette)) {
        store_rng(a.st, path, rng);
        return out;
    }
    a.st.prev[path]  = f4(sh.position, sample.probability);
    a.st.flags[path] = sample.discrete ? 1u : 0u;
    a.st.ray_o[path] = f4(origin, 0.0f);
    a.st.ray_d[path] = f4(next, INFINITY);
    a.st.beta[path]  = f4(beta, eta_scale);
    store_rng(a.st, path, rng);
    out.continue_path = true;
    out.sort_key      = a.q.staging ? coherence_key(s, slot, origin, next) : 0u;
    return out;
}

template <bool BATCH, bool TWO>
__global__ void __launch_bounds__(128, 5) shade_kernel(KernelArgs a) {
    BounceCounters* ctr = a.q.counters + a.bounce;
    uint32_t        prefix[kBinCount + 1];
    prefix[0] = 0;
    for (int k = 0; k < kBinCount; ++k) {
        prefix[k + 1] = prefix[k] + ctr->bins[k];
    }
    const uint32_t total  = prefix[kBinCount];
    uint32_t*      next   = a.q.ext[(a.bounce + 1) & 1];
    BounceCounters* nctr  = a.q.counters + a.bounce + 1;
    ShadeStats     stats;
    unsigned       error  = 0;
    const uint32_t warps  = (gridDim.x * blockDim.x) >> 5;
    const uint32_t warp   = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (uint32_t base = warp * 32; base < total; base += warps * 32) {
        const uint32_t i      = base + lane_id();
        uint32_t       path   = 0;
        uint32_t       ext_key = kNone, shadow_key = kNone, sort_key = kNone, shadow_sort = kNone;
        if (i < total) {
            int bin = 0;
            while (i >= prefix[bin + 1]) {
                ++bin;
            }
            path                 = a.q.bins[bin * static_cast<size_t>(a.capacity) + (i - prefix[bin])];
            unsigned          e  = 0;
            const ShadeResult r  = shade_surface<BATCH, TWO>(a, path, bin, stats, e);
            note_error<BATCH>(segment_of<BATCH>(a, path), e, error);
            ext_key              = r.continue_path ? 0u : kNone;
            shadow_key           = r.shadow ? 0u : kNone;
            sort_key             = r.continue_path ? r.sort_key : kNone;
            shadow_sort          = r.shadow ? r.shadow_sort_key : kNone;
        }
        if (a.q.staging) {
            // Both queues are staged for the coherence sort: each entry's key beside it, one
            // count per distinct key per warp (shadow keys in the second half of the counts).
            const uint32_t pos = warp_append(shadow_key, path, &ctr->shadow, a.q.shadow_staging, 0);
            if (shadow_key != kNone) {
                a.q.shadow_keys[pos] = shadow_sort;
            }
            const unsigned same = __match_any_sync(0xffffffffu, shadow_sort);
            if (shadow_sort != kNone && lane_id() == __ffs(same) - 1) {
                atomicAdd(a.q.buckets + kSortBuckets + shadow_sort, static_cast<uint32_t>(__popc(same)));
            }
        } else {
            warp_append(shadow_key, path, &ctr->shadow, a.q.shadow, 0);
        }
        if (a.q.staging) {
            const uint32_t pos = warp_append(ext_key, path, &nctr->ext, a.q.staging, 0);
            if (ext_key != kNone) {
                a.q.keys[pos] = sort_key;
            }
            const unsigned same = __match_any_sync(0xffffffffu, sort_key);
            if (sort_key != kNone && lane_id() == __ffs(same) - 1) {
                atomicAdd(a.q.buckets + sort_key, static_cast<uint32_t>(__popc(same)));
            }
        } else {
            warp_append(ext_key, path, &nctr->ext, next, 0);
        }
    }
    warp_add_stat(a.q.stats + kStatShadowRays, stats.shadow_rays);
    warp_add_stat(a.q.stats + kStatScattering, stats.scattering);
    warp_add_stat(a.q.stats + kStatRoulette, stats.roulette);
    warp_add_stat(a.q.stats + kStatMedium, stats.medium);
    if (error) {
        atomicOr(a.q.error, error);
    }
}

// ---- coherence sort of the next bounce's extension rays ----

// Exclusive scan of the bucket counts into the cursors, in three launches over blocks of 1,024
// buckets (256 threads, 4 consecutive buckets each): block sums, a scan of the block sums, then
// each block's scan from its base. The extension keys fill the first half of the buckets and the
// shadow keys the second; each half's cursors start at 0. The counts are cleared for the next
// bounce.
constexpr uint32_t kSortScanBlock  = 1024;
constexpr uint32_t kSortScanBlocks = 2 * kSortBuckets / kSortScanBlock;

__device__ __forceinline__ uint32_t block_exclusive_scan_256(uint32_t v, uint32_t* warp_sums,
                                                             uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t       x    = v;
    for (uint32_t offset = 1; offset < 32; offset <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, offset);
        x += lane >= offset ? y : 0u;
    }
    if (lane == 31) {
        warp_sums[warp] = x;
    }
    __syncthreads();
    uint32_t before = 0;
    total           = 0;
    for (uint32_t w = 0; w < 8; ++w) {
        before += w < warp ? warp_sums[w] : 0u;
        total += warp_sums[w];
    }
    return before + x - v;
}

__global__ void __launch_bounds__(256) sort_block_sums_kernel(const uint32_t* buckets, uint32_t* sums) {
    const uint4 c = reinterpret_cast<const uint4*>(buckets + blockIdx.x * kSortScanBlock)[threadIdx.x];
    const uint32_t v = __reduce_add_sync(0xffffffffu, c.x + c.y + c.z + c.w);
    __shared__ uint32_t warp_sums[8];
    if ((threadIdx.x & 31) == 0) {
        warp_sums[threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) {
            t += warp_sums[w];
        }
        sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(256) sort_block_bases_kernel(uint32_t* sums) {
    static_assert(kSortScanBlocks == 256, "one thread per block of buckets");
    __shared__ uint32_t warp_sums[8];
    const uint32_t      v = sums[threadIdx.x];
    uint32_t            total;
    uint32_t            base = block_exclusive_scan_256(v, warp_sums, total);
    __syncthreads();
    // The shadow half (blocks 128-255) starts again at 0.
    __shared__ uint32_t extension_total;
    if (threadIdx.x == kSortScanBlocks / 2) {
        extension_total = base;
    }
    __syncthreads();
    if (threadIdx.x >= kSortScanBlocks / 2) {
        base -= extension_total;
    }
    sums[kSortScanBlocks + threadIdx.x] = base;
}

__global__ void __launch_bounds__(256) sort_cursors_kernel(uint32_t* buckets, const uint32_t* sums) {
    __shared__ uint32_t warp_sums[8];
    uint4*         counts = reinterpret_cast<uint4*>(buckets + blockIdx.x * kSortScanBlock);
    uint4*         cursors =
        reinterpret_cast<uint4*>(buckets + 2 * kSortBuckets + blockIdx.x * kSortScanBlock);
    const uint4    c = counts[threadIdx.x];
    uint32_t       total;
    const uint32_t start = sums[kSortScanBlocks + blockIdx.x] +
                           block_exclusive_scan_256(c.x + c.y + c.z + c.w, warp_sums, total);
    cursors[threadIdx.x] = make_uint4(start, start + c.x, start + c.x + c.y, start + c.x + c.y + c.z);
    counts[threadIdx.x]  = make_uint4(0, 0, 0, 0);
}

__host__ void enqueue_sort_scan(uint32_t* buckets, cudaStream_t stream) {
    uint32_t* sums = buckets + 4 * kSortBuckets;
    sort_block_sums_kernel<<<kSortScanBlocks, 256, 0, stream>>>(buckets, sums);
    sort_block_bases_kernel<<<1, 256, 0, stream>>>(sums);
    sort_cursors_kernel<<<kSortScanBlocks, 256, 0, stream>>>(buckets, sums);
}

// Moves the staged paths into the next bounce's extension queue and the staged shadow rays into
// the shadow queue, each in key order (within a key, in the order the warps claim their places:
// path results do not depend on queue order).
__global__ void sort_scatter_kernel(KernelArgs a) {
    const uint32_t n_ext    = a.q.counters[a.bounce + 1].ext;
    const uint32_t n_shadow = a.q.counters[a.bounce].shadow;
    const uint32_t n        = n_ext + n_shadow;
    uint32_t*      next     = a.q.ext[(a.bounce + 1) & 1];
    const uint32_t step     = gridDim.x * blockDim.x;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n; base += step) {
        const uint32_t i      = base + lane_id();
        const bool     shadow = i >= n_ext;
        uint32_t       key    = kNone;
        if (i < n) {
            key = shadow ? kSortBuckets + a.q.shadow_keys[i - n_ext] : a.q.keys[i];
        }
        const unsigned same = __match_any_sync(0xffffffffu, key);
        if (key != kNone) {
            const int leader = __ffs(same) - 1;
            uint32_t  pos    = 0;
            if (lane_id() == leader) {
                pos = atomicAdd(a.q.buckets + 2 * kSortBuckets + key, static_cast<uint32_t>(__popc(same)));
            }
            pos = __shfl_sync(same, pos, leader) + __popc(same & ((1u << lane_id()) - 1u));
            if (shadow) {
                a.q.shadow[pos] = a.q.shadow_staging[i - n_ext];
            } else {
                next[pos] = a.q.staging[i];
            }
        }
    }
}

// ---- pixel accumulation ----

__device__ __forceinline__ void neumaier(float& sum, float& comp, float v) {
    const float t = sum + v;
    comp += fabsf(sum) >= fabsf(v) ? (sum - t) + v : (v - t) + sum;
    sum = t;
}

// Adds the wave's per-path radiance to the pixels in sample order; checks every path result
// like check_radiance (src/render/path_tracer.cpp:22-26).
__global__ void resolve_kernel(PathField<float4> radiance, uint32_t x0, uint32_t y0, uint32_t w,
                               uint32_t h, uint32_t ns, uint32_t width, float4* accumulator,
                               uint32_t accumulator_row0, unsigned* error) {
    const uint32_t r    = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t area = w * h;
    if (r >= area) {
        return;
    }
    const uint32_t ry    = r / w;
    const size_t   pixel = static_cast<size_t>(y0 + ry - accumulator_row0) * width + x0 + (r - ry * w);
    float4         sum   = accumulator[2 * pixel];
    float4         comp  = accumulator[2 * pixel + 1];
    bool           bad   = false;
    for (uint32_t s = 0; s < ns; ++s) {
        const float4 v = radiance[static_cast<size_t>(s) * area + r];
        bad |= !(isfinite(v.x) && isfinite(v.y) && isfinite(v.z)) || v.x < 0 || v.y < 0 || v.z < 0;
        neumaier(sum.x, comp.x, v.x);
        neumaier(sum.y, comp.y, v.y);
        neumaier(sum.z, comp.z, v.z);
    }
    if (bad) {
        atomicOr(error, kErrorRadiance);
    }
    accumulator[2 * pixel]     = sum;
    accumulator[2 * pixel + 1] = comp;
}

// Multi-job resolve: every pixel of every segment adds its ns samples to its job's accumulator
// in sample order (continuing the job's earlier samples; a segment starting at sample 0 starts
// from zero), and a pixel whose last sample this is gets its mean written to the job's image with
// the overflow check. Same arithmetic as resolve_kernel + finalize_kernel, so a job's image does
// not depend on which wave carried which of its samples.
__global__ void __launch_bounds__(256) resolve_batch_kernel(PathField<float4> radiance, const WaveDesc* w,
                                                            unsigned* error) {
    const uint32_t n        = w->pixels;
    const uint32_t segments = w->segments;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t     k     = find_segment(w->first_pixel, segments, p);
        const WaveSegment& g     = w->seg[k];
        const uint32_t     r     = p - __ldg(w->first_pixel + k);
        const uint32_t     area  = g.w * g.h;
        const uint32_t     ry    = r / g.w;
        const size_t       pixel = static_cast<size_t>(g.y0 + ry) * g.width + g.x0 + (r - ry * g.w);
        float4 sum  = make_float4(0, 0, 0, 0);
        float4 comp = make_float4(0, 0, 0, 0);
        if (g.s0 > 0) {
            sum  = g.accumulator[2 * pixel];
            comp = g.accumulator[2 * pixel + 1];
        }
        bool bad = false;
        for (uint32_t s = 0; s < g.ns; ++s) {
            const float4 v = radiance[g.first_path + static_cast<size_t>(s) * area + r];
            bad |= !(isfinite(v.x) && isfinite(v.y) && isfinite(v.z)) || v.x < 0 || v.y < 0 || v.z < 0;
            neumaier(sum.x, comp.x, v.x);
            neumaier(sum.y, comp.y, v.y);
            neumaier(sum.z, comp.z, v.z);
        }
        unsigned e = bad ? kErrorRadiance : 0u;
        g.accumulator[2 * pixel]     = sum;
        g.accumulator[2 * pixel + 1] = comp;
        if (g.s0 + g.ns == g.spp) {
            const float count = static_cast<float>(g.spp);
            const float cr = (sum.x + comp.x) / count, cg = (sum.y + comp.y) / count,
                        cb = (sum.z + comp.z) / count;
            if (!(isfinite(cr) && isfinite(cg) && isfinite(cb))) {
                e |= kErrorOverflow;
            }
            g.rgb[3 * pixel]     = cr;
            g.rgb[3 * pixel + 1] = cg;
            g.rgb[3 * pixel + 2] = cb;
        }
        if (e) {
            atomicOr(g.error, e);
            atomicOr(error, e);
        }
    }
}

// Pixel mean and the overflow check of PathTracer::render (src/render/path_tracer.cpp:394-401).
__global__ void finalize_kernel(const float4* accumulator, size_t pixels, uint32_t spp, float* rgb,
                                unsigned* error) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= pixels) {
        return;
    }
    const float4 s = accumulator[2 * i];
    const float4 c = accumulator[2 * i + 1];
    const float  n = static_cast<float>(spp);
    const float  r = (s.x + c.x) / n, g = (s.y + c.y) / n, b = (s.z + c.z) / n;
    if (!(isfinite(r) && isfinite(g) && isfinite(b))) {
        atomicOr(error, kErrorOverflow);
    }
    rgb[3 * i]     = r;
    rgb[3 * i + 1] = g;
    rgb[3 * i + 2] = b;
}

// Diagnostics: copies the first-bounce shadow rays of the queued paths.
__global__ void capture_shadow_kernel(KernelArgs a, float4* rays, uint8_t* has_shadow) {
    const uint32_t count = a.q.counters[0].shadow;
    const uint32_t i     = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const uint32_t path = a.q.shadow[i];
        rays[2 * path]      = a.st.shadow_o[path];
        rays[2 * path + 1]  = a.st.shadow_d[path];
        has_shadow[path]    = 1;
    }
}

__global__ void copy_radiance_kernel(PathField<float4> radiance, uint32_t count, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const float4 v = radiance[i];
        out[3 * i]     = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    }
}

// ---- launch helpers ----

struct LaunchShape {
    int trace_blocks[4]  = {0, 0, 0, 0};  // by media + 2 * two_level
    int shade_blocks     = 0;
    int shade_blocks_two = 0;
};

LaunchShape& launch_shape() {
    static thread_local int         device = -1;
    static thread_local LaunchShape shape;
    int current = 0;
    cudaGetDevice(&current);
    if (device != current) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, current);
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, trace_kernel<false, false, false>, 128, 0);
        shape.trace_blocks[0] = sms * std::max(1, per);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, trace_kernel<true, false, false>, 128, 0);
        shape.trace_blocks[1] = sms * std::max(1, per);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, trace_kernel<false, false, true>, 128, 0);
        shape.trace_blocks[2] = sms * std::max(1, per);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, trace_kernel<true, false, true>, 128, 0);
        shape.trace_blocks[3] = sms * std::max(1, per);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, shade_kernel<false, false>, 128, 0);
        shape.shade_blocks = sms * std::max(1, per);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, shade_kernel<false, true>, 128, 0);
        shape.shade_blocks_two = sms * std::max(1, per);
        device = current;
    }
    return shape;
}

size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

KernelTiming& kernel_timing() {
    static KernelTiming timing;
    return timing;
}

Workspace::~Workspace() {
    if (memory) {
        cudaFree(memory);
    }
}

namespace {

std::shared_ptr<Workspace> allocate_workspace(size_t capacity, uint32_t max_bounces, size_t pixels) {
    auto   ws     = std::make_shared<Workspace>();
    size_t offset = 0;
    const auto field = [&](size_t bytes) {
        const size_t at = offset;
        offset += align_up(bytes);
        return at;
    };
    const size_t o_paths   = field(capacity * kPathRecordBytes);
    const size_t o_shadows = field(capacity * kShadowRecordBytes);
    const size_t o_e0 = field(capacity * sizeof(uint32_t));
    const size_t o_e1 = field(capacity * sizeof(uint32_t));
    const size_t o_bins = field(capacity * kBinCount * sizeof(uint32_t));
    const size_t o_shadow = field(capacity * sizeof(uint32_t));
    const size_t o_stage = field(capacity * sizeof(uint32_t));
    const size_t o_keys  = field(capacity * sizeof(uint32_t));
    const size_t o_sstage = field(capacity * sizeof(uint32_t));
    const size_t o_skeys  = field(capacity * sizeof(uint32_t));
    const size_t o_buck  = field((4 * kSortBuckets + 2 * kSortScanBlocks) * sizeof(uint32_t));
    const size_t o_ctr = field((max_bounces + 2) * sizeof(BounceCounters));
    const size_t o_stats = field(kStatCount * sizeof(unsigned long long));
    const size_t o_err = field(sizeof(unsigned));
    const size_t o_acc = field(2 * pixels * sizeof(float4));
    void*        mem   = nullptr;
    MR_CUDA(cudaMalloc(&mem, offset));
    char* base              = static_cast<char*>(mem);
    ws->memory              = mem;
    ws->bytes               = offset;
    ws->capacity            = capacity;
    ws->max_bounces         = max_bounces;
    ws->pixels              = pixels;
    ws->state.view(reinterpret_cast<unsigned char*>(base + o_paths),
                   reinterpret_cast<unsigned char*>(base + o_shadows), true);
    ws->queues.ext[0]       = reinterpret_cast<uint32_t*>(base + o_e0);
    ws->queues.ext[1]       = reinterpret_cast<uint32_t*>(base + o_e1);
    ws->queues.bins         = reinterpret_cast<uint32_t*>(base + o_bins);
    ws->queues.shadow       = reinterpret_cast<uint32_t*>(base + o_shadow);
    ws->queues.staging      = reinterpret_cast<uint32_t*>(base + o_stage);
    ws->queues.keys         = reinterpret_cast<uint32_t*>(base + o_keys);
    ws->queues.shadow_staging = reinterpret_cast<uint32_t*>(base + o_sstage);
    ws->queues.shadow_keys    = reinterpret_cast<uint32_t*>(base + o_skeys);
    ws->queues.buckets      = reinterpret_cast<uint32_t*>(base + o_buck);
    MR_CUDA(cudaMemset(ws->queues.buckets, 0, 2 * kSortBuckets * sizeof(uint32_t)));
    ws->queues.counters     = reinterpret_cast<BounceCounters*>(base + o_ctr);
    ws->queues.stats        = reinterpret_cast<unsigned long long*>(base + o_stats);
    ws->queues.error        = reinterpret_cast<unsigned*>(base + o_err);
    ws->accumulator         = reinterpret_cast<float4*>(base + o_acc);
    return ws;
}

std::mutex                              pool_mutex;
std::vector<std::shared_ptr<Workspace>> pool;

}  // namespace

// Workspaces are pooled per process: a request takes the smallest pooled workspace of its device
// that is large enough in every dimension, and requests are rounded up (powers of two, bounces to
// a multiple of 16) so that one workspace serves many job shapes. When more than four are pooled
// the smallest goes: large ones serve every smaller request, so a stream of uneven jobs settles
// on reuse instead of reallocating (a device-wide synchronising cudaFree each time).
std::shared_ptr<Workspace> acquire_workspace(size_t capacity, uint32_t max_bounces, size_t pixels) {
    int device = 0;
    MR_CUDA(cudaGetDevice(&device));
    const auto round_up = [](size_t v, size_t floor) {
        size_t r = floor;
        while (r < v) {
            r <<= 1;
        }
        return r;
    };
    capacity    = round_up(capacity, size_t(1) << 16);
    pixels      = pixels ? round_up(pixels, size_t(1) << 16) : 0;
    max_bounces = (max_bounces + 15u) & ~15u;
    {
        std::lock_guard<std::mutex> lock(pool_mutex);
        long best = -1;
        for (size_t i = 0; i < pool.size(); ++i) {
            const auto& w = pool[i];
            if (w->device == device && w->capacity >= capacity && w->max_bounces >= max_bounces &&
                w->pixels >= pixels && (best < 0 || w->bytes < pool[best]->bytes)) {
                best = static_cast<long>(i);
            }
        }
        if (best >= 0) {
            auto out = pool[best];
            pool.erase(pool.begin() + best);
            return out;
        }
    }
    auto ws    = allocate_workspace(capacity, max_bounces, pixels);
    ws->device = device;
    return ws;
}

void release_workspace(std::shared_ptr<Workspace> ws) {
    if (!ws) {
        return;
    }
    std::lock_guard<std::mutex> lock(pool_mutex);
    pool.push_back(std::move(ws));
    if (pool.size() > 4) {
        auto smallest = std::min_element(pool.begin(), pool.end(), [](const auto& a, const auto& b) {
            return a->bytes < b->bytes;
        });
        pool.erase(smallest);
    }
}

void reset_statistics(Workspace& ws, cudaStream_t stream) {
    MR_CUDA(cudaMemsetAsync(ws.queues.stats, 0, kStatCount * sizeof(unsigned long long), stream));
    MR_CUDA(cudaMemsetAsync(ws.queues.error, 0, sizeof(unsigned), stream));
}

void read_statistics(Workspace& ws, cudaStream_t stream, mr_path_statistics* out, unsigned* error) {
    unsigned long long stats[kStatCount];
    unsigned           e = 0;
    MR_CUDA(cudaMemcpyAsync(stats, ws.queues.stats, sizeof(stats), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaMemcpyAsync(&e, ws.queues.error, sizeof(e), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->paths                    = stats[kStatPaths];
        out->shadow_rays              = stats[kStatShadowRays];
        out->scattering_events        = stats[kStatScattering];
        out->roulette_terminations    = stats[kStatRoulette];
        out->medium_scattering_events = stats[kStatMedium];
        out->geometry.bounds_tests    = stats[kStatExtendBounds] + stats[kStatShadowBounds];
        out->geometry.triangle_tests  = stats[kStatExtendTriangles] + stats[kStatShadowTriangles];
    }
    if (error) {
        *error = e;
    }
}

mr_status error_status(unsigned error, std::string& message) {
    if (error & kErrorOverflow) {
        message = "Rendered radiance exceeds the float image range";
        return MR_OVERFLOW;
    }
    if (error & kErrorRadiance) {
        message = "Path contribution is nonfinite or negative";
        return MR_RUNTIME_ERROR;
    }
    if (error & kErrorMedium) {
        message = "Medium sample has zero mixture probability";
        return MR_RUNTIME_ERROR;
    }
    if (error & kErrorRay) {
        message = "A ray with a nonfinite origin or direction reached traversal";
        return MR_RUNTIME_ERROR;
    }
    if (error & kErrorVisits) {
        message = "BVH traversal exceeded its node-visit bound";
        return MR_RUNTIME_ERROR;
    }
    if (error & kErrorStack) {
        message = "BVH traversal stack exhausted";
        return MR_RUNTIME_ERROR;
    }
    return MR_OK;
}

void Engine::run_wave(const Scene& scene, const IntegratorParams& params, const WaveInit& init,
                      Workspace& ws, cudaStream_t stream) {
    if (init.count == 0) {
        return;
    }
    if (init.count > ws.capacity || params.maximum_depth + 1 > ws.max_bounces) {
        fail(MR_LENGTH_ERROR, "Wave exceeds the workspace capacity");
    }
    KernelArgs a;
    a.scene    = scene.d;
    a.st       = ws.state;
    a.q        = ws.queues;
    a.p        = params;
    a.capacity = static_cast<uint32_t>(ws.capacity);
    a.bounce   = 0;
    a.occluded_out = nullptr;
    a.wave         = nullptr;
    MR_CUDA(cudaMemsetAsync(ws.queues.counters, 0, (params.maximum_depth + 2) * sizeof(BounceCounters),
                            stream));
    const unsigned blocks = (init.count + 127) / 128;
    if (init.kind == kInitRays) {
        init_rays_kernel<<<blocks, 128, 0, stream>>>(a, init);
    } else {
        init_camera_kernel<<<blocks, 128, 0, stream>>>(a, init);
    }
    const LaunchShape& shape = launch_shape();
    const bool         media = scene.d.medium_count > 0;
    const bool         two   = scene.d.two_level != 0;
    // Large waves sort each bounce's extension rays by origin cell and direction; small ones
    // keep their order (the sort's fixed cost would outweigh the coherence it buys).
    const bool         ray_sort = ws.queues.staging != nullptr && init.count >= kRaySortMinPaths &&
                                  scene.d.slot_count >= kRaySortMinSlots;
    if (!ray_sort) {
        a.q.staging = nullptr;
    }
    KernelTiming&      timing = kernel_timing();
    bool               timed  = false;
    timed = timing.enabled.load();
    note_launches(1 + 2ull * (params.maximum_depth + 1) + (ray_sort ? 4ull * params.maximum_depth : 0ull) +
                  (init.capture ? 1 : 0));
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    // The timed launches are the trace kernels: nearest-hit and shadow tests both count.
    unsigned long long before[4] = {0, 0, 0, 0};
    if (timed) {
        MR_CUDA(cudaMemcpyAsync(before, ws.queues.stats + kStatExtendBounds, sizeof(before),
                                cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
    }
    for (uint32_t bounce = 0; bounce <= params.maximum_depth; ++bounce) {
        a.bounce = bounce;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (timed) {
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, stream);
        }
        // The first shadow rays (queued by bounce 0's shading) are traced with bounce 1.
        a.occluded_out = bounce == 1 && init.capture ? init.capture->occluded : nullptr;
        const int variant = (media ? 1 : 0) + (two ? 2 : 0);
        switch (variant) {
        case 0: trace_kernel<false, false, false><<<shape.trace_blocks[0], 128, 0, stream>>>(a); break;
        case 1: trace_kernel<true, false, false><<<shape.trace_blocks[1], 128, 0, stream>>>(a); break;
        case 2: trace_kernel<false, false, true><<<shape.trace_blocks[2], 128, 0, stream>>>(a); break;
        default: trace_kernel<true, false, true><<<shape.trace_blocks[3], 128, 0, stream>>>(a); break;
        }
        a.occluded_out = nullptr;
        if (timed) {
            cudaEventRecord(e1, stream);
            events.emplace_back(e0, e1);
        }
        if (two) {
            shade_kernel<false, true><<<shape.shade_blocks_two, 128, 0, stream>>>(a);
        } else {
            shade_kernel<false, false><<<shape.shade_blocks, 128, 0, stream>>>(a);
        }
        if (ray_sort && bounce < params.maximum_depth) {
            enqueue_sort_scan(a.q.buckets, stream);
            sort_scatter_kernel<<<shape.shade_blocks, 128, 0, stream>>>(a);
        }
        if (bounce == 0 && init.capture) {
            capture_shadow_kernel<<<(init.count + 127) / 128, 128, 0, stream>>>(a, init.capture->rays,
                                                                                init.capture->has_shadow);
        }
    }
    MR_CUDA(cudaGetLastError());
    if (timed) {
        unsigned long long after[4] = {0, 0, 0, 0};
        MR_CUDA(cudaMemcpyAsync(after, ws.queues.stats + kStatExtendBounds, sizeof(after),
                                cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        double seconds = 0;
        for (auto& [e0, e1] : events) {
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            seconds += ms * 1e-3;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
        std::lock_guard<std::mutex> lock(timing.mutex);
        timing.launches += events.size();
        timing.seconds += seconds;
        timing.counted.bounds_tests += (after[0] - before[0]) + (after[2] - before[2]);
        timing.counted.triangle_tests += (after[1] - before[1]) + (after[3] - before[3]);
    }
}

void Engine::batch_occupancy(int& trace_blocks_per_sm, int& shade_blocks_per_sm) {
    int a = 0, b = 0, c = 0;
    int f = 0;
    MR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, trace_kernel<false, true, false>, 128, 0));
    MR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, trace_kernel<true, true, false>, 128, 0));
    MR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, shade_kernel<true, false>, 128, 0));
    MR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&f, shade_kernel<true, true>, 128, 0));
    trace_blocks_per_sm = std::max(1, std::min(a, b));
    shade_blocks_per_sm = std::max(1, std::min(c, f));
}

void Engine::enqueue_batch_paths(const WaveDesc* wave, uint32_t maximum_depth, bool media, bool two,
                                 bool ray_sort, const BatchShape& shape, Workspace& ws,
                                 cudaStream_t stream) {
    if (maximum_depth + 1 > ws.max_bounces || !ws.state.segment) {
        fail(MR_LENGTH_ERROR, "Wave exceeds the workspace capacity");
    }
    int device = 0, sms = 0;
    MR_CUDA(cudaGetDevice(&device));
    MR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    KernelArgs a{};
    a.st           = ws.state;
    a.q            = ws.queues;
    a.capacity     = static_cast<uint32_t>(ws.capacity);
    a.occluded_out = nullptr;
    a.wave         = wave;
    ray_sort       = ray_sort && ws.queues.staging != nullptr;
    if (!ray_sort) {
        a.q.staging = nullptr;
    }
    // The two-level variants keep fewer blocks resident (more registers per thread): their grid
    // is capped at what fits, the persistent loop takes the work either way.
    int trace_blocks = shape.trace_blocks;
    if (two) {
        int per = 0;
        MR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per, media ? trace_kernel<true, true, true> : trace_kernel<false, true, true>, 128, 0));
        trace_blocks = std::min(trace_blocks, sms * std::max(1, per));
    }
    MR_CUDA(cudaMemsetAsync(ws.queues.counters, 0, (maximum_depth + 2) * sizeof(BounceCounters), stream));
    init_batch_kernel<<<sms * 8, 256, 0, stream>>>(a);
    for (uint32_t bounce = 0; bounce <= maximum_depth; ++bounce) {
        a.bounce = bounce;
        switch ((media ? 1 : 0) + (two ? 2 : 0)) {
        case 0: trace_kernel<false, true, false><<<shape.trace_blocks, 128, 0, stream>>>(a); break;
        case 1: trace_kernel<true, true, false><<<shape.trace_blocks, 128, 0, stream>>>(a); break;
        case 2: trace_kernel<false, true, true><<<trace_blocks, 128, 0, stream>>>(a); break;
        default: trace_kernel<true, true, true><<<trace_blocks, 128, 0, stream>>>(a); break;
        }
        if (two) {
            shade_kernel<true, true><<<shape.shade_blocks, 128, 0, stream>>>(a);
        } else {
            shade_kernel<true, false><<<shape.shade_blocks, 128, 0, stream>>>(a);
        }
        if (ray_sort && bounce < maximum_depth) {
            enqueue_sort_scan(a.q.buckets, stream);
            sort_scatter_kernel<<<shape.shade_blocks, 128, 0, stream>>>(a);
        }
    }
    MR_CUDA(cudaGetLastError());
}

void Engine::enqueue_batch_resolve(const WaveDesc* wave, Workspace& ws, cudaStream_t stream) {
    int device = 0, sms = 0;
    MR_CUDA(cudaGetDevice(&device));
    MR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    resolve_batch_kernel<<<sms * 8, 256, 0, stream>>>(ws.state.radiance, wave, ws.queues.error);
    MR_CUDA(cudaGetLastError());
}

void render_tile(const Scene& scene, const IntegratorParams& params, const mr_render_settings& render,
                 uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t s0, uint32_t ns,
                 float4* accumulator, Workspace& ws, cudaStream_t stream, uint32_t accumulator_row0,
                 const TileLane* more, uint32_t more_count) {
    const size_t area = static_cast<size_t>(w) * h;
    if (area == 0 || ns == 0) {
        return;
    }
    constexpr uint32_t kMaxLanes = 4;
    TileLane           lanes[kMaxLanes];
    uint32_t           lane_count = 1;
    lanes[0]                      = TileLane{&ws, stream};
    for (uint32_t i = 0; i < more_count && lane_count < kMaxLanes; ++i) {
        if (more[i].ws && more[i].stream) {
            lanes[lane_count++] = more[i];
        }
    }
    // Events of the multi-lane mode: the start, each lane's last resolve, each lane's end.
    struct Events {
        cudaEvent_t start = nullptr;
        cudaEvent_t resolved[kMaxLanes] = {};
        cudaEvent_t done[kMaxLanes]     = {};
        ~Events() {
            for (cudaEvent_t x : resolved) {
                if (x) {
                    cudaEventDestroy(x);
                }
            }
            for (cudaEvent_t x : done) {
                if (x) {
                    cudaEventDestroy(x);
                }
            }
            if (start) {
                cudaEventDestroy(start);
            }
        }
    } events;
    size_t capacity = ws.capacity;
    if (lane_count > 1) {
        MR_CUDA(cudaEventCreateWithFlags(&events.start, cudaEventDisableTiming));
        MR_CUDA(cudaEventRecord(events.start, stream));  // the accumulator is ready
        for (uint32_t i = 0; i < lane_count; ++i) {
            MR_CUDA(cudaEventCreateWithFlags(&events.resolved[i], cudaEventDisableTiming));
            MR_CUDA(cudaEventCreateWithFlags(&events.done[i], cudaEventDisableTiming));
            capacity = std::min(capacity, lanes[i].ws->capacity);
            if (i > 0) {
                MR_CUDA(cudaStreamWaitEvent(lanes[i].stream, events.start, 0));
            }
        }
    }
    // Split the sample range (and, for huge tiles, the rows) into waves that fit the workspace.
    const uint32_t rows_per_wave =
        area <= capacity ? h : static_cast<uint32_t>(std::max<size_t>(1, capacity / w));
    uint32_t wave = 0;
    for (uint32_t ry = 0; ry < h; ry += rows_per_wave) {
        const uint32_t hh      = std::min(rows_per_wave, h - ry);
        const size_t   a       = static_cast<size_t>(w) * hh;
        const uint32_t per     = static_cast<uint32_t>(std::max<size_t>(1, std::min<size_t>(ns, capacity / a)));
        for (uint32_t s = 0; s < ns; s += per, ++wave) {
            const uint32_t     li   = wave % lane_count;
            Workspace&         lane = *lanes[li].ws;
            const cudaStream_t ls   = lanes[li].stream;
            WaveInit init{};
            init.kind   = kInitCamera;
            init.x0     = x0;
            init.y0     = y0 + ry;
            init.w      = w;
            init.h      = hh;
            init.s0     = s0 + s;
            init.ns     = std::min(per, ns - s);
            init.width  = static_cast<uint32_t>(render.width);
            init.height = static_cast<uint32_t>(render.height);
            init.seed   = render.seed;
            init.count  = static_cast<uint32_t>(a * init.ns);
            Engine::run_wave(scene, params, init, lane, ls);
            if (lane_count > 1 && wave > 0) {  // after the previous wave's resolve, on its lane
                MR_CUDA(cudaStreamWaitEvent(ls, events.resolved[(wave - 1) % lane_count], 0));
            }
            note_launches(1);
            resolve_kernel<<<static_cast<unsigned>((a + 255) / 256), 256, 0, ls>>>(
                lane.state.radiance, init.x0, init.y0, w, hh, init.ns, init.width, accumulator,
                accumulator_row0, lane.queues.error);
            if (lane_count > 1) {
                MR_CUDA(cudaEventRecord(events.resolved[li], ls));
            }
        }
    }
    for (uint32_t i = 1; i < lane_count; ++i) {
        MR_CUDA(cudaEventRecord(events.done[i], lanes[i].stream));
        MR_CUDA(cudaStreamWaitEvent(stream, events.done[i], 0));
    }
    MR_CUDA(cudaGetLastError());
}

void render_frame(const Scene& scene, const IntegratorParams& params, const mr_render_settings& render,
                  float* device_rgb, cudaStream_t stream, mr_path_statistics* statistics,
                  size_t max_paths, uint32_t row_begin, uint32_t row_end) {
    row_end               = std::min<uint32_t>(row_end, static_cast<uint32_t>(render.height));
    const uint32_t rows   = row_end > row_begin ? row_end - row_begin : 0;
    const size_t pixels   = static_cast<size_t>(render.width) * rows;
    const size_t total    = pixels * render.samples_per_pixel;
    if (total == 0) {
        if (statistics) {
            *statistics = {};
        }
        return;
    }
    const size_t capacity = std::min(total, max_paths ? max_paths : (size_t(1) << 23));
    auto         ws       = acquire_workspace(capacity, params.maximum_depth + 1, pixels);
    // A frame of several waves goes round kFrameLanes workspaces, each with its own stream.
    // The extra workspaces go back to the pool only once the frame has finished; after an error
    // they are freed (cudaFree waits for the work still queued on them).
    struct MoreLanes {
        std::shared_ptr<Workspace> ws[kFrameLanes - 1];
        TileLane                   lanes[kFrameLanes - 1];
        uint32_t                   count    = 0;
        bool                       finished = false;
        ~MoreLanes() {
            for (uint32_t i = 0; i < count; ++i) {
                if (lanes[i].stream) {
                    cudaStreamDestroy(lanes[i].stream);
                }
                if (finished) {
                    release_workspace(ws[i]);
                }
            }
        }
    } more;
    if (total > capacity && max_paths == 0) {
        const size_t waves = (total + capacity - 1) / capacity;
        for (uint32_t i = 0; i + 1 < kFrameLanes && i + 1 < waves; ++i) {
            // A lane that does not fit in device memory is left out: the frame renders on the
            // lanes it has (the same image, less overlap).
            try {
                more.ws[i] = acquire_workspace(capacity, params.maximum_depth + 1, 0);
            } catch (const Error& e) {
                if (e.status != MR_OUT_OF_MEMORY) {
                    throw;
                }
                (void)cudaGetLastError();  // a failed allocation is not a sticky error
                break;
            }
            more.lanes[i].ws = more.ws[i].get();
            ++more.count;
            MR_CUDA(cudaStreamCreateWithFlags(&more.lanes[i].stream, cudaStreamNonBlocking));
            reset_statistics(*more.ws[i], stream);
        }
    }
    reset_statistics(*ws, stream);
    MR_CUDA(cudaMemsetAsync(ws->accumulator, 0, 2 * pixels * sizeof(float4), stream));
    render_tile(scene, params, render, 0, row_begin, static_cast<uint32_t>(render.width), rows, 0,
                render.samples_per_pixel, ws->accumulator, *ws, stream, row_begin, more.lanes, more.count);
    note_launches(1);
    finalize_kernel<<<static_cast<unsigned>((pixels + 255) / 256), 256, 0, stream>>>(
        ws->accumulator, pixels, render.samples_per_pixel, device_rgb, ws->queues.error);
    MR_CUDA(cudaGetLastError());
    unsigned error = 0;
    read_statistics(*ws, stream, statistics, &error);
    for (uint32_t i = 0; i < more.count; ++i) {
        mr_path_statistics other{};
        unsigned           other_error = 0;
        read_statistics(*more.ws[i], stream, statistics ? &other : nullptr, &other_error);
        error |= other_error;
        if (statistics) {
            statistics->paths += other.paths;
            statistics->shadow_rays += other.shadow_rays;
            statistics->scattering_events += other.scattering_events;
            statistics->roulette_terminations += other.roulette_terminations;
            statistics->medium_scattering_events += other.medium_scattering_events;
            statistics->geometry.bounds_tests += other.geometry.bounds_tests;
            statistics->geometry.triangle_tests += other.geometry.triangle_tests;
        }
    }
    more.finished = true;
    release_workspace(ws);
    std::string message;
    const mr_status status = error_status(error, message);
    if (status != MR_OK) {
        fail(status, message);
    }
}

// Per-path radiance of an explicit wave (trace_paths / sample_pixels).
void copy_path_radiance(Workspace& ws, uint32_t count, float* device_out, cudaStream_t stream) {
    copy_radiance_kernel<<<(count + 255) / 256, 256, 0, stream>>>(ws.state.radiance, count, device_out);
    MR_CUDA(cudaGetLastError());
}

}  // namespace mr
