// abi.cu — the C ABI of include/minirender_b200.h: argument validation, exception-to-status
// mapping, ray queries, path queries, frame rendering and render sessions.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "errors.hpp"
#include "instancing.cuh"
#include "shading.cuh"
#include "validation.hpp"
#include "wavefront.cuh"

struct mr_scene {
    std::unique_ptr<mr::Scene> impl;
};

struct mr_session {
    std::mutex              control;
    std::condition_variable changed;
    uint32_t                state   = MR_STATE_IDLE;
    uint64_t                job     = 0;
    uint64_t                total   = 0;
    std::atomic<uint64_t>   recorded{0};
    std::atomic<uint64_t>   completed_pixels{0};
    bool                    pause_requested  = false;
    bool                    cancel_requested = false;
    std::string             error;
    std::chrono::steady_clock::time_point started{}, finished{};
    mr_path_statistics      statistics{};
    std::thread             controller;
    int                     device = 0;
    // Film: device accumulator (sum, compensation per pixel) and its host mirror for previews.
    mr_render_settings      render{};
    std::mutex              film;
    std::vector<float>      image;   // mean per pixel of the committed samples (host)
    uint64_t                revision = 0;
    uint32_t                committed_samples = 0;  // per pixel (whole-image batches)
    std::shared_ptr<std::vector<float>> result;

    void set_state(uint32_t s) {
        std::lock_guard<std::mutex> lock(control);
        state = s;
        changed.notify_all();
    }
};


namespace mr {

void copy_path_radiance(Workspace& ws, uint32_t count, float* device_out, cudaStream_t stream);

namespace {

// A non-blocking stream owned by one API call.
struct CallStream {
    cudaStream_t stream = nullptr;
    CallStream() { MR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); }
    ~CallStream() { cudaStreamDestroy(stream); }
    CallStream(const CallStream&)            = delete;
    CallStream& operator=(const CallStream&) = delete;
};

thread_local std::string last_error;

template <typename F> mr_status guarded(F&& f) {
    try {
        f();
        return MR_OK;
    } catch (const Error& e) {
        last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        last_error = "Host allocation failed";
        return MR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        last_error = e.what();
        return MR_RUNTIME_ERROR;
    }
}

// RayQuery constructor and RayInterval::validate (src/render/intersection.cpp:22-26,52-61).
void validate_ray(const mr_ray& r) {
    for (int a = 0; a < 3; ++a) {
        require(std::isfinite(r.origin[a]) && std::isfinite(r.direction[a]),
                "Ray origin and direction must be finite");
    }
    const double d2 = double(r.direction[0]) * r.direction[0] + double(r.direction[1]) * r.direction[1] +
                      double(r.direction[2]) * r.direction[2];
    require(std::fabs(d2 - 1) <= 1e-4, "Ray direction must have unit length");
    require(std::isfinite(r.minimum) && r.minimum >= 0 && !std::isnan(r.maximum) && r.maximum >= r.minimum,
            "Ray interval must satisfy 0 <= minimum <= maximum");
}

const Scene& scene_of(const mr_scene* s) {
    require(s != nullptr && s->impl != nullptr, "Scene handle is null");
    return *s->impl;
}

// Device copy helpers.
template <typename T> DeviceBuffer<T> upload(const T* host, size_t count, cudaStream_t stream) {
    DeviceBuffer<T> b;
    b.allocate(std::max<size_t>(1, count));
    if (count) {
        MR_CUDA(cudaMemcpyAsync(b.ptr, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
    }
    return b;
}

__global__ void query_kernel(DeviceScene s, const mr_ray* rays, size_t count, int any_hit,
                             mr_hit* hits, uint8_t* occluded, unsigned long long* counters,
                             unsigned* error) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    TraceCounters tc{0, 0};
    unsigned      err = 0;
    if (i < count) {
        const mr_ray r = rays[i];
        RayQuery     q;
        q.init(make(r.origin[0], r.origin[1], r.origin[2]),
               make(r.direction[0], r.direction[1], r.direction[2]));
        if (any_hit) {
            const TraceResult t = s.two_level ? trace2<true>(s, q, r.minimum, r.maximum, tc, err)
                                              : trace<true>(s, q, r.minimum, r.maximum, tc, err);
            occluded[i]         = t.slot != kNone ? 1 : 0;
        } else {
            const TraceResult t = s.two_level ? trace2<false>(s, q, r.minimum, r.maximum, tc, err)
                                              : trace<false>(s, q, r.minimum, r.maximum, tc, err);
            mr_hit            h{};
            h.primitive = kNone;
            if (t.slot != kNone) {
                const float b0 = __fdiv_rn(t.a, t.det), b1 = __fdiv_rn(t.b, t.det),
                            b2 = __fdiv_rn(t.c, t.det);
                const SurfaceHit sh = surface_hit<true>(s, q.d, t.slot, b0, b1, b2);
                h.distance       = t.t;
                h.instance_index = sh.instance;
                h.triangle_index = sh.triangle;
                h.primitive      = t.prim;
                h.barycentric[0] = b0;
                h.barycentric[1] = b1;
                h.barycentric[2] = b2;
                h.front_face     = sh.front_face ? 1u : 0u;
            }
            hits[i] = h;
        }
    }
    const uint32_t b = __reduce_add_sync(0xffffffffu, tc.bounds);
    const uint32_t t = __reduce_add_sync(0xffffffffu, tc.triangles);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counters, static_cast<unsigned long long>(b));
        atomicAdd(counters + 1, static_cast<unsigned long long>(t));
    }
    if (err) {
        atomicOr(error, err);
    }
}

void run_query(const Scene& scene, const mr_ray* rays, size_t count, int any_hit, mr_hit* hits,
               uint8_t* occluded, mr_trace_statistics* statistics) {
    require(rays != nullptr || count == 0, "Ray buffer is null");
    require((any_hit ? occluded != nullptr : hits != nullptr) || count == 0, "Output buffer is null");
    for (size_t i = 0; i < count; ++i) {
        validate_ray(rays[i]);
    }
    cudaStream_t stream = nullptr;
    auto         d_rays = upload(rays, count, stream);
    DeviceBuffer<mr_hit>             d_hits;
    DeviceBuffer<uint8_t>            d_occ;
    DeviceBuffer<unsigned long long> d_counters;
    DeviceBuffer<unsigned>           d_error;
    d_hits.allocate(any_hit ? 1 : std::max<size_t>(1, count));
    d_occ.allocate(any_hit ? std::max<size_t>(1, count) : 1);
    d_counters.allocate(2);
    d_error.allocate(1);
    MR_CUDA(cudaMemsetAsync(d_counters.ptr, 0, 2 * sizeof(unsigned long long), stream));
    MR_CUDA(cudaMemsetAsync(d_error.ptr, 0, sizeof(unsigned), stream));
    if (count) {
        query_kernel<<<static_cast<unsigned>((count + 127) / 128), 128, 0, stream>>>(
            scene.d, d_rays.ptr, count, any_hit, d_hits.ptr, d_occ.ptr, d_counters.ptr, d_error.ptr);
        MR_CUDA(cudaGetLastError());
        if (any_hit) {
            MR_CUDA(cudaMemcpyAsync(occluded, d_occ.ptr, count, cudaMemcpyDeviceToHost, stream));
        } else {
            MR_CUDA(cudaMemcpyAsync(hits, d_hits.ptr, count * sizeof(mr_hit), cudaMemcpyDeviceToHost, stream));
        }
    }
    unsigned long long counters[2] = {0, 0};
    unsigned           error       = 0;
    MR_CUDA(cudaMemcpyAsync(counters, d_counters.ptr, sizeof(counters), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaMemcpyAsync(&error, d_error.ptr, sizeof(error), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    std::string message;
    const mr_status status = error_status(error, message);
    if (status != MR_OK) {
        fail(status, message);
    }
    if (statistics) {
        statistics->bounds_tests += counters[0];
        statistics->triangle_tests += counters[1];
    }
}

// Explicit-path waves (PathTracer::trace / sample_pixel) in chunks of at most 4M paths.
void run_paths(const Scene& scene, const IntegratorParams& params, WaveInit init, size_t count,
               const mr_ray* rays, const uint64_t* keys, const uint32_t* pixels,
               const uint64_t* samples, float* radiance, mr_ray* camera_rays,
               mr_path_statistics* statistics, mr_ray* shadow_rays = nullptr,
               uint8_t* has_shadow = nullptr, uint8_t* occluded = nullptr) {
    cudaStream_t stream = nullptr;
    const size_t chunk  = std::min<size_t>(std::max<size_t>(1, count), size_t(1) << 22);
    auto         ws     = acquire_workspace(chunk, params.maximum_depth + 1, 1);
    reset_statistics(*ws, stream);
    DeviceBuffer<float>    d_out;
    DeviceBuffer<float4>   d_rays, d_cam;
    DeviceBuffer<uint64_t> d_keys, d_samples;
    DeviceBuffer<uint32_t> d_pixels;
    d_out.allocate(3 * chunk);
    if (camera_rays) {
        d_cam.allocate(2 * chunk);
    }
    DeviceBuffer<float4>  d_shadow;
    DeviceBuffer<uint8_t> d_has, d_occ;
    ShadowCapture         capture{};
    if (shadow_rays) {
        d_shadow.allocate(2 * chunk);
        d_has.allocate(chunk);
        d_occ.allocate(chunk);
        capture = {d_shadow.ptr, d_has.ptr, d_occ.ptr};
    }
    for (size_t begin = 0; begin < count; begin += chunk) {
        const size_t n = std::min(chunk, count - begin);
        WaveInit     w = init;
        w.count        = static_cast<uint32_t>(n);
        if (init.kind == kInitRays) {
            std::vector<float4> packed(2 * n);
            for (size_t i = 0; i < n; ++i) {
                const mr_ray& r = rays[begin + i];
                packed[2 * i]     = make_float4(r.origin[0], r.origin[1], r.origin[2], r.minimum);
                packed[2 * i + 1] = make_float4(r.direction[0], r.direction[1], r.direction[2], r.maximum);
            }
            d_rays = upload(packed.data(), packed.size(), stream);
            d_keys = upload(keys + 3 * begin, 3 * n, stream);
            w.rays = d_rays.ptr;
            w.keys = d_keys.ptr;
        } else {
            d_pixels  = upload(pixels + 2 * begin, 2 * n, stream);
            d_samples = upload(samples + begin, n, stream);
            w.pixels  = d_pixels.ptr;
            w.samples = d_samples.ptr;
            w.camera_rays_out = camera_rays ? d_cam.ptr : nullptr;
        }
        if (shadow_rays) {
            MR_CUDA(cudaMemsetAsync(d_has.ptr, 0, n, stream));
            MR_CUDA(cudaMemsetAsync(d_occ.ptr, 0, n, stream));
            w.capture = &capture;
        }
        Engine::run_wave(scene, params, w, *ws, stream);
        copy_path_radiance(*ws, static_cast<uint32_t>(n), d_out.ptr, stream);
        if (shadow_rays) {
            std::vector<float4> sr(2 * n);
            MR_CUDA(cudaMemcpyAsync(sr.data(), d_shadow.ptr, 2 * n * sizeof(float4), cudaMemcpyDeviceToHost,
                                    stream));
            MR_CUDA(cudaMemcpyAsync(has_shadow + begin, d_has.ptr, n, cudaMemcpyDeviceToHost, stream));
            MR_CUDA(cudaMemcpyAsync(occluded + begin, d_occ.ptr, n, cudaMemcpyDeviceToHost, stream));
            MR_CUDA(cudaStreamSynchronize(stream));
            for (size_t i = 0; i < n; ++i) {
                mr_ray& r = shadow_rays[begin + i];
                r.origin[0] = sr[2 * i].x, r.origin[1] = sr[2 * i].y, r.origin[2] = sr[2 * i].z;
                r.direction[0] = sr[2 * i + 1].x, r.direction[1] = sr[2 * i + 1].y,
                r.direction[2] = sr[2 * i + 1].z;
                r.minimum = 0.0f;
                r.maximum = sr[2 * i].w;
            }
        }
        MR_CUDA(cudaMemcpyAsync(radiance + 3 * begin, d_out.ptr, 3 * n * sizeof(float),
                                cudaMemcpyDeviceToHost, stream));
        if (camera_rays) {
            std::vector<float4> cam(2 * n);
            MR_CUDA(cudaMemcpyAsync(cam.data(), d_cam.ptr, 2 * n * sizeof(float4), cudaMemcpyDeviceToHost,
                                    stream));
            MR_CUDA(cudaStreamSynchronize(stream));
            for (size_t i = 0; i < n; ++i) {
                mr_ray& r      = camera_rays[begin + i];
                r.origin[0]    = cam[2 * i].x;
                r.origin[1]    = cam[2 * i].y;
                r.origin[2]    = cam[2 * i].z;
                r.minimum      = cam[2 * i].w;
                r.direction[0] = cam[2 * i + 1].x;
                r.direction[1] = cam[2 * i + 1].y;
                r.direction[2] = cam[2 * i + 1].z;
                r.maximum      = cam[2 * i + 1].w;
            }
        }
        MR_CUDA(cudaStreamSynchronize(stream));
    }
    unsigned error = 0;
    read_statistics(*ws, stream, statistics, &error);
    release_workspace(ws);
    std::string message;
    const mr_status status = error_status(error, message);
    if (status != MR_OK) {
        fail(status, message);
    }
    for (size_t i = 0; i < 3 * count; ++i) {
        if (!std::isfinite(radiance[i]) || radiance[i] < 0) {
            fail(MR_RUNTIME_ERROR, "Path contribution is nonfinite or negative");
        }
    }
}

// ---- render session (RenderSession, src/render/render_session.cpp) ----

bool terminal(uint32_t s) {
    return s == MR_STATE_IDLE || s == MR_STATE_CANCELLED || s == MR_STATE_COMPLETED ||
           s == MR_STATE_FAILED;
}

}  // namespace

}  // namespace mr

namespace mr {
namespace {

__global__ void mean_kernel(const float4* accumulator, size_t pixels, uint32_t samples, float* rgb) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < pixels) {
        const float4 s = accumulator[2 * i], c = accumulator[2 * i + 1];
        const float  n = static_cast<float>(samples);
        rgb[3 * i]     = (s.x + c.x) / n;
        rgb[3 * i + 1] = (s.y + c.y) / n;
        rgb[3 * i + 2] = (s.z + c.z) / n;
    }
}

// Controller thread: whole-image sample batches of `batch_samples`, each committed to the film
// before the next; pause parks between batches, cancel stops between batches (worker loop of
// src/render/render_session.cpp:412-459 with the image as one tile).
void session_run(mr_session* s, const Scene* scene, IntegratorParams params, mr_render_settings render,
                 mr_session_settings settings) {
    try {
        MR_CUDA(cudaSetDevice(s->device));
        cudaStream_t stream;
        MR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        const size_t pixels = static_cast<size_t>(render.width) * render.height;
        const size_t capacity =
            std::min<size_t>(pixels * std::min<uint32_t>(render.samples_per_pixel, settings.batch_samples),
                             size_t(1) << 23);
        auto ws = acquire_workspace(std::max<size_t>(1, capacity), params.maximum_depth + 1, pixels);
        reset_statistics(*ws, stream);
        MR_CUDA(cudaMemsetAsync(ws->accumulator, 0, 2 * pixels * sizeof(float4), stream));
        DeviceBuffer<float> mean;
        mean.allocate(3 * pixels);
        s->set_state(MR_STATE_RUNNING);
        bool cancelled = false;
        for (uint32_t s0 = 0; s0 < render.samples_per_pixel;) {
            {
                std::unique_lock<std::mutex> lock(s->control);
                if (s->pause_requested && !s->cancel_requested) {
                    s->state = MR_STATE_PAUSED;
                    s->changed.notify_all();
                    s->changed.wait(lock, [&] { return !s->pause_requested || s->cancel_requested; });
                    if (!s->cancel_requested) {
                        s->state = MR_STATE_RUNNING;
                    }
                }
                if (s->cancel_requested) {
                    cancelled = true;
                    break;
                }
            }
            const uint32_t ns = std::min(settings.batch_samples, render.samples_per_pixel - s0);
            render_tile(*scene, params, render, 0, 0, static_cast<uint32_t>(render.width),
                        static_cast<uint32_t>(render.height), s0, ns, ws->accumulator, *ws, stream);
            mean_kernel<<<static_cast<unsigned>((pixels + 255) / 256), 256, 0, stream>>>(
                ws->accumulator, pixels, s0 + ns, mean.ptr);
            unsigned           error = 0;
            mr_path_statistics stats{};
            read_statistics(*ws, stream, &stats, &error);
            std::string     message;
            const mr_status status = error_status(error, message);
            if (status != MR_OK) {
                fail(status, message);
            }
            {
                std::lock_guard<std::mutex> lock(s->film);
                MR_CUDA(cudaMemcpyAsync(s->image.data(), mean.ptr, 3 * pixels * sizeof(float),
                                        cudaMemcpyDeviceToHost, stream));
                MR_CUDA(cudaStreamSynchronize(stream));
                s->committed_samples = s0 + ns;
                ++s->revision;
            }
            s0 += ns;
            s->recorded.store(pixels * s0);
            if (s0 == render.samples_per_pixel) {
                s->completed_pixels.store(pixels);
            }
            std::lock_guard<std::mutex> lock(s->control);
            s->statistics = stats;
        }
        release_workspace(ws);
        cudaStreamDestroy(stream);
        if (cancelled) {
            std::lock_guard<std::mutex> lock(s->control);
            s->state    = MR_STATE_CANCELLED;
            s->finished = std::chrono::steady_clock::now();
            s->changed.notify_all();
            return;
        }
        s->set_state(MR_STATE_FINALIZING);
        // Overflow check of the final image (src/render/render_session.cpp:39-74).
        for (float v : s->image) {
            if (!std::isfinite(v)) {
                fail(MR_OVERFLOW, "Render sample exceeds the float image range");
            }
        }
        {
            std::lock_guard<std::mutex> lock(s->film);
            s->result = std::make_shared<std::vector<float>>(s->image);
        }
        std::lock_guard<std::mutex> lock(s->control);
        s->state    = s->cancel_requested ? MR_STATE_CANCELLED : MR_STATE_COMPLETED;
        s->finished = std::chrono::steady_clock::now();
        s->changed.notify_all();
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lock(s->control);
        if (s->error.empty()) {
            s->error = e.what();
        }
        s->state    = MR_STATE_FAILED;
        s->finished = std::chrono::steady_clock::now();
        s->changed.notify_all();
    }
}

}  // namespace

// Lets the other C-ABI translation units report through mr_last_error.
void set_last_error(const std::string& message) { last_error = message; }

}  // namespace mr

using namespace mr;

extern "C" {

uint32_t mr_abi_version(void) { return MR_ABI_VERSION; }

size_t mr_last_error(char* buffer, size_t capacity) {
    if (buffer && capacity) {
        const size_t n = std::min(capacity - 1, last_error.size());
        std::memcpy(buffer, last_error.data(), n);
        buffer[n] = 0;
    }
    return last_error.size();
}

mr_status mr_scene_create(const mr_scene_desc* desc, const mr_bvh_desc* bvh, mr_scene** scene) {
    return guarded([&] {
        require(desc != nullptr && scene != nullptr, "Scene descriptor or output is null");
        auto s  = std::make_unique<mr_scene>();
        s->impl = create_scene(*desc, bvh);
        *scene  = s.release();
    });
}

mr_status mr_scene_create_with(const mr_scene_desc* desc, const mr_bvh_desc* bvh,
                               const mr_build_settings* build, mr_scene** scene) {
    return guarded([&] {
        require(desc != nullptr && scene != nullptr, "Scene descriptor or output is null");
        require(!(bvh && build && (build->split_references || build->two_level)),
                "Split references and two levels apply to the GPU builder, not to an imported tree");
        auto s  = std::make_unique<mr_scene>();
        s->impl = create_scene(*desc, bvh, build);
        *scene  = s.release();
    });
}

mr_status mr_scene_destroy(mr_scene* scene) {
    return guarded([&] { delete scene; });
}

mr_status mr_scene_update_instances(mr_scene* scene, uint32_t first, uint32_t count,
                                    const mr_instance* instances) {
    return guarded([&] {
        require(scene != nullptr && scene->impl != nullptr, "Scene handle is null");
        update_instances(*scene->impl, first, count, instances);
    });
}

mr_status mr_scene_update_mesh(mr_scene* scene, uint32_t mesh, const float* positions,
                               uint32_t position_count) {
    return guarded([&] {
        require(scene != nullptr && scene->impl != nullptr, "Scene handle is null");
        update_mesh(*scene->impl, mesh, positions, position_count);
    });
}

mr_status mr_scene_device_bytes(const mr_scene* scene, uint64_t* bytes) {
    return guarded([&] {
        require(bytes != nullptr, "Output is null");
        *bytes = scene_of(scene).device_bytes;
    });
}

mr_status mr_scene_bvh_statistics(const mr_scene* scene, mr_bvh_statistics* statistics) {
    return guarded([&] {
        require(statistics != nullptr, "Output is null");
        *statistics = scene_of(scene).statistics;
    });
}

mr_status mr_scene_export_bvh(const mr_scene* scene, mr_bvh_node* nodes, uint32_t node_capacity,
                              uint32_t* order, uint32_t order_capacity, uint32_t* node_count,
                              uint32_t* primitive_count) {
    return guarded([&] {
        const Scene&   s = scene_of(scene);
        const uint32_t n = static_cast<uint32_t>(s.ref_nodes.count);
        const uint32_t p = s.d.primitive_count;
        if (s.two) {
            fail(MR_LOGIC_ERROR, "A two-level scene has no reference-layout export");
        }
        if (s.references != p) {
            fail(MR_LOGIC_ERROR, "A tree with split references has no reference-layout export");
        }
        if (node_count) {
            *node_count = n;
        }
        if (primitive_count) {
            *primitive_count = p;
        }
        if (nodes) {
            require(node_capacity >= n, "Node buffer is too small");
            if (n) {
                MR_CUDA(cudaMemcpy(nodes, s.ref_nodes.ptr, n * sizeof(mr_bvh_node), cudaMemcpyDeviceToHost));
            }
        }
        if (order) {
            require(order_capacity >= p, "Order buffer is too small");
            if (p) {
                MR_CUDA(cudaMemcpy(order, s.ref_order.ptr, p * sizeof(uint32_t), cudaMemcpyDeviceToHost));
            }
        }
    });
}

mr_status mr_scene_sah_cost(const mr_scene* scene, double* cost) {
    return guarded([&] {
        require(cost != nullptr, "Output is null");
        const Scene& s = scene_of(scene);
        if (s.two) {
            fail(MR_LOGIC_ERROR, "A two-level scene has no single tree whose SAH cost compares "
                                 "with the reference builder's");
        }
        const size_t n = s.ref_nodes.count;
        *cost          = 0;
        if (n == 0) {
            return;
        }
        std::vector<mr_bvh_node> nodes(n);
        MR_CUDA(cudaMemcpy(nodes.data(), s.ref_nodes.ptr, n * sizeof(mr_bvh_node), cudaMemcpyDeviceToHost));
        // Areas as the reference computes them (Bounds3::surface_area, intersection.cpp:44-50).
        const auto area = [](const mr_bvh_node& b) {
            const double ex = double(b.maximum[0]) - b.minimum[0];
            const double ey = double(b.maximum[1]) - b.minimum[1];
            const double ez = double(b.maximum[2]) - b.minimum[2];
            if (ex < 0 || ey < 0 || ez < 0) {
                return 0.0;
            }
            return 2 * (ex * ey + ey * ez + ez * ex);
        };
        const double root = area(nodes[0]);
        double       sum  = 0;
        for (const auto& b : nodes) {
            sum += (b.count ? double(b.count) : 1.0) * area(b) / root;
        }
        *cost = sum;
    });
}

mr_status mr_scene_build_seconds(const mr_scene* scene, double* seconds) {
    return guarded([&] {
        require(seconds != nullptr, "Output is null");
        *seconds = scene_of(scene).build_seconds;
    });
}

mr_status mr_intersect(const mr_scene* scene, const mr_ray* rays, size_t count, mr_hit* hits,
                       mr_trace_statistics* statistics) {
    return guarded([&] { run_query(scene_of(scene), rays, count, 0, hits, nullptr, statistics); });
}

mr_status mr_occluded(const mr_scene* scene, const mr_ray* rays, size_t count, uint8_t* occluded,
                      mr_trace_statistics* statistics) {
    return guarded([&] { run_query(scene_of(scene), rays, count, 1, nullptr, occluded, statistics); });
}

mr_status mr_trace_paths(const mr_scene* scene, const mr_integrator_settings* integrator,
                         const mr_ray* rays, const uint64_t* keys, size_t count, float* radiance,
                         mr_path_statistics* statistics) {
    return guarded([&] {
        const Scene&           s = scene_of(scene);
        const IntegratorParams p = integrator_params(integrator);
        require((rays && keys && radiance) || count == 0, "Path buffers are null");
        for (size_t i = 0; i < count; ++i) {
            validate_ray(rays[i]);
        }
        WaveInit init{};
        init.kind = kInitRays;
        if (count) {
            run_paths(s, p, init, count, rays, keys, nullptr, nullptr, radiance, nullptr, statistics);
        } else if (statistics) {
            std::memset(statistics, 0, sizeof(*statistics));
        }
    });
}

mr_status mr_sample_pixels(const mr_scene* scene, const mr_integrator_settings* integrator,
                           const mr_render_settings* render, const uint32_t* pixels,
                           const uint64_t* samples, size_t count, float* radiance, mr_ray* rays,
                           mr_path_statistics* statistics) {
    return guarded([&] {
        const Scene&           s = scene_of(scene);
        const IntegratorParams p = integrator_params(integrator);
        validate_render(render);
        require((pixels && samples && radiance) || count == 0, "Pixel buffers are null");
        for (size_t i = 0; i < count; ++i) {
            if (pixels[2 * i] >= render->width || pixels[2 * i + 1] >= render->height) {
                fail(MR_OUT_OF_RANGE, "Pixel coordinates are outside the render image");
            }
        }
        WaveInit init{};
        init.kind   = kInitPixelList;
        init.width  = static_cast<uint32_t>(render->width);
        init.height = static_cast<uint32_t>(render->height);
        init.seed   = render->seed;
        if (count) {
            run_paths(s, p, init, count, nullptr, nullptr, pixels, samples, radiance, rays, statistics);
        } else if (statistics) {
            std::memset(statistics, 0, sizeof(*statistics));
        }
    });
}

mr_status mr_capture_shadow_rays(const mr_scene* scene, const mr_integrator_settings* integrator,
                                 const mr_render_settings* render, const uint32_t* pixels,
                                 const uint64_t* samples, size_t count, mr_ray* shadow_rays,
                                 uint8_t* has_shadow, uint8_t* occluded) {
    return guarded([&] {
        const Scene&           s = scene_of(scene);
        const IntegratorParams p = integrator_params(integrator);
        validate_render(render);
        require((pixels && samples && shadow_rays && has_shadow && occluded) || count == 0,
                "Capture buffers are null");
        for (size_t i = 0; i < count; ++i) {
            if (pixels[2 * i] >= render->width || pixels[2 * i + 1] >= render->height) {
                fail(MR_OUT_OF_RANGE, "Pixel coordinates are outside the render image");
            }
        }
        WaveInit init{};
        init.kind   = kInitPixelList;
        init.width  = static_cast<uint32_t>(render->width);
        init.height = static_cast<uint32_t>(render->height);
        init.seed   = render->seed;
        if (count) {
            std::vector<float> radiance(3 * count);
            mr_path_statistics stats{};
            run_paths(s, p, init, count, nullptr, nullptr, pixels, samples, radiance.data(), nullptr,
                      &stats, shadow_rays, has_shadow, occluded);
        }
    });
}

mr_status mr_render_device(const mr_scene* scene, const mr_integrator_settings* integrator,
                           const mr_render_settings* render, float* device_rgb, void* stream,
                           mr_path_statistics* statistics) {
    return guarded([&] {
        const Scene&           s = scene_of(scene);
        const IntegratorParams p = integrator_params(integrator);
        validate_render(render);
        require(device_rgb != nullptr, "Output image is null");
        mr_path_statistics local{};
        render_frame(s, p, *render, device_rgb, static_cast<cudaStream_t>(stream),
                     statistics ? statistics : &local);
    });
}

mr_status mr_render_rows(const mr_scene* scene, const mr_integrator_settings* integrator,
                         const mr_render_settings* render, uint64_t row_begin, uint64_t row_end,
                         float* rgb, mr_path_statistics* statistics) {
    return guarded([&] {
        const Scene&           s = scene_of(scene);
        const IntegratorParams p = integrator_params(integrator);
        validate_render(render);
        require(row_begin <= row_end && row_end <= render->height, "Row range is outside the image");
        require(rgb != nullptr || row_begin == row_end, "Output image is null");
        const size_t pixels = static_cast<size_t>(render->width) * (row_end - row_begin);
        mr_path_statistics local{};
        if (pixels == 0) {
            if (statistics) {
                *statistics = local;
            }
            return;
        }
        CallStream          call;
        AllocationScope     scope(call.stream);
        DeviceBuffer<float> image;
        image.allocate(3 * pixels);
        render_frame(s, p, *render, image.ptr, call.stream, statistics ? statistics : &local, 0,
                     static_cast<uint32_t>(row_begin), static_cast<uint32_t>(row_end));
        MR_CUDA(cudaMemcpyAsync(rgb, image.ptr, 3 * pixels * sizeof(float), cudaMemcpyDeviceToHost,
                                call.stream));
        MR_CUDA(cudaStreamSynchronize(call.stream));
    });
}

mr_status mr_render(const mr_scene* scene, const mr_integrator_settings* integrator,
                    const mr_render_settings* render, float* rgb, mr_path_statistics* statistics) {
    return guarded([&] {
        const Scene&           s = scene_of(scene);
        const IntegratorParams p = integrator_params(integrator);
        validate_render(render);
        require(rgb != nullptr, "Output image is null");
        const size_t        pixels = static_cast<size_t>(render->width) * render->height;
        // The call's own stream and stream-ordered image buffer: no device-wide synchronisation
        // from an allocation or from the legacy stream.
        CallStream          call;
        AllocationScope     scope(call.stream);
        DeviceBuffer<float> image;
        image.allocate(3 * pixels);
        mr_path_statistics local{};
        render_frame(s, p, *render, image.ptr, call.stream, statistics ? statistics : &local);
        MR_CUDA(cudaMemcpyAsync(rgb, image.ptr, 3 * pixels * sizeof(float), cudaMemcpyDeviceToHost,
                                call.stream));
        MR_CUDA(cudaStreamSynchronize(call.stream));
    });
}

mr_status mr_display_image(const float* linear, uint64_t width, uint64_t height, double exposure,
                           float* display) {
    return guarded([&] {
        require(linear && display, "Image buffers are null");
        require(std::isfinite(exposure) && std::fabs(exposure) <= 64,
                "Display exposure must be finite and in [-64,64]");
        const float scale = std::exp2(static_cast<float>(exposure));
        for (uint64_t i = 0; i < 3 * width * height; ++i) {
            require(std::isfinite(linear[i]), "Display input contains nonfinite radiance");
        }
        for (uint64_t i = 0; i < 3 * width * height; ++i) {
            const float p = std::max(linear[i], 0.0f) * scale;
            display[i]    = p / (1.0f + p);
        }
    });
}

mr_status mr_set_kernel_timing(int enabled) {
    return guarded([&] {
        KernelTiming&               t = kernel_timing();
        std::lock_guard<std::mutex> lock(t.mutex);
        t.enabled  = enabled != 0;
        t.all_launches = 0;
        t.launches = 0;
        t.seconds  = 0;
        t.counted  = {};
    });
}

mr_status mr_kernel_timing(uint64_t* launches, double* seconds, mr_trace_statistics* counted,
                           uint64_t* all_launches) {
    return guarded([&] {
        KernelTiming&               t = kernel_timing();
        std::lock_guard<std::mutex> lock(t.mutex);
        if (launches) *launches = t.launches;
        if (seconds) *seconds = t.seconds;
        if (counted) *counted = t.counted;
        if (all_launches) *all_launches = t.all_launches.load();
    });
}

mr_status mr_session_create(mr_session** session) {
    return guarded([&] {
        require(session != nullptr, "Output is null");
        *session = new mr_session();
    });
}

mr_status mr_session_destroy(mr_session* session) {
    return guarded([&] {
        if (!session) {
            return;
        }
        {
            std::lock_guard<std::mutex> lock(session->control);
            session->cancel_requested = true;
            session->pause_requested  = false;
            session->changed.notify_all();
        }
        if (session->controller.joinable()) {
            session->controller.join();
        }
        delete session;
    });
}

mr_status mr_session_start(mr_session* session, const mr_scene* scene, const mr_render_settings* render,
                           const mr_integrator_settings* integrator, const mr_session_settings* settings) {
    return guarded([&] {
        require(session != nullptr, "Session handle is null");
        const Scene&           s = scene_of(scene);
        validate_render(render);
        const IntegratorParams p = integrator_params(integrator);
        mr_session_settings    ss{0, 16, 4};
        if (settings) {
            ss = *settings;
        }
        // SessionSettings::validate (src/render/render_session.cpp:192-198).
        if (ss.threads > 32 || ss.tile_size == 0 || ss.tile_size > 128 || ss.batch_samples == 0 ||
            ss.batch_samples > 1024) {
            fail(MR_INVALID_ARGUMENT, "Session requires <=32 threads, tile size in [1,128], batch in [1,1024]");
        }
        {
            std::lock_guard<std::mutex> lock(session->control);
            if (!terminal(session->state)) {
                fail(MR_LOGIC_ERROR, "Render session is still active");
            }
        }
        if (session->controller.joinable()) {
            session->controller.join();
        }
        const size_t pixels = static_cast<size_t>(render->width) * render->height;
        {
            std::lock_guard<std::mutex> lock(session->control);
            session->state            = MR_STATE_PREPARING;
            ++session->job;
            session->total            = pixels * render->samples_per_pixel;
            session->recorded         = 0;
            session->completed_pixels = 0;
            session->pause_requested  = false;
            session->cancel_requested = false;
            session->error.clear();
            session->statistics = {};
            session->started    = std::chrono::steady_clock::now();
            session->finished   = {};
            session->render     = *render;
        }
        {
            std::lock_guard<std::mutex> lock(session->film);
            session->image.assign(3 * pixels, 0.0f);
            session->revision          = 0;
            session->committed_samples = 0;
            session->result.reset();
        }
        MR_CUDA(cudaGetDevice(&session->device));
        session->controller = std::thread(session_run, session, &s, p, *render, ss);
    });
}

mr_status mr_session_pause(mr_session* session, int* accepted) {
    return guarded([&] {
        require(session != nullptr, "Session handle is null");
        std::lock_guard<std::mutex> lock(session->control);
        const bool ok = session->state == MR_STATE_RUNNING;
        if (ok) {
            session->pause_requested = true;
            session->state           = MR_STATE_PAUSING;
        }
        if (accepted) *accepted = ok ? 1 : 0;
    });
}

mr_status mr_session_resume(mr_session* session, int* accepted) {
    return guarded([&] {
        require(session != nullptr, "Session handle is null");
        std::lock_guard<std::mutex> lock(session->control);
        const bool ok = session->state == MR_STATE_PAUSED || session->state == MR_STATE_PAUSING;
        if (ok) {
            session->pause_requested = false;
            session->state           = MR_STATE_RUNNING;
            session->changed.notify_all();
        }
        if (accepted) *accepted = ok ? 1 : 0;
    });
}

mr_status mr_session_cancel(mr_session* session) {
    return guarded([&] {
        require(session != nullptr, "Session handle is null");
        std::lock_guard<std::mutex> lock(session->control);
        if (terminal(session->state)) {
            return;
        }
        session->cancel_requested = true;
        session->pause_requested  = false;
        session->state            = MR_STATE_CANCELLING;
        session->changed.notify_all();
    });
}

mr_status mr_session_wait(mr_session* session) {
    return guarded([&] {
        require(session != nullptr, "Session handle is null");
        if (session->controller.joinable()) {
            session->controller.join();
        }
    });
}

mr_status mr_session_wait_for(mr_session* session, uint32_t milliseconds, int* is_terminal) {
    return guarded([&] {
        require(session != nullptr, "Session handle is null");
        std::unique_lock<std::mutex> lock(session->control);
        const bool done = session->changed.wait_for(lock, std::chrono::milliseconds(milliseconds),
                                                    [&] { return terminal(session->state); });
        if (is_terminal) *is_terminal = done ? 1 : 0;
    });
}

mr_status mr_session_progress(const mr_session* session, mr_render_progress* progress) {
    return guarded([&] {
        require(session != nullptr && progress != nullptr, "Session or output is null");
        auto* s = const_cast<mr_session*>(session);
        std::lock_guard<std::mutex> lock(s->control);
        std::memset(progress, 0, sizeof(*progress));
        progress->state            = s->state;
        progress->job_id           = s->job;
        progress->completed_pixels = s->completed_pixels.load();
        progress->recorded_samples = s->recorded.load();
        progress->total_samples    = s->total;
        progress->worker_count     = s->state == MR_STATE_IDLE ? 0 : 1;
        const auto end = terminal(s->state) ? s->finished : std::chrono::steady_clock::now();
        progress->elapsed_seconds =
            s->state == MR_STATE_IDLE ? 0 : std::chrono::duration<double>(end - s->started).count();
        progress->statistics = s->statistics;
        std::strncpy(progress->error, s->error.c_str(), sizeof(progress->error) - 1);
    });
}

mr_status mr_session_preview(const mr_session* session, uint64_t maximum_dimension, float* rgb,
                             size_t capacity, mr_render_preview* preview) {
    return guarded([&] {
        require(session != nullptr && preview != nullptr, "Session or output is null");
        auto* s = const_cast<mr_session*>(session);
        std::memset(preview, 0, sizeof(*preview));
        {
            std::lock_guard<std::mutex> lock(s->control);
            preview->job_id = s->job;
        }
        std::unique_lock<std::mutex> lock(s->film, std::try_to_lock);
        if (!lock.owns_lock() || s->image.empty()) {
            return;
        }
        // Nearest-pixel downscale of Film::make_image (src/render/render_session.cpp:113-139).
        const uint64_t W = s->render.width, H = s->render.height;
        const double   scale = maximum_dimension
                                   ? std::max(1.0, double(std::max(W, H)) / double(maximum_dimension))
                                   : 1.0;
        const uint64_t w = std::max<uint64_t>(1, uint64_t(double(W) / scale));
        const uint64_t h = std::max<uint64_t>(1, uint64_t(double(H) / scale));
        preview->width  = w;
        preview->height = h;
        preview->revision = s->revision;
        preview->recorded_samples = static_cast<uint64_t>(s->committed_samples) * W * H;
        preview->available = 1;
        if (!rgb) {
            return;
        }
        require(capacity >= 3 * w * h, "Preview buffer is too small");
        for (uint64_t y = 0; y < h; ++y) {
            const uint64_t sy = std::min(H - 1, (y * H + H / 2) / h);
            for (uint64_t x = 0; x < w; ++x) {
                const uint64_t sx = std::min(W - 1, (x * W + W / 2) / w);
                for (int c = 0; c < 3; ++c) {
                    rgb[3 * (y * w + x) + c] = s->image[3 * (sy * W + sx) + c];
                }
            }
        }
    });
}

mr_status mr_session_result(const mr_session* session, float* rgb, size_t capacity, uint64_t* width,
                            uint64_t* height) {
    return guarded([&] {
        require(session != nullptr, "Session handle is null");
        auto* s = const_cast<mr_session*>(session);
        {
            std::lock_guard<std::mutex> lock(s->control);
            if (s->state != MR_STATE_COMPLETED) {
                fail(MR_OUT_OF_RANGE, "Render session has no completed result");
            }
        }
        std::lock_guard<std::mutex> lock(s->film);
        if (width) *width = s->render.width;
        if (height) *height = s->render.height;
        if (rgb) {
            require(s->result && capacity >= s->result->size(), "Result buffer is too small");
            std::memcpy(rgb, s->result->data(), s->result->size() * sizeof(float));
        }
    });
}

}  // extern "C"
