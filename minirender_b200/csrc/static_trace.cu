// static_trace.cu — mr_trace_paths_static: PathTracer::trace for a bounded batch of paths whose
// working memory is a file-scope device array instead of a cudaMalloc'd workspace.
//
// Some callers cannot allocate device memory while they render: a serving process that
// reserves its whole HBM budget in its own pool at start-up and forbids later allocations, or a
// host loop that must not risk the implicit device synchronisation an allocation can cause.
// This entry point gives them the same per-path results as mr_trace_paths with zero
// allocations: the wavefront's path state, queues, counters and a staging copy of the rays live
// in `g_trace_scratch` (about 4.3 MB, resident on every device that loads the library until the
// process exits). Inputs and outputs stay in the caller's device memory.
//
// The array's device address is resolved once per device with cudaGetSymbolAddress (the name in
// host code is only a host-side stand-in). The first call on a device does this, and with CUDA's
// lazy module loading that lookup is also what loads the module and places the array in device
// memory (which can allocate and synchronise): make that first call a zero-length one (count 0),
// before any stream capture and before the caller's no-allocation phase. The cached address
// belongs to the device's primary context: the entry point must not be used across a
// cudaDeviceReset of that device. Every call reuses the same array, which keeps the previous
// call's contents: counters, statistics and error words are cleared at the start of each call,
// and calls whose GPU work overlaps (several streams or threads at once) race on it.
#include <array>
#include <cmath>
#include <mutex>

#include "errors.hpp"
#include "validation.hpp"
#include "wavefront.cuh"

struct mr_scene {
    std::unique_ptr<mr::Scene> impl;
};

namespace mr {

void copy_path_radiance(Workspace& ws, uint32_t count, float* device_out, cudaStream_t stream);
void set_last_error(const std::string& message);

namespace {

constexpr size_t   kStaticPaths   = MR_STATIC_MAX_PATHS;
constexpr uint32_t kStaticBounces = 129;  // maximum_depth <= 128

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Byte size of the carved regions (same fields as a pooled Workspace, plus ray staging and a
// validation word).
constexpr size_t kScratchBytes =
    align256(kStaticPaths * kPathRecordBytes) + align256(kStaticPaths * kShadowRecordBytes) +
    2 * align256(kStaticPaths * sizeof(uint32_t)) +
    align256(kStaticPaths * kBinCount * sizeof(uint32_t)) + align256(kStaticPaths * sizeof(uint32_t)) +
    align256((kStaticBounces + 2) * sizeof(BounceCounters)) +
    align256(kStatCount * sizeof(unsigned long long)) + align256(sizeof(unsigned)) +
    align256(2 * kStaticPaths * sizeof(float4)) + align256(sizeof(unsigned));

static __device__ __align__(256) unsigned char g_trace_scratch[kScratchBytes];

std::mutex                   setup_mutex;
std::array<unsigned char*, 64> scratch_address{};

unsigned char* device_scratch() {
    int device = 0;
    MR_CUDA(cudaGetDevice(&device));
    require(device >= 0 && device < 64, "Device ordinal out of range");
    std::lock_guard<std::mutex> lock(setup_mutex);
    if (!scratch_address[device]) {
        void* ptr = nullptr;
        MR_CUDA(cudaGetSymbolAddress(&ptr, g_trace_scratch));
        scratch_address[device] = static_cast<unsigned char*>(ptr);
    }
    return scratch_address[device];
}

// Carves the static array into a workspace view (owns nothing: memory stays null).
void carve(unsigned char* base, Workspace& ws, float4*& staging, unsigned*& invalid) {
    size_t offset = 0;
    const auto take = [&](size_t bytes) {
        unsigned char* p = base + offset;
        offset += align256(bytes);
        return p;
    };
    ws.capacity          = kStaticPaths;
    ws.max_bounces       = kStaticBounces;
    ws.memory            = nullptr;
    ws.pixels            = 0;
    ws.accumulator       = nullptr;
    unsigned char* paths = take(kStaticPaths * kPathRecordBytes);
    ws.state.view(paths, take(kStaticPaths * kShadowRecordBytes), false);
    ws.queues.ext[0]     = reinterpret_cast<uint32_t*>(take(kStaticPaths * sizeof(uint32_t)));
    ws.queues.ext[1]     = reinterpret_cast<uint32_t*>(take(kStaticPaths * sizeof(uint32_t)));
    ws.queues.bins       = reinterpret_cast<uint32_t*>(take(kStaticPaths * kBinCount * sizeof(uint32_t)));
    ws.queues.shadow     = reinterpret_cast<uint32_t*>(take(kStaticPaths * sizeof(uint32_t)));
    ws.queues.counters   = reinterpret_cast<BounceCounters*>(take((kStaticBounces + 2) * sizeof(BounceCounters)));
    ws.queues.stats      = reinterpret_cast<unsigned long long*>(take(kStatCount * sizeof(unsigned long long)));
    ws.queues.error      = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
    staging              = reinterpret_cast<float4*>(take(2 * kStaticPaths * sizeof(float4)));
    invalid              = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
    if (offset > kScratchBytes) {
        fail(MR_RUNTIME_ERROR, "Static scratch layout exceeds its array");
    }
}

// RayQuery / RayInterval validation (src/render/intersection.cpp:22-26,52-61) on the device,
// plus the copy into the wave's ray records. The unit-length check evaluates the squared length
// in FP64 with the host check's operation order (validate_ray in abi.cu), so this entry point
// rejects exactly the rays mr_trace_paths rejects; no path arithmetic uses FP64.
__global__ void stage_rays_kernel(const mr_ray* rays, uint32_t count, float4* staging,
                                  unsigned* invalid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) {
        return;
    }
    const mr_ray r = rays[i];
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
        ok = ok && isfinite(r.origin[a]) && isfinite(r.direction[a]);
    }
    const double x = r.direction[0], y = r.direction[1], z = r.direction[2];
    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
    ok = ok && fabs(d2 - 1.0) <= 1e-4 && isfinite(r.minimum) && r.minimum >= 0 &&
         !isnan(r.maximum) && r.maximum >= r.minimum;
    if (!ok) {
        atomicOr(invalid, 1u);
    }
    staging[2 * i]     = make_float4(r.origin[0], r.origin[1], r.origin[2], r.minimum);
    staging[2 * i + 1] = make_float4(r.direction[0], r.direction[1], r.direction[2], r.maximum);
}

// check_radiance (src/render/path_tracer.cpp:22-26) on the caller's output.
__global__ void check_output_kernel(const float* radiance, uint32_t count, unsigned* error) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 3 * count) {
        const float v = radiance[i];
        if (!isfinite(v) || v < 0) {
            atomicOr(error, kErrorRadiance);
        }
    }
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" mr_status mr_trace_paths_static(const mr_scene* scene,
                                           const mr_integrator_settings* integrator,
                                           const mr_ray* device_rays, const uint64_t* device_keys,
                                           size_t count, float* device_radiance, void* stream) {
    try {
        require(scene != nullptr && scene->impl != nullptr, "Scene handle is null");
        const IntegratorParams p = integrator_params(integrator);
        if (count > kStaticPaths) {
            fail(MR_INVALID_ARGUMENT,
                 "mr_trace_paths_static takes at most MR_STATIC_MAX_PATHS (16384) paths per call");
        }
        // Resolved before the zero-length return, so a call with count 0 is the warm-up.
        unsigned char* base = device_scratch();
        if (count == 0) {
            return MR_OK;
        }
        require(device_rays && device_keys && device_radiance, "Path buffers are null");
        cudaStream_t   s    = static_cast<cudaStream_t>(stream);
        Workspace      ws;
        float4*        staging = nullptr;
        unsigned*      invalid = nullptr;
        carve(base, ws, staging, invalid);
        const uint32_t n = static_cast<uint32_t>(count);
        MR_CUDA(cudaMemsetAsync(invalid, 0, sizeof(unsigned), s));
        stage_rays_kernel<<<(n + 127) / 128, 128, 0, s>>>(device_rays, n, staging, invalid);
        MR_CUDA(cudaGetLastError());
        unsigned bad = 0;
        MR_CUDA(cudaMemcpyAsync(&bad, invalid, sizeof(bad), cudaMemcpyDeviceToHost, s));
        MR_CUDA(cudaStreamSynchronize(s));
        if (bad) {
            fail(MR_INVALID_ARGUMENT,
                 "Ray origin and direction must be finite, direction of unit length, and "
                 "0 <= minimum <= maximum");
        }
        reset_statistics(ws, s);
        WaveInit init{};
        init.kind  = kInitRays;
        init.rays  = staging;
        init.keys  = device_keys;
        init.count = n;
        Engine::run_wave(*scene->impl, p, init, ws, s);
        copy_path_radiance(ws, n, device_radiance, s);
        check_output_kernel<<<(3 * n + 255) / 256, 256, 0, s>>>(device_radiance, n, ws.queues.error);
        MR_CUDA(cudaGetLastError());
        unsigned error = 0;
        read_statistics(ws, s, nullptr, &error);
        std::string     message;
        const mr_status status = error_status(error, message);
        if (status != MR_OK) {
            fail(status, message);
        }
        return MR_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return MR_RUNTIME_ERROR;
    }
}
