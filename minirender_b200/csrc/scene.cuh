// scene.cuh — host-side scene object behind the opaque mr_scene handle.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "device_scene.cuh"
#include "errors.hpp"

namespace mr {

// The library's stream-ordered device memory pool of the current device (created on first use;
// keeps up to 2 GB of freed memory for reuse).
cudaMemPool_t library_pool();

// While an AllocationScope is alive on a thread, DeviceBuffers allocated on that thread come from
// the library pool, ordered on the scope's stream, and those released inside the same scope are
// freed ordered on it too: no device-wide synchronisation, so scene construction can run beside
// rendering and beside other constructions. Buffers that outlive the scope are freed with
// cudaFree later. Outside any scope DeviceBuffer uses cudaMalloc/cudaFree.
struct AllocationScope {
    static inline thread_local cudaStream_t current    = nullptr;
    static inline thread_local uint64_t     current_id = 0;
    static inline thread_local uint64_t     next_id    = 0;
    cudaStream_t previous;
    uint64_t     previous_id;
    explicit AllocationScope(cudaStream_t stream) : previous(current), previous_id(current_id) {
        current    = stream;
        current_id = ++next_id;
    }
    ~AllocationScope() {
        current    = previous;
        current_id = previous_id;
    }
    AllocationScope(const AllocationScope&)            = delete;
    AllocationScope& operator=(const AllocationScope&) = delete;
};

// Owning device allocation, movable only.
template <typename T> struct DeviceBuffer {
    T*       ptr   = nullptr;
    size_t   count = 0;
    uint64_t scope = 0;  // AllocationScope id of a pooled allocation, 0 for cudaMalloc
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), count(o.count), scope(o.scope) {
        o.ptr   = nullptr;
        o.count = 0;
        o.scope = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        release();
        ptr     = o.ptr;
        count   = o.count;
        scope   = o.scope;
        o.ptr   = nullptr;
        o.count = 0;
        o.scope = 0;
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) {
            if (scope != 0 && scope == AllocationScope::current_id) {
                cudaFreeAsync(ptr, AllocationScope::current);
            } else {
                cudaFree(ptr);
            }
            ptr   = nullptr;
            count = 0;
            scope = 0;
        }
    }
    void allocate(size_t n) {  // throws Error (MR_OUT_OF_MEMORY / MR_CUDA_ERROR)
        release();
        if (n == 0) {
            return;
        }
        if (AllocationScope::current_id != 0) {
            MR_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ptr), n * sizeof(T), library_pool(),
                                            AllocationScope::current));
            scope = AllocationScope::current_id;
        } else {
            MR_CUDA(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)));
        }
        count = n;
    }
    size_t bytes() const { return count * sizeof(T); }
};

struct TwoLevel;

// Host copy of the light table: area lights and their fixed weights, directional lights and the
// environment, whose weights scale with the scene's projected area (LightSampler's constructor,
// src/render/light.cpp:197-264).
struct LightTable {
    std::vector<DeviceLight> lights;
    std::vector<float>       weights;      // area lights: final; others: per unit projected area
    std::vector<uint8_t>     scales;       // 1 where the weight scales with the projected area
};

struct Scene {
    int         device = 0;
    DeviceScene d{};
    std::unique_ptr<TwoLevel, void (*)(TwoLevel*)> two{nullptr, nullptr};  // two-level scenes only
    LightTable                                     light_table;

    DeviceBuffer<float4>         nodes;
    DeviceBuffer<float4>         tris;
    DeviceBuffer<float4>         shading;
    DeviceBuffer<DeviceMaterial> materials;
    DeviceBuffer<DeviceLight>    lights;
    DeviceBuffer<float>          light_cdf;
    DeviceBuffer<uint32_t>       prim_emitter;
    DeviceBuffer<DeviceMedium>   media;
    DeviceBuffer<float4>         texels;
    DeviceBuffer<DeviceTexture>  texture_table;
    DeviceBuffer<float2>         uvs;  // flattened scenes with textures: corner UVs per primitive
    DeviceBuffer<float>          env_row_cdf, env_col_cdf, env_solid_angle;

    // Reference-layout BVH (mr_bvh_node + order) kept on the device for export and SAH.
    DeviceBuffer<mr_bvh_node> ref_nodes;
    DeviceBuffer<uint32_t>    ref_order;
    mr_bvh_statistics        statistics{};
    uint32_t                 references    = 0;  // leaf slots; above the triangle count when split
    double                   build_seconds = 0;
    double                   sah_cost      = 0;
    size_t                   device_bytes  = 0;
};

// Wide (4-child) traversal nodes collapsed from a binary tree, with the binary children each
// wide node was made from (for refit) and the root's reference and box.
struct WideTree {
    DeviceBuffer<float4> nodes;
    DeviceBuffer<int4>   children;
    uint32_t             count      = 0;
    uint32_t             root_count = 0;  // primitives when the root is a leaf (then no nodes)
    float                lo[3] = {}, hi[3] = {};
};
WideTree collapse_tree(const mr_bvh_node* nodes, uint32_t node_count, cudaStream_t stream);
// Sets kTriLeafEnd on the last triangle slot of every leaf of a binary tree.
void mark_leaf_ends(const mr_bvh_node* nodes, uint32_t node_count, float4* tris, cudaStream_t stream);
float determinant3(const float* m);
// Validates and uploads the scene's textures (environment.cu).
void upload_textures(Scene& scene, const mr_scene_desc& desc, cudaStream_t stream);
// The environment map's device fields and importance distribution; returns the map's luminance
// integral (strength x the integral over level 0) for light selection (environment.cu).
double prepare_environment(Scene& scene, const mr_scene_desc& desc, cudaStream_t stream);
// Uploads the light table weighted by the projected area of the world bounds [lo, hi].
void upload_light_table(Scene& scene, const float* lo, const float* hi, cudaStream_t stream);

// Scene construction (scene.cu). `build` (optional) selects split references for the builder.
std::unique_ptr<Scene> create_scene(const mr_scene_desc& desc, const mr_bvh_desc* bvh,
                                    const mr_build_settings* build = nullptr);

// Early split clipping (split.cu): references (bounds, centroid, triangle) of the triangles,
// oversized ones entered once per nonempty cell of a grid over their box. count == 0 when no
// triangle is worth splitting (build over the triangles themselves).
struct SplitReferences {
    DeviceBuffer<float4>   lo, hi, centroid;
    DeviceBuffer<uint32_t> prim;
    uint32_t               count = 0;
};
SplitReferences split_references(const float4* world, const float4* lo, const float4* hi, uint32_t prims,
                                  float factor, uint64_t max_references, cudaStream_t stream);
// Replaces the reference indices of a built leaf order by their triangles.
void map_order_to_primitives(uint32_t* order, const uint32_t* prim, uint32_t count, cudaStream_t stream);

// GPU binned-SAH builder (builder.cu): from per-primitive FP32 bounds and centroids on the
// device to a reference-layout tree (DFS-independent node numbering, root at index 0).
struct BuildResult {
    DeviceBuffer<mr_bvh_node> nodes;
    DeviceBuffer<uint32_t>    order;
    uint32_t                  node_count    = 0;
    uint64_t                  leaves        = 0;
    uint64_t                  maximum_depth = 0;
    double                    seconds       = 0;
};
BuildResult build_bvh_device(const float4* lo, const float4* hi, const float4* centroid,
                             uint32_t count, cudaStream_t stream);

}  // namespace mr
