// instancing.cuh — host side of two-level scenes (instancing.cu).
#pragma once

#include <memory>
#include <vector>

#include "scene.cuh"

namespace mr {

// One mesh's object-space tree: the binary tree (kept for refit), its wide nodes' place in the
// shared node array and the binary children each wide node was collapsed from.
struct MeshTree {
    uint32_t                  triangles = 0, positions = 0;
    DeviceBuffer<mr_bvh_node> nodes;
    DeviceBuffer<uint32_t>    order;
    DeviceBuffer<int4>        wide_children;
    uint32_t                  node_count = 0, wide_count = 0, node_base = 0, slot_base = 0;
    uint64_t                  leaves = 0, depth = 0;
    int                       root   = 0;   // ref in the shared arrays (node, or ~slot for a leaf)
    float                     box[6] = {};  // object-space root box (lo, hi)
};

struct TwoLevel {
    DeviceBuffer<float>          positions;  // every mesh's positions, resident for shading
    DeviceBuffer<mr_mesh_corner> corners;
    std::vector<uint32_t>        position_offset, corner_offset;  // per mesh
    std::vector<uint8_t>         used, emissive_mesh;             // per mesh
    std::vector<MeshTree>        mesh;
    DeviceBuffer<float4>         blas_nodes, blas_tris;
    std::vector<DeviceInstance2> host_instances;
    std::vector<uint32_t>        instance_mesh, instance_material;
    DeviceBuffer<DeviceInstance2> instances;
    DeviceBuffer<float4>         tlas_nodes;
    DeviceBuffer<uint32_t>       tlas_items;
    uint32_t                     tlas_node_count = 0;
    uint64_t                     tlas_depth      = 0;
    float                        world_lo[3] = {}, world_hi[3] = {};  // exact world bounds
};

// Transform fields of an instance record (matrices, FP32 inverse affine, norms).
void fill_instance_transform(const mr_instance& in, DeviceInstance2& d);
// Builds every used mesh's tree and the shared node and slot arrays.
void build_mesh_trees(Scene& scene, const mr_scene_desc& desc, cudaStream_t stream);
void write_mesh_tree(Scene& scene, uint32_t mesh, const WideTree& wide, cudaStream_t stream);
// Instance boxes, validation and exact bounds of every instance triangle, the instance tree.
void build_instance_tree(Scene& scene, cudaStream_t stream);
// Points the device view at the two-level arrays; statistics and device bytes.
void publish_two_level(Scene& scene);
void update_instances(Scene& scene, uint32_t first, uint32_t count, const mr_instance* instances);
void update_mesh(Scene& scene, uint32_t mesh, const float* positions, uint32_t position_count);
void rebuild_after_refit(Scene& scene);

}  // namespace mr
