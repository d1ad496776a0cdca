// device_scene.cuh — the scene as it lives in HBM.
//
// Traversal data and shading data are separate streams, each an array of 16-byte records:
//  - nodes:  8 float4 (128 B, one cache line) per 4-wide node collapsed from the binary SAH
//            tree. One fetch serves up to four slab tests, so a ray needs about half as many
//            dependent node fetches as on the binary tree.
//              [0..5] = lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of children 0..3 (x4 vectors;
//                       unused children hold an empty box)
//              [6]    = child refs (int bits): >= 0 wide node index; < 0 leaf whose triangles
//                       occupy slots ~ref .. the slot flagged kTriLeafEnd
//              [7].x  = number of children (int bits)
//  - tris:   3 float4 per triangle slot, in leaf order (no index indirection during traversal):
//              [0] = v0.xyz, flat primitive id (uint bits)
//              [1] = v1.xyz, flags (uint bits: kTriSingleSided | kTriMirrored | kind << 8)
//              [2] = v2.xyz, 0
//  - shading (per primitive, primitive order): 3 float4 = world-space unit corner normals
//            (normalize(normal_to_world * n), src/render/bvh.cpp:319-320) with
//            w = instance index, triangle index, material index (uint bits).
//  - materials, lights and the camera basis are small tables.
#pragma once

#include "common.cuh"

namespace mr {

enum TriFlags : unsigned {
    kTriSingleSided = 1u,
    kTriMirrored    = 2u,
    kTriEmissive    = 4u,
    kTriLeafEnd     = 8u,  // last triangle of its leaf in the triangle stream
};

struct DeviceMaterial {
    f3       base_color;
    f3       emission;
    float    alpha;  // roughness^2 (src/render/bsdf.cpp:125)
    float    ior;
    uint32_t kind;
    uint32_t double_sided;
};

enum LightKindCode : uint32_t { kLightArea = 0, kLightDirectional = 1, kLightEnvironment = 2 };

struct DeviceLight {
    f3       v0, v1, v2;   // area: world vertices
    f3       normal;       // area: unit normal (mirrored-aware); directional: -direction
    f3       radiance;
    float    area;
    uint32_t kind;
    uint32_t double_sided;
};

struct DeviceMedium {
    f3    minimum, maximum;
    f3    absorption, scattering, extinction;
    float anisotropy;
    int   scatters;  // any scattering coefficient nonzero
    int   enabled;
};

constexpr int kMaxMedia = 32;  // maximum_medium_regions (include/minirender/scene/medium.hpp:43)

struct CameraBasis {
    f3    position;
    f3    forward, right, up;
    float half_height;
    float near_plane, far_plane;
    float aperture_radius, focus_distance;
};

struct DeviceScene {
    const float4*         nodes;
    const float4*         tris;
    const float4*         shading;
    const DeviceMaterial* materials;
    const DeviceLight*    lights;
    const float*          light_cdf;        // light_count + 1 entries
    const uint32_t*       prim_emitter;     // primitive -> light choice index, kNone if none
    const DeviceMedium*   media;
    int                   root;             // root ref (node index, or ~slot for a lone leaf)
    uint32_t              root_count;       // triangle count when the root is a leaf
    float                 root_lo[3], root_hi[3];
    int                   has_nodes;        // 0 for an empty scene
    uint32_t              node_count;
    uint32_t              primitive_count;
    uint32_t              light_count;
    int                   environment_choice;  // light index of the environment, -1 if none
    f3                    environment;
    int                   medium_count;
    int                   media_scatter;    // any region scatters
    CameraBasis           camera;
};

}  // namespace mr
