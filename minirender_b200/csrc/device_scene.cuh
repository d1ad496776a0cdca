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

// glm::vec3(object_to_world * glm::vec4(p, 1)) in float with GLM's evaluation order
// (m0*x + m1*y) + (m2*z + m3*w) and no fused operations (src/render/bvh.cpp:68-69). Host and
// device produce identical world vertices; a two-level scene evaluates it during traversal and
// gets the flattened scene's vertices bit for bit.
MR_HD f3 transform_point(const float* m, float x, float y, float z) {
#ifdef __CUDA_ARCH__
    const auto row = [&](int r) {
        return __fadd_rn(__fadd_rn(__fmul_rn(m[r], x), __fmul_rn(m[4 + r], y)),
                         __fadd_rn(__fmul_rn(m[8 + r], z), __fmul_rn(m[12 + r], 1.0f)));
    };
#else
    const auto row = [&](int r) {
        volatile float a = m[r] * x, b = m[4 + r] * y, c = m[8 + r] * z, d = m[12 + r] * 1.0f;
        volatile float ab = a + b, cd = c + d;
        return static_cast<float>(ab + cd);
    };
#endif
    return {row(0), row(1), row(2)};
}

// normalize(normal_to_world * n) of a mesh corner normal (src/render/bvh.cpp:319-320). Every
// operation is rounded explicitly (fused multiply-adds for the product, then a squared length,
// square root and reciprocal with no contraction), so the flattening, which stores these
// normals, and a two-level scene, which evaluates them at each hit in another kernel, get the
// same bits whatever the compiler fuses around them.
__device__ __forceinline__ f3 world_normal(const float* m, const float* n) {
    const f3 w = {fmaf(m[6], n[2], fmaf(m[3], n[1], __fmul_rn(m[0], n[0]))),
                  fmaf(m[7], n[2], fmaf(m[4], n[1], __fmul_rn(m[1], n[0]))),
                  fmaf(m[8], n[2], fmaf(m[5], n[1], __fmul_rn(m[2], n[0])))};
    const float length2 = __fadd_rn(__fadd_rn(__fmul_rn(w.x, w.x), __fmul_rn(w.y, w.y)), __fmul_rn(w.z, w.z));
    const float inverse = __fdiv_rn(1.0f, __fsqrt_rn(length2));
    return {__fmul_rn(w.x, inverse), __fmul_rn(w.y, inverse), __fmul_rn(w.z, inverse)};
}

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
    int      base_texture;    // index into the scene's textures, -1 none
    int      normal_texture;  // index into the scene's textures, -1 none
    uint32_t filter;          // mr_texture_filter
    float    normal_scale;
    uint32_t normal_flip_y;
};

// Level 0 of a texture: width x height texels (linear RGB in xyz) from `offset` of the scene's
// texel array, row 0 at the top of the image.
struct DeviceTexture {
    uint32_t width, height;
    uint64_t offset;
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

// One instance of a two-level scene: where its mesh tree (BLAS) starts, how it maps to world
// space, and the bounds the traversal needs. `to_world` is the column-major object_to_world of
// the snapshot (the flattening's matrix); `to_object` its FP32 inverse affine, row-major 3x4.
struct DeviceInstance2 {
    float    to_world[16];
    float    to_object[12];
    float    normal_to_world[9];
    float    lo[3], hi[3];    // world box of the instance's triangles, grown to cover rounding
    float    margin_static;   // object-space growth of mesh boxes for the world vertices' rounding
    float    a_norm, b_norm;  // infinity norms of to_object's linear part and translation
    int      blas_root;       // >= 0 wide node of blas_nodes, < 0 leaf ~slot of blas_tris
    uint32_t first_prim;      // flat primitive id of the instance's first triangle
    uint32_t position_offset; // into mesh_positions (vertices)
    uint32_t corner_offset;   // into mesh_corners (3 per triangle)
    uint32_t material;
    uint32_t flags;           // kTriSingleSided | kTriMirrored | kTriEmissive | kind << 8
};

// The instance of a two-level scene holding flat primitive `prim` (the last instance whose first
// primitive is at most `prim`).
__device__ __forceinline__ uint32_t find_instance2(const DeviceInstance2* instances, uint32_t count,
                                                   uint32_t prim) {
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&instances[mid].first_prim) <= prim) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

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
    uint32_t              slot_count;       // triangle slots in leaf order (two-level: primitives)
    uint32_t              light_count;
    int                   environment_choice;  // light index of the environment, -1 if none
    f3                    environment;
    int                   medium_count;
    int                   media_scatter;    // any region scatters
    CameraBasis           camera;
    // Two-level scenes (two_level != 0): `nodes` and `root` are the instance-level tree, whose
    // leaves list instance ids in tlas_items (bit 31 marks a leaf's last item); every mesh has
    // its own object-space tree in blas_nodes over object-space triangle slots in blas_tris
    // ([0] = v0.xyz + triangle index within the mesh, [1] = v1.xyz + kTriLeafEnd, [2] = v2.xyz).
    // The meshes' positions and corners stay resident for shading.
    // Textures (any material or the environment uses one): texels, per-texture records, and for
    // flattened scenes the corner UVs of every primitive (3 per primitive, null without textures).
    const float4*          texels;
    const DeviceTexture*   textures;
    const float2*          uvs;
    // Environment map: texture index (-1: constant environment only), strength, rotation about
    // +Y in radians, and its importance distribution over a grid of env_w x env_h texels (a mip
    // level): the row marginal CDF (env_h + 1 entries), each row's conditional CDF (env_w + 1
    // entries per row) and each row's texel solid angle; env_uniform: sample the sphere
    // uniformly (no map, zero strength, or a map without radiance).
    int                    env_texture;
    float                  env_strength, env_rotation;
    int                    env_uniform;
    uint32_t               env_w, env_h;
    const float*           env_row_cdf;
    const float*           env_col_cdf;
    const float*           env_solid_angle;
    int                    two_level;
    uint32_t               instance_count;
    const DeviceInstance2* instances;
    const uint32_t*        tlas_items;
    const float4*          blas_nodes;
    const float4*          blas_tris;
    const float*           mesh_positions;
    const mr_mesh_corner*  mesh_corners;
};

}  // namespace mr
