// scene.cu — validation, upload and device layout of a scene snapshot.
//
// Follows the reference's PathTracer construction (src/render/path_tracer.cpp:111-120):
// snapshot validation (src/scene/scene.cpp:38-66,141-155,241-267; src/scene/medium.cpp:31-65),
// world-space triangle flattening (src/render/bvh.cpp:31-99), BVH, light table
// (src/render/light.cpp:197-264) and media. All arithmetic is FP32; the flattening uses
// explicit unfused multiply/add so host and device produce identical world vertices.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>

#include "errors.hpp"
#include "instancing.cuh"
#include "scan.cuh"
#include "scene.cuh"

namespace mr {

namespace {

struct DeviceInstance {
    float    object_to_world[16];
    float    normal_to_world[9];
    uint32_t position_offset;
    uint32_t corner_offset;  // in corners (3 per triangle)
    uint32_t first_prim;
    uint32_t triangle_count;
    uint32_t material;
    uint32_t flags;  // kTriSingleSided | kTriMirrored | kTriEmissive | kind << 8
};

__device__ __forceinline__ uint32_t find_instance(const DeviceInstance* instances, uint32_t count,
                                                  uint32_t prim) {
    uint32_t lo = 0, hi = count;  // last instance with first_prim <= prim
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (instances[mid].first_prim <= prim) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// One thread per primitive: world vertices, build bounds/centroid, shading normals, flags.
__global__ void flatten_kernel(const float* positions, const mr_mesh_corner* corners,
                               const DeviceInstance* instances, uint32_t instance_count,
                               uint32_t prim_count, float4* world, float4* shading, float4* lo,
                               float4* hi, float4* centroid, unsigned* error, float2* uvs) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prim_count) {
        return;
    }
    const uint32_t        ii   = find_instance(instances, instance_count, p);
    const DeviceInstance& inst = instances[ii];
    const uint32_t        tri  = p - inst.first_prim;
    f3                    v[3];
    f3                    n[3];
    for (int c = 0; c < 3; ++c) {
        const mr_mesh_corner& corner = corners[inst.corner_offset + 3 * tri + c];
        const float*          q      = positions + 3 * (static_cast<size_t>(inst.position_offset) + corner.position);
        v[c] = transform_point(inst.object_to_world, q[0], q[1], q[2]);
        n[c] = world_normal(inst.normal_to_world, corner.normal);
        if (uvs) {
            uvs[3 * static_cast<size_t>(p) + c] = make_float2(corner.uv[0], corner.uv[1]);
        }
    }
    if (!finite3(v[0]) || !finite3(v[1]) || !finite3(v[2])) {
        atomicOr(error, 1u);
    }
    const f3 e1 = v[1] - v[0], e2 = v[2] - v[0];
    const f3 cr = {difference_of_products(e1.y, e2.z, e2.y, e1.z),
                   difference_of_products(e1.z, e2.x, e2.z, e1.x),
                   difference_of_products(e1.x, e2.y, e2.x, e1.y)};
    if (cr.x == 0 && cr.y == 0 && cr.z == 0) {
        atomicOr(error, 2u);
    }
    world[3 * p + 0] = f4(v[0], __uint_as_float(p));
    world[3 * p + 1] = f4(v[1], __uint_as_float(inst.flags));
    world[3 * p + 2] = f4(v[2], 0.0f);
    shading[3 * p + 0] = f4(n[0], __uint_as_float(ii));
    shading[3 * p + 1] = f4(n[1], __uint_as_float(tri));
    shading[3 * p + 2] = f4(n[2], __uint_as_float(inst.material));
    const f3 mn = {fminf(fminf(v[0].x, v[1].x), v[2].x), fminf(fminf(v[0].y, v[1].y), v[2].y),
                   fminf(fminf(v[0].z, v[1].z), v[2].z)};
    const f3 mx = {fmaxf(fmaxf(v[0].x, v[1].x), v[2].x), fmaxf(fmaxf(v[0].y, v[1].y), v[2].y),
                   fmaxf(fmaxf(v[0].z, v[1].z), v[2].z)};
    lo[p] = f4(mn, 0.0f);
    hi[p] = f4(mx, 0.0f);
    // Centroid as the reference accumulates it: ((v0/3) + v1/3) + v2/3.
    const f3 third = {((v[0].x / 3.0f) + v[1].x / 3.0f) + v[2].x / 3.0f,
                      ((v[0].y / 3.0f) + v[1].y / 3.0f) + v[2].y / 3.0f,
                      ((v[0].z / 3.0f) + v[1].z / 3.0f) + v[2].z / 3.0f};
    centroid[p] = f4(third, 0.0f);
}

// Collapse of the binary tree (reference layout) into 4-wide traversal nodes, one level of wide
// nodes per launch pair. A wide node starts from a binary interior node's two children and
// repeatedly opens the interior child with the largest surface area until it has four children
// or only leaves remain.
__device__ __forceinline__ float node_area(const mr_bvh_node& n) {
    const float ex = n.maximum[0] - n.minimum[0], ey = n.maximum[1] - n.minimum[1],
                ez = n.maximum[2] - n.minimum[2];
    return ex * ey + ey * ez + ez * ex;
}

__global__ void collapse_count_kernel(const mr_bvh_node* nodes, const uint32_t* roots, uint32_t count,
                                      int4* children, uint32_t* interior_counts) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) {
        return;
    }
    const mr_bvh_node& root = nodes[roots[k]];
    int c[4] = {static_cast<int>(root.first), static_cast<int>(root.right), -1, -1};
    int n    = 2;
    while (n < 4) {
        int   best = -1;
        float area = -1.0f;
        for (int i = 0; i < n; ++i) {
            const mr_bvh_node& child = nodes[c[i]];
            if (child.count == 0 && node_area(child) > area) {
                area = node_area(child);
                best = i;
            }
        }
        if (best < 0) {
            break;
        }
        const mr_bvh_node& open = nodes[c[best]];
        c[best]  = static_cast<int>(open.first);
        c[n++]   = static_cast<int>(open.right);
    }
    uint32_t interior = 0;
    for (int i = 0; i < n; ++i) {
        interior += nodes[c[i]].count == 0 ? 1u : 0u;
    }
    children[k]        = make_int4(c[0], c[1], c[2], c[3]);
    interior_counts[k] = interior;
}

// Writes wide node `base + k`: children's boxes as six x4 vectors, refs, child count.
__global__ void collapse_write_kernel(const mr_bvh_node* nodes, const int4* children, uint32_t count,
                                      const uint32_t* offsets, uint32_t base, uint32_t next_base,
                                      float4* wide, uint32_t* next_roots) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) {
        return;
    }
    const int4 c4   = children[k];
    const int  c[4] = {c4.x, c4.y, c4.z, c4.w};
    float      lo[3][4], hi[3][4];
    int        ref[4];
    int        valid = 0;
    uint32_t   rank  = 0;
    for (int i = 0; i < 4; ++i) {
        if (c[i] < 0) {
            for (int a = 0; a < 3; ++a) {
                lo[a][i] = INFINITY;  // empty box: every slab test misses
                hi[a][i] = -INFINITY;
            }
            ref[i] = 0;
            continue;
        }
        const mr_bvh_node& n = nodes[c[i]];
        for (int a = 0; a < 3; ++a) {
            lo[a][i] = n.minimum[a];
            hi[a][i] = n.maximum[a];
        }
        if (n.count == 0) {
            const uint32_t slot = offsets[k] + rank++;
            next_roots[slot]    = static_cast<uint32_t>(c[i]);
            ref[i]              = static_cast<int>(next_base + slot);
        } else {
            ref[i] = ~static_cast<int>(n.first);
        }
        ++valid;
    }
    float4* o = wide + 8 * static_cast<size_t>(base + k);
    for (int a = 0; a < 3; ++a) {
        o[2 * a]     = make_float4(lo[a][0], lo[a][1], lo[a][2], lo[a][3]);
        o[2 * a + 1] = make_float4(hi[a][0], hi[a][1], hi[a][2], hi[a][3]);
    }
    o[6] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(ref[2]),
                       __int_as_float(ref[3]));
    o[7] = make_float4(__int_as_float(valid), 0.0f, 0.0f, 0.0f);
}

__global__ void interior_count_kernel(const mr_bvh_node* nodes, uint32_t count, uint32_t* total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned m = __ballot_sync(0xffffffffu, i < count && nodes[i].count == 0);
    if ((threadIdx.x & 31) == 0 && m) {
        atomicAdd(total, static_cast<uint32_t>(__popc(m)));
    }
}

// Triangle stream in leaf order; marks the last slot of every leaf.
__global__ void gather_triangles_kernel(const float4* world, const uint32_t* order, uint32_t count,
                                        float4* tris) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= count) {
        return;
    }
    const uint32_t p = order[slot];
    tris[3 * slot + 0] = world[3 * p + 0];
    tris[3 * slot + 1] = world[3 * p + 1];
    tris[3 * slot + 2] = world[3 * p + 2];
}

__global__ void mark_leaf_end_kernel(const mr_bvh_node* nodes, uint32_t count, float4* tris) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count || nodes[i].count == 0) {
        return;
    }
    float4& t = tris[3 * static_cast<size_t>(nodes[i].first + nodes[i].count - 1) + 1];
    t.w       = __uint_as_float(__float_as_uint(t.w) | kTriLeafEnd);
}

bool finite3h(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

float luminance(f3 c) { return (c.x * 0.2126f + c.y * 0.7152f) + c.z * 0.0722f; }

// Camera::validate (src/scene/scene.cpp:141-155).
void validate_camera(const mr_camera& c) {
    require(finite3h(c.position) && finite3h(c.target) && finite3h(c.up),
            "Camera vectors must be finite");
    const f3 p = {c.position[0], c.position[1], c.position[2]};
    const f3 t = {c.target[0], c.target[1], c.target[2]};
    const f3 u = {c.up[0], c.up[1], c.up[2]};
    require(length(t - p) > 1e-6f, "Camera position and target must differ");
    require(length(cross(t - p, u)) > 1e-6f, "Camera up must not be parallel to view direction");
    require(std::isfinite(c.vertical_fov_degrees) && c.vertical_fov_degrees > 0 &&
                c.vertical_fov_degrees < 179,
            "Camera FOV must be between 0 and 179 degrees");
    require(std::isfinite(c.near_plane) && std::isfinite(c.far_plane) && c.near_plane > 0 &&
                c.far_plane > c.near_plane,
            "Camera clipping planes must satisfy 0 < near < far");
    require(std::isfinite(c.aperture_radius) && c.aperture_radius >= 0 &&
                std::isfinite(c.focus_distance) && c.focus_distance > 0,
            "Camera lens requires nonnegative aperture and positive focus distance");
}

// Material::validate (src/scene/scene.cpp:241-267) for the supported kinds.
void validate_material(const mr_material& m) {
    require(finite3h(m.base_color) && m.base_color[0] >= 0 && m.base_color[1] >= 0 &&
                m.base_color[2] >= 0 && m.base_color[0] <= 1 && m.base_color[1] <= 1 &&
                m.base_color[2] <= 1,
            "Material base color must be in [0,1]");
    require(finite3h(m.emission) && m.emission[0] >= 0 && m.emission[1] >= 0 && m.emission[2] >= 0,
            "Material emission must be nonnegative");
    require(std::isfinite(m.roughness) && m.roughness >= 0 && m.roughness <= 1,
            "Roughness must be in [0,1]");
    require(std::isfinite(m.ior) && m.ior > 0, "IOR must be positive");
    require(m.kind <= MR_MATERIAL_SUBSURFACE, "Invalid material kind");
    require(m.kind <= MR_MATERIAL_DIELECTRIC,
            "Cloth and subsurface materials are not supported by the GPU path tracer");
}

// MeshData::validate (src/scene/scene.cpp:38-66).
void validate_mesh(const mr_mesh& m) {
    require(m.position_count > 0 && m.triangle_count > 0 && m.positions && m.corners,
            "Mesh must contain positions and triangles");
    for (uint32_t i = 0; i < m.position_count; ++i) {
        require(finite3h(m.positions + 3 * i), "Mesh position must be finite");
    }
    for (uint32_t t = 0; t < m.triangle_count; ++t) {
        for (int c = 0; c < 3; ++c) {
            const mr_mesh_corner& k = m.corners[3 * t + c];
            require(k.position < m.position_count, "Mesh position index is out of range");
            const f3 n = {k.normal[0], k.normal[1], k.normal[2]};
            require(finite3(n) && dot(n, n) > 1e-12f, "Mesh normal must be finite and nonzero");
            require(std::isfinite(k.uv[0]) && std::isfinite(k.uv[1]), "Mesh UV must be finite");
        }
        const float* a = m.positions + 3 * m.corners[3 * t].position;
        const float* b = m.positions + 3 * m.corners[3 * t + 1].position;
        const float* c = m.positions + 3 * m.corners[3 * t + 2].position;
        const f3 e1 = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const f3 e2 = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        const f3 area = cross(e1, e2);
        require(dot(area, area) > 1e-20f, "Degenerate mesh triangle");
    }
}

// MediumRegion / validate_medium_regions (src/scene/medium.cpp:31-65).
void validate_media(const mr_medium_region* media, uint32_t count) {
    require(count <= kMaxMedia, "Scene supports at most 32 medium regions");
    for (uint32_t i = 0; i < count; ++i) {
        const auto& r = media[i];
        bool ok = true;
        for (int a = 0; a < 3; ++a) {
            const double e = r.absorption[a] + r.scattering[a];
            ok = ok && std::isfinite(r.absorption[a]) && std::isfinite(r.scattering[a]) &&
                 std::isfinite(e) && r.absorption[a] >= 0 && r.scattering[a] >= 0;
        }
        require(ok && std::isfinite(r.anisotropy) && std::fabs(r.anisotropy) < 1,
                "Medium coefficients must be finite/nonnegative and |g| < 1");
        bool box = true;
        for (int a = 0; a < 3; ++a) {
            box = box && std::isfinite(r.minimum[a]) && std::isfinite(r.maximum[a]) &&
                  std::isfinite(r.maximum[a] - r.minimum[a]) && r.minimum[a] < r.maximum[a];
        }
        require(box, "Medium region requires an ID and a finite positive box");
        if (!r.enabled) {
            continue;
        }
        for (uint32_t j = 0; j < i; ++j) {
            const auto& o = media[j];
            if (!o.enabled) {
                continue;
            }
            bool overlap = true;
            for (int a = 0; a < 3; ++a) {
                overlap = overlap && std::max(r.minimum[a], o.minimum[a]) < std::min(r.maximum[a], o.maximum[a]);
            }
            require(!overlap, "Medium region interiors overlap");
        }
    }
}


void validate_imported(const mr_bvh_desc& b, uint32_t prims) {
    require(b.primitive_count == prims, "Imported BVH primitive count differs from the scene");
    require(prims == 0 || (b.node_count > 0 && b.nodes && b.order),
            "Imported BVH has no nodes");
    std::vector<uint8_t> seen(prims, 0);
    for (uint32_t i = 0; i < prims; ++i) {
        require(b.order[i] < prims && !seen[b.order[i]], "Imported BVH order is not a permutation");
        seen[b.order[i]] = 1;
    }
    std::vector<uint32_t> covered(prims, 0);
    for (uint32_t i = 0; i < b.node_count; ++i) {
        const auto& n = b.nodes[i];
        if (n.count) {
            require(uint64_t(n.first) + n.count <= prims, "Imported BVH leaf range is out of range");
            for (uint32_t k = n.first; k < n.first + n.count; ++k) {
                covered[k]++;
            }
        } else {
            require(n.first < b.node_count && n.right < b.node_count && n.first != i &&
                        n.right != i,
                    "Imported BVH child index is out of range");
        }
    }
    for (uint32_t k = 0; k < prims; ++k) {
        require(covered[k] == 1, "Imported BVH leaves do not cover every slot exactly once");
    }
}

}  // namespace

float determinant3(const float* m) {
    const auto e = [m](int c, int r) { return m[4 * c + r]; };
    return e(0, 0) * (e(1, 1) * e(2, 2) - e(2, 1) * e(1, 2)) -
           e(1, 0) * (e(0, 1) * e(2, 2) - e(2, 1) * e(0, 2)) +
           e(2, 0) * (e(0, 1) * e(1, 2) - e(1, 1) * e(0, 2));
}

WideTree collapse_tree(const mr_bvh_node* ref_nodes, uint32_t node_count, cudaStream_t stream) {
    WideTree out;
    if (node_count == 0) {
        return out;
    }
    mr_bvh_node root{};
    MR_CUDA(cudaMemcpyAsync(&root, ref_nodes, sizeof(root), cudaMemcpyDeviceToHost, stream));
    DeviceBuffer<uint32_t> total;
    total.allocate(1);
    MR_CUDA(cudaMemsetAsync(total.ptr, 0, sizeof(uint32_t), stream));
    interior_count_kernel<<<(node_count + 255) / 256, 256, 0, stream>>>(ref_nodes, node_count, total.ptr);
    uint32_t interior = 0;
    MR_CUDA(cudaMemcpyAsync(&interior, total.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    for (int a = 0; a < 3; ++a) {
        out.lo[a] = root.minimum[a];
        out.hi[a] = root.maximum[a];
    }
    out.root_count = root.count;
    out.nodes.allocate(std::max<uint32_t>(1, interior) * 8ull);
    out.children.allocate(std::max<uint32_t>(1, interior));
    if (interior == 0) {
        return out;
    }
    DeviceBuffer<uint32_t> roots[2], counts, offsets, scratch;
    roots[0].allocate(interior);
    roots[1].allocate(interior);
    counts.allocate(interior);
    offsets.allocate(interior);
    scratch.allocate(scan_scratch_size(interior));
    MR_CUDA(cudaMemsetAsync(roots[0].ptr, 0, sizeof(uint32_t), stream));  // the root
    uint32_t level = 1, base = 0, cur = 0;
    while (level > 0) {
        int4* children = out.children.ptr + base;
        collapse_count_kernel<<<(level + 127) / 128, 128, 0, stream>>>(ref_nodes, roots[cur].ptr, level,
                                                                       children, counts.ptr);
        exclusive_scan(counts.ptr, offsets.ptr, level, scratch.ptr, total.ptr, stream);
        collapse_write_kernel<<<(level + 127) / 128, 128, 0, stream>>>(
            ref_nodes, children, level, offsets.ptr, base, base + level, out.nodes.ptr, roots[cur ^ 1].ptr);
        uint32_t next = 0;
        MR_CUDA(cudaMemcpyAsync(&next, total.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        base += level;
        level = next;
        cur ^= 1;
    }
    out.count = base;
    return out;
}

void mark_leaf_ends(const mr_bvh_node* nodes, uint32_t node_count, float4* tris, cudaStream_t stream) {
    if (node_count) {
        mark_leaf_end_kernel<<<(node_count + 255) / 256, 256, 0, stream>>>(nodes, node_count, tris);
        MR_CUDA(cudaGetLastError());
    }
}

// DiscreteDistribution (src/core/sampling.cpp:109-127) in FP32 over the light weights, the
// directional and environment weights scaled by the projected area of the world bounds.
void upload_light_table(Scene& scene, const float* lo, const float* hi, cudaStream_t stream) {
    const LightTable& t = scene.light_table;
    float projected_area = kPi;
    if (scene.d.primitive_count) {
        const f3 extent = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
        projected_area  = kPi * std::max(dot(extent, extent) * 0.25f, 1e-12f);
    }
    std::vector<float> weights(t.weights.size());
    for (size_t i = 0; i < weights.size(); ++i) {
        weights[i] = t.scales[i] ? projected_area * t.weights[i] : t.weights[i];
    }
    std::vector<float> cdf(weights.size() + 1, 0.0f);
    float maximum = 0;
    for (float w : weights) {
        require(std::isfinite(w) && w >= 0, "Distribution weights must be finite and nonnegative");
        maximum = std::max(maximum, w);
    }
    for (size_t i = 0; i < weights.size(); ++i) {
        cdf[i + 1] = cdf[i] + (maximum > 0 ? weights[i] / maximum : 1.0f);
    }
    if (!weights.empty()) {
        const float integral_cdf = cdf.back();
        for (auto& v : cdf) {
            v /= integral_cdf;
        }
    }
    scene.d.light_count = static_cast<uint32_t>(t.lights.size());
    if (!scene.lights.ptr) {
        scene.lights.allocate(std::max<size_t>(1, t.lights.size()));
        if (!t.lights.empty()) {
            MR_CUDA(cudaMemcpyAsync(scene.lights.ptr, t.lights.data(), t.lights.size() * sizeof(DeviceLight),
                                    cudaMemcpyHostToDevice, stream));
        }
    }
    if (!scene.light_cdf.ptr) {
        scene.light_cdf.allocate(cdf.size());
    }
    MR_CUDA(cudaMemcpyAsync(scene.light_cdf.ptr, cdf.data(), cdf.size() * sizeof(float), cudaMemcpyHostToDevice,
                            stream));
    // The copy reads host memory that goes away with this function.
    MR_CUDA(cudaStreamSynchronize(stream));
    scene.d.lights    = scene.lights.ptr;
    scene.d.light_cdf = scene.light_cdf.ptr;
}

// The host light table and the primitive -> emitter map: area lights in instance and triangle
// order, then directional lights, then the constant environment.
void build_light_table(Scene& scene, const mr_scene_desc& desc, const std::vector<uint32_t>& first_prim,
                       double map_integral, cudaStream_t stream) {
    LightTable&           t     = scene.light_table;
    const uint32_t        prims = scene.d.primitive_count;
    std::vector<uint32_t> emitter_of_prim(std::max<uint32_t>(1, prims), kNone);
    t = LightTable{};
    for (uint32_t i = 0; i < desc.instance_count; ++i) {
        const mr_instance& in  = desc.instances[i];
        const mr_material& mat = desc.materials[in.material];
        const f3 radiance = {mat.emission[0], mat.emission[1], mat.emission[2]};
        if (luminance(radiance) == 0) {
            continue;
        }
        const mr_mesh& mesh        = desc.meshes[in.mesh];
        const float    orientation = determinant3(in.object_to_world) < 0 ? -1.0f : 1.0f;
        for (uint32_t tri = 0; tri < mesh.triangle_count; ++tri) {
            f3 v[3];
            for (int c = 0; c < 3; ++c) {
                const float* p = mesh.positions + 3 * mesh.corners[3 * tri + c].position;
                v[c]           = transform_point(in.object_to_world, p[0], p[1], p[2]);
            }
            const f3    cr   = cross(v[1] - v[0], v[2] - v[0]);
            const float area = length(cr) * 0.5f;
            if (area == 0) {
                continue;
            }
            DeviceLight l{};
            l.v0 = v[0];
            l.v1 = v[1];
            l.v2 = v[2];
            l.normal       = cr * orientation / (2.0f * area);
            l.radiance     = radiance;
            l.area         = area;
            l.kind         = kLightArea;
            l.double_sided = mat.double_sided;
            emitter_of_prim[first_prim[i] + tri] = static_cast<uint32_t>(t.lights.size());
            t.lights.push_back(l);
            t.weights.push_back((mat.double_sided ? 2.0f : 1.0f) * kPi * area * luminance(radiance));
            t.scales.push_back(0);
        }
    }
    for (uint32_t i = 0; i < desc.directional_light_count; ++i) {
        const auto& dl       = desc.directional_lights[i];
        const f3    radiance = f3{dl.color[0], dl.color[1], dl.color[2]} * dl.intensity;
        if (luminance(radiance) > 0) {
            DeviceLight l{};
            l.normal   = -normalize(f3{dl.direction[0], dl.direction[1], dl.direction[2]});
            l.radiance = radiance;
            l.kind     = kLightDirectional;
            t.lights.push_back(l);
            t.weights.push_back(luminance(radiance));
            t.scales.push_back(1);
        }
    }
    const f3 environment        = {desc.environment[0], desc.environment[1], desc.environment[2]};
    scene.d.environment         = environment;
    scene.d.environment_choice  = -1;
    const float integral        = 4.0f * kPi * luminance(environment) + static_cast<float>(map_integral);
    if (integral > 0) {
        DeviceLight l{};
        l.radiance                 = environment;
        l.kind                     = kLightEnvironment;
        scene.d.environment_choice = static_cast<int>(t.lights.size());
        t.lights.push_back(l);
        t.weights.push_back(integral);
        t.scales.push_back(1);
    }
    scene.prim_emitter.allocate(emitter_of_prim.size());
    MR_CUDA(cudaMemcpyAsync(scene.prim_emitter.ptr, emitter_of_prim.data(),
                            emitter_of_prim.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    MR_CUDA(cudaStreamSynchronize(stream));  // the source vector goes away with this function
    scene.d.prim_emitter = scene.prim_emitter.ptr;
}

cudaMemPool_t library_pool() {
    static std::mutex                  mutex;
    static std::vector<cudaMemPool_t> pools;
    int device = 0;
    MR_CUDA(cudaGetDevice(&device));
    std::lock_guard<std::mutex> lock(mutex);
    if (pools.size() <= static_cast<size_t>(device)) {
        pools.resize(device + 1, nullptr);
    }
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType     = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id   = device;
        cudaMemPool_t pool  = nullptr;
        MR_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = 2ull << 30;
        MR_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[device] = pool;
    }
    return pools[device];
}

std::unique_ptr<Scene> create_scene(const mr_scene_desc& desc, const mr_bvh_desc* bvh,
                                    const mr_build_settings* build) {
    int device_count = 0;
    if (cudaGetDeviceCount(&device_count) != cudaSuccess || device_count == 0) {
        fail(MR_CUDA_ERROR, "No CUDA device is available");
    }
    auto scene = std::make_unique<Scene>();
    MR_CUDA(cudaGetDevice(&scene->device));

    // ---- validation (make_snapshot) ----
    validate_camera(desc.camera);
    require(finite3h(desc.environment) && desc.environment[0] >= 0 && desc.environment[1] >= 0 &&
                desc.environment[2] >= 0,
            "Environment must be finite and nonnegative");
    require(desc.mesh_count == 0 || desc.meshes, "Mesh table is missing");
    require(desc.material_count == 0 || desc.materials, "Material table is missing");
    require(desc.instance_count == 0 || desc.instances, "Instance table is missing");
    for (uint32_t i = 0; i < desc.material_count; ++i) {
        validate_material(desc.materials[i]);
    }
    for (uint32_t i = 0; i < desc.mesh_count; ++i) {
        validate_mesh(desc.meshes[i]);
    }
    validate_media(desc.media, desc.medium_count);
    for (uint32_t i = 0; i < desc.directional_light_count; ++i) {
        const auto& l = desc.directional_lights[i];
        const f3    d = {l.direction[0], l.direction[1], l.direction[2]};
        require(finite3(d) && length(d) > 1e-6f, "Light direction must be nonzero");
        require(finite3h(l.color) && l.color[0] >= 0 && l.color[1] >= 0 && l.color[2] >= 0 &&
                    std::isfinite(l.intensity) && l.intensity >= 0,
                "Light color/intensity must be nonnegative");
    }
    uint64_t total = 0;
    std::vector<DeviceInstance> instances(desc.instance_count);
    std::vector<uint32_t> mesh_position_offset(desc.mesh_count), mesh_corner_offset(desc.mesh_count);
    uint64_t positions_total = 0, corners_total = 0;
    for (uint32_t m = 0; m < desc.mesh_count; ++m) {
        mesh_position_offset[m] = static_cast<uint32_t>(positions_total);
        mesh_corner_offset[m]   = static_cast<uint32_t>(corners_total);
        positions_total += desc.meshes[m].position_count;
        corners_total += 3ull * desc.meshes[m].triangle_count;
        if (positions_total > 0xffffffffull || corners_total > 0xffffffffull) {
            fail(MR_LENGTH_ERROR, "Scene mesh data exceeds the 32-bit index range");
        }
    }
    for (uint32_t i = 0; i < desc.instance_count; ++i) {
        const mr_instance& in = desc.instances[i];
        require(in.mesh < desc.mesh_count, "Object references missing mesh");
        require(in.material < desc.material_count, "Object references missing material");
        bool finite = true;
        for (int k = 0; k < 16; ++k) finite = finite && std::isfinite(in.object_to_world[k]);
        for (int k = 0; k < 9; ++k) finite = finite && std::isfinite(in.normal_to_world[k]);
        require(finite, "Transform must be finite");
        const uint32_t tris = desc.meshes[in.mesh].triangle_count;
        if (tris > 0x7fffffffull - total) {
            fail(MR_LENGTH_ERROR, "Scene triangle count exceeds BVH index range");
        }
        DeviceInstance& d = instances[i];
        std::memcpy(d.object_to_world, in.object_to_world, sizeof(d.object_to_world));
        std::memcpy(d.normal_to_world, in.normal_to_world, sizeof(d.normal_to_world));
        d.position_offset = mesh_position_offset[in.mesh];
        d.corner_offset   = mesh_corner_offset[in.mesh];
        d.first_prim      = static_cast<uint32_t>(total);
        d.triangle_count  = tris;
        d.material        = in.material;
        const mr_material& mat = desc.materials[in.material];
        d.flags = (mat.double_sided ? 0u : kTriSingleSided) |
                  (determinant3(in.object_to_world) < 0 ? kTriMirrored : 0u) |
                  ((mat.emission[0] > 0 || mat.emission[1] > 0 || mat.emission[2] > 0) ? kTriEmissive : 0u) |
                  (mat.kind << 8);
        total += tris;
    }
    const uint32_t prims = static_cast<uint32_t>(total);
    scene->d.primitive_count = prims;
    if (bvh) {
        validate_imported(*bvh, prims);
    }

    // Construction runs on its own stream with stream-ordered buffers (see AllocationScope).
    struct OwnedStream {
        cudaStream_t stream = nullptr;
        OwnedStream() { MR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); }
        ~OwnedStream() { cudaStreamDestroy(stream); }
    } owned;
    cudaStream_t    stream = owned.stream;
    AllocationScope scope(stream);
    size_t          bytes = 0;

    // ---- upload meshes and instances ----
    DeviceBuffer<float>          positions;
    DeviceBuffer<mr_mesh_corner> corners;
    DeviceBuffer<uint8_t>        instance_buffer;
    positions.allocate(3 * positions_total);
    corners.allocate(corners_total);
    for (uint32_t m = 0; m < desc.mesh_count; ++m) {
        const mr_mesh& mesh = desc.meshes[m];
        MR_CUDA(cudaMemcpyAsync(positions.ptr + 3ull * mesh_position_offset[m], mesh.positions,
                                3ull * mesh.position_count * sizeof(float), cudaMemcpyHostToDevice, stream));
        MR_CUDA(cudaMemcpyAsync(corners.ptr + mesh_corner_offset[m], mesh.corners,
                                3ull * mesh.triangle_count * sizeof(mr_mesh_corner),
                                cudaMemcpyHostToDevice, stream));
    }
    instance_buffer.allocate(std::max<size_t>(1, instances.size() * sizeof(DeviceInstance)));
    if (!instances.empty()) {
        MR_CUDA(cudaMemcpyAsync(instance_buffer.ptr, instances.data(),
                                instances.size() * sizeof(DeviceInstance), cudaMemcpyHostToDevice, stream));
    }

    std::vector<uint32_t> first_prim(desc.instance_count);
    for (uint32_t i = 0; i < desc.instance_count; ++i) {
        first_prim[i] = instances[i].first_prim;
    }
    if (build && build->two_level) {
        // ---- two levels: a tree per mesh in object space under a tree over the instances ----
        require(!bvh, "A two-level scene builds its own trees; an imported tree is a flattened one");
        require(!build->split_references, "Split references apply to the flattened tree only");
        scene->two = {new TwoLevel, [](TwoLevel* t) { delete t; }};
        TwoLevel& t       = *scene->two;
        t.positions       = std::move(positions);
        t.corners         = std::move(corners);
        t.position_offset = mesh_position_offset;
        t.corner_offset   = mesh_corner_offset;
        t.used.assign(desc.mesh_count, 0);
        t.emissive_mesh.assign(desc.mesh_count, 0);
        t.host_instances.resize(desc.instance_count);
        t.instance_mesh.resize(desc.instance_count);
        t.instance_material.resize(desc.instance_count);
        for (uint32_t i = 0; i < desc.instance_count; ++i) {
            const mr_instance& in = desc.instances[i];
            DeviceInstance2&   d  = t.host_instances[i];
            d                     = DeviceInstance2{};
            fill_instance_transform(in, d);
            d.first_prim          = instances[i].first_prim;
            d.position_offset     = instances[i].position_offset;
            d.corner_offset       = instances[i].corner_offset;
            d.material            = in.material;
            d.flags               = instances[i].flags;
            t.instance_mesh[i]     = in.mesh;
            t.instance_material[i] = in.material;
            if (instances[i].triangle_count) {
                t.used[in.mesh] = 1;
            }
            if (instances[i].flags & kTriEmissive) {
                t.emissive_mesh[in.mesh] = 1;
            }
        }
        build_mesh_trees(*scene, desc, stream);
        build_instance_tree(*scene, stream);
        scene->references           = prims;
        scene->statistics.triangles = prims;
    } else {
        // ---- flatten ----
        DeviceBuffer<float4>   world, lo, hi, centroid;
        DeviceBuffer<uint32_t> error;
        world.allocate(3ull * prims);
        scene->shading.allocate(3ull * prims);
        lo.allocate(prims);
        hi.allocate(prims);
        centroid.allocate(prims);
        error.allocate(1);
        MR_CUDA(cudaMemsetAsync(error.ptr, 0, sizeof(uint32_t), stream));
        if (prims) {
            if (desc.texture_count) {  // corner UVs for texture lookups and normal maps
                scene->uvs.allocate(3ull * prims);
            }
            flatten_kernel<<<(prims + 255) / 256, 256, 0, stream>>>(
                positions.ptr, corners.ptr, reinterpret_cast<const DeviceInstance*>(instance_buffer.ptr),
                desc.instance_count, prims, world.ptr, scene->shading.ptr, lo.ptr, hi.ptr, centroid.ptr,
                error.ptr, scene->uvs.ptr);
            MR_CUDA(cudaGetLastError());
        }
        uint32_t flatten_error = 0;
        MR_CUDA(cudaMemcpyAsync(&flatten_error, error.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        require(!(flatten_error & 1u), "Transformed triangle position is not finite");
        require(!(flatten_error & 2u), "Transform collapses a triangle at float precision");
        positions.release();
        corners.release();

        // ---- BVH (reference layout on the device) ----
        DeviceBuffer<mr_bvh_node> ref_nodes;
        DeviceBuffer<uint32_t>    ref_order;
        uint32_t                  node_count = 0;
        if (prims) {
            if (bvh) {
                node_count = bvh->node_count;
                ref_nodes.allocate(node_count);
                ref_order.allocate(prims);
                MR_CUDA(cudaMemcpyAsync(ref_nodes.ptr, bvh->nodes, node_count * sizeof(mr_bvh_node),
                                        cudaMemcpyHostToDevice, stream));
                MR_CUDA(cudaMemcpyAsync(ref_order.ptr, bvh->order, prims * sizeof(uint32_t),
                                        cudaMemcpyHostToDevice, stream));
                // Statistics of the imported tree (host walk).
                std::vector<std::pair<uint32_t, uint32_t>> stack{{0u, 0u}};
                uint64_t leaves = 0, depth = 0;
                while (!stack.empty()) {
                    const auto [i, d] = stack.back();
                    stack.pop_back();
                    depth = std::max<uint64_t>(depth, d);
                    const auto& n = bvh->nodes[i];
                    if (n.count) {
                        ++leaves;
                    } else {
                        require(d < 64, "Imported BVH is deeper than 64 levels");
                        stack.push_back({n.first, d + 1});
                        stack.push_back({n.right, d + 1});
                    }
                }
                scene->statistics.leaves        = leaves;
                scene->statistics.maximum_depth = depth;
            } else {
                SplitReferences split;
                if (build && build->split_references) {
                    const float    factor = build->split_factor > 0 ? build->split_factor : 16.0f;
                    const uint64_t cap    = build->max_references
                                                ? build->max_references
                                                : std::max<uint64_t>(2ull * prims, prims + 65536ull);
                    require(std::isfinite(factor) && cap >= prims && cap <= 0xFFFFFFFFull,
                            "Split settings need a finite factor and a reference cap of at least the "
                            "triangle count");
                    split = split_references(world.ptr, lo.ptr, hi.ptr, prims, factor, cap, stream);
                }
                const uint32_t refs  = split.count ? split.count : prims;
                BuildResult    built = split.count
                                           ? build_bvh_device(split.lo.ptr, split.hi.ptr, split.centroid.ptr, refs, stream)
                                           : build_bvh_device(lo.ptr, hi.ptr, centroid.ptr, prims, stream);
                if (split.count) {
                    map_order_to_primitives(built.order.ptr, split.prim.ptr, refs, stream);
                }
                ref_nodes             = std::move(built.nodes);
                ref_order             = std::move(built.order);
                node_count            = built.node_count;
                scene->statistics.leaves        = built.leaves;
                scene->statistics.maximum_depth = built.maximum_depth;
                scene->build_seconds  = built.seconds;
                scene->references     = refs;
            }
        }
        if (scene->references == 0) {
            scene->references = prims;
        }
        const uint32_t slots = scene->references;
        scene->statistics.triangles = prims;
        scene->statistics.nodes     = node_count;
        lo.release();
        hi.release();
        centroid.release();

        // ---- traversal layout: 4-wide nodes collapsed from the binary tree ----
        uint32_t wide_count = 0;
        if (prims) {
            WideTree wide = collapse_tree(ref_nodes.ptr, node_count, stream);
            scene->nodes  = std::move(wide.nodes);
            wide_count    = wide.count;
            scene->tris.allocate(3ull * slots);
            scene->d.slot_count = slots;
            gather_triangles_kernel<<<(slots + 255) / 256, 256, 0, stream>>>(world.ptr, ref_order.ptr, slots,
                                                                             scene->tris.ptr);
            mark_leaf_end_kernel<<<(node_count + 255) / 256, 256, 0, stream>>>(ref_nodes.ptr, node_count,
                                                                               scene->tris.ptr);
            MR_CUDA(cudaGetLastError());
            mr_bvh_node root{};
            MR_CUDA(cudaMemcpyAsync(&root, ref_nodes.ptr, sizeof(root), cudaMemcpyDeviceToHost, stream));
            MR_CUDA(cudaStreamSynchronize(stream));
            scene->d.has_nodes  = 1;
            scene->d.root       = root.count == 0 ? 0 : ~static_cast<int>(root.first);
            scene->d.root_count = root.count;
            for (int a = 0; a < 3; ++a) {
                scene->d.root_lo[a] = root.minimum[a];
                scene->d.root_hi[a] = root.maximum[a];
            }
        }
        scene->d.node_count = wide_count;
        scene->ref_nodes    = std::move(ref_nodes);
        scene->ref_order    = std::move(ref_order);
    }

    // ---- materials ----
    std::vector<DeviceMaterial> materials(std::max<uint32_t>(1, desc.material_count));
    for (uint32_t i = 0; i < desc.material_count; ++i) {
        const mr_material& m = desc.materials[i];
        require(m.base_color_texture <= desc.texture_count && m.normal_texture <= desc.texture_count,
                "Material references missing texture");
        require(m.texture_filter <= MR_FILTER_TRILINEAR, "Unknown texture filter");
        require(std::isfinite(m.normal_scale), "Normal scale must be finite");
        materials[i] = {{m.base_color[0], m.base_color[1], m.base_color[2]},
                        {m.emission[0], m.emission[1], m.emission[2]},
                        m.roughness * m.roughness, m.ior, m.kind, m.double_sided,
                        static_cast<int>(m.base_color_texture) - 1, static_cast<int>(m.normal_texture) - 1,
                        m.texture_filter, m.normal_scale, m.normal_flip_y};
    }
    scene->materials.allocate(materials.size());
    MR_CUDA(cudaMemcpyAsync(scene->materials.ptr, materials.data(), materials.size() * sizeof(DeviceMaterial),
                            cudaMemcpyHostToDevice, stream));

    // ---- lights (LightSampler constructor, src/render/light.cpp:197-264) ----
    upload_textures(*scene, desc, stream);
    build_light_table(*scene, desc, first_prim, prepare_environment(*scene, desc, stream), stream);
    if (scene->two) {
        upload_light_table(*scene, scene->two->world_lo, scene->two->world_hi, stream);
    } else {
        upload_light_table(*scene, scene->d.root_lo, scene->d.root_hi, stream);
    }

    // ---- media ----
    std::vector<DeviceMedium> media(std::max<uint32_t>(1, desc.medium_count));
    int scatter = 0;
    for (uint32_t i = 0; i < desc.medium_count; ++i) {
        const auto& r = desc.media[i];
        DeviceMedium& m = media[i];
        m.minimum    = {float(r.minimum[0]), float(r.minimum[1]), float(r.minimum[2])};
        m.maximum    = {float(r.maximum[0]), float(r.maximum[1]), float(r.maximum[2])};
        m.absorption = {float(r.absorption[0]), float(r.absorption[1]), float(r.absorption[2])};
        m.scattering = {float(r.scattering[0]), float(r.scattering[1]), float(r.scattering[2])};
        m.extinction = m.absorption + m.scattering;
        m.anisotropy = float(r.anisotropy);
        m.scatters   = (m.scattering.x != 0 || m.scattering.y != 0 || m.scattering.z != 0) ? 1 : 0;
        m.enabled    = r.enabled ? 1 : 0;
        scatter |= m.scatters && m.enabled;
    }
    scene->media.allocate(media.size());
    MR_CUDA(cudaMemcpyAsync(scene->media.ptr, media.data(), media.size() * sizeof(DeviceMedium),
                            cudaMemcpyHostToDevice, stream));
    scene->d.medium_count  = static_cast<int>(desc.medium_count);
    scene->d.media_scatter = scatter;

    // ---- camera basis (src/scene/scene.cpp:176-180) ----
    const mr_camera& c = desc.camera;
    CameraBasis&     b = scene->d.camera;
    b.position        = {c.position[0], c.position[1], c.position[2]};
    b.forward         = normalize(f3{c.target[0], c.target[1], c.target[2]} - b.position);
    b.right           = normalize(cross(b.forward, f3{c.up[0], c.up[1], c.up[2]}));
    b.up              = cross(b.right, b.forward);
    b.half_height     = std::tan(c.vertical_fov_degrees * (kPi / 180.0f) * 0.5f);
    b.near_plane      = c.near_plane;
    b.far_plane       = c.far_plane;
    b.aperture_radius = c.aperture_radius;
    b.focus_distance  = c.focus_distance;

    MR_CUDA(cudaStreamSynchronize(stream));
    scene->d.nodes        = scene->nodes.ptr;
    scene->d.tris         = scene->tris.ptr;
    scene->d.shading      = scene->shading.ptr;
    scene->d.materials    = scene->materials.ptr;
    scene->d.lights       = scene->lights.ptr;
    scene->d.light_cdf    = scene->light_cdf.ptr;
    scene->d.prim_emitter = scene->prim_emitter.ptr;
    scene->d.media        = scene->media.ptr;
    scene->d.uvs          = scene->uvs.ptr;
    bytes = scene->nodes.bytes() + scene->tris.bytes() + scene->shading.bytes() +
            scene->ref_nodes.bytes() + scene->ref_order.bytes() + scene->prim_emitter.bytes() +
            scene->materials.bytes() + scene->lights.bytes() + scene->light_cdf.bytes() +
            scene->media.bytes() + scene->uvs.bytes() + scene->texels.bytes() + scene->texture_table.bytes() +
            scene->env_row_cdf.bytes() + scene->env_col_cdf.bytes() + scene->env_solid_angle.bytes();
    scene->device_bytes = bytes;
    if (scene->two) {
        publish_two_level(*scene);
    }
    return scene;
}

}  // namespace mr
