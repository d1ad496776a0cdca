// instancing.cu — two-level scenes: one object-space BVH per mesh (the BLAS) under a BVH over
// the instances (the TLAS), and their refit.
//
// The reference flattens every instance into one world-space BVH (src/render/bvh.cpp:31-99), so
// a mesh instanced n times costs n copies of its triangles and tree. Here each mesh is stored and
// built once in object space; the instance tree is built over the instances' world boxes. The
// traversal (traverse.cuh: trace2) maps the ray into object space only to cull mesh boxes, and
// tests every candidate triangle in world space after transforming its object-space vertices
// with the flattening's own arithmetic (transform_point): the vertices, ray and test are the
// flattened scene's, so hits are too. What the flattened build gets from its world triangles
// (finite positions, no triangle collapsed by the transform, the exact world bounds that weight
// the directional and environment lights) comes from one pass over every instance triangle that
// stores nothing.
//
// Refit: new instance transforms rebuild only the instance tree; new mesh positions refit that
// mesh's binary tree bottom-up (same topology), collapse it again into the same wide-node slots
// and rebuild the instance tree.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "errors.hpp"
#include "instancing.cuh"
#include "scan.cuh"

namespace mr {

namespace {

constexpr float kBoxPadScale = 3.814697265625e-06f;  // 2^-18 = 64 FP32 unit roundoffs

__device__ __forceinline__ uint32_t ordered(float f) {  // order-preserving float -> uint
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
float unordered(uint32_t o) {
    uint32_t b = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    float    f;
    std::memcpy(&f, &b, sizeof(f));
    return f;
}

// Object-space triangle bounds and centroids of one mesh: the builder's inputs, computed as the
// flattening computes them for world triangles (centroid ((v0/3) + v1/3) + v2/3).
// With `error`, also MeshData::validate's degenerate-triangle check (src/scene/scene.cpp:38-66)
// with the host check's unfused FP32 arithmetic, for positions replaced by a refit.
__global__ void mesh_bounds_kernel(const float* positions, const mr_mesh_corner* corners, uint32_t tris,
                                   float4* lo, float4* hi, float4* centroid, unsigned* error = nullptr) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tris) {
        return;
    }
    f3 v[3];
    for (int c = 0; c < 3; ++c) {
        const float* p = positions + 3 * static_cast<size_t>(corners[3 * t + c].position);
        v[c]           = {p[0], p[1], p[2]};
    }
    if (error) {
        const f3 e1 = {__fsub_rn(v[1].x, v[0].x), __fsub_rn(v[1].y, v[0].y), __fsub_rn(v[1].z, v[0].z)};
        const f3 e2 = {__fsub_rn(v[2].x, v[0].x), __fsub_rn(v[2].y, v[0].y), __fsub_rn(v[2].z, v[0].z)};
        const f3 a  = {__fsub_rn(__fmul_rn(e1.y, e2.z), __fmul_rn(e2.y, e1.z)),
                       __fsub_rn(__fmul_rn(e1.z, e2.x), __fmul_rn(e2.z, e1.x)),
                       __fsub_rn(__fmul_rn(e1.x, e2.y), __fmul_rn(e2.x, e1.y))};
        const float area2 = __fadd_rn(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fmul_rn(a.z, a.z));
        if (!(area2 > 1e-20f)) {
            atomicOr(error, 4u);
        }
    }
    lo[t] = make_float4(fminf(fminf(v[0].x, v[1].x), v[2].x), fminf(fminf(v[0].y, v[1].y), v[2].y),
                        fminf(fminf(v[0].z, v[1].z), v[2].z), 0.0f);
    hi[t] = make_float4(fmaxf(fmaxf(v[0].x, v[1].x), v[2].x), fmaxf(fmaxf(v[0].y, v[1].y), v[2].y),
                        fmaxf(fmaxf(v[0].z, v[1].z), v[2].z), 0.0f);
    centroid[t] = make_float4(((v[0].x / 3.0f) + v[1].x / 3.0f) + v[2].x / 3.0f,
                              ((v[0].y / 3.0f) + v[1].y / 3.0f) + v[2].y / 3.0f,
                              ((v[0].z / 3.0f) + v[1].z / 3.0f) + v[2].z / 3.0f, 0.0f);
}

// Object-space triangle slots of one mesh in leaf order (slot_base.. of blas_tris): vertices and
// the triangle's index within the mesh. Leaf ends are marked separately.
__global__ void mesh_slots_kernel(const float* positions, const mr_mesh_corner* corners, const uint32_t* order,
                                  uint32_t count, float4* slots) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) {
        return;
    }
    const uint32_t t = order[k];
    for (int c = 0; c < 3; ++c) {
        const float* p = positions + 3 * static_cast<size_t>(corners[3 * t + c].position);
        slots[3 * static_cast<size_t>(k) + c] =
            make_float4(p[0], p[1], p[2], c == 0 ? __uint_as_float(t) : 0.0f);
    }
}

// Rebases one mesh tree's wide nodes into the shared array: interior refs by the node base, leaf
// refs (~slot) by the slot base. Empty children keep an empty box and are never followed.
__global__ void rebase_nodes_kernel(const float4* in, uint32_t count, uint32_t node_base, uint32_t slot_base,
                                    float4* out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) {
        return;
    }
    for (int r = 0; r < 8; ++r) {
        out[8 * static_cast<size_t>(k) + r] = in[8 * static_cast<size_t>(k) + r];
    }
    float4&    refs = out[8 * static_cast<size_t>(k) + 6];
    int        r4[4] = {__float_as_int(refs.x), __float_as_int(refs.y), __float_as_int(refs.z),
                        __float_as_int(refs.w)};
    for (int i = 0; i < 4; ++i) {
        r4[i] = r4[i] >= 0 ? r4[i] + static_cast<int>(node_base) : ~(~r4[i] + static_cast<int>(slot_base));
    }
    refs = make_float4(__int_as_float(r4[0]), __int_as_float(r4[1]), __int_as_float(r4[2]),
                       __int_as_float(r4[3]));
}

// One thread per instance triangle: the flattening's world vertices, checked as the flattened
// build checks them, reduced to the exact world bounds (ordered-integer atomics). Nothing is
// stored per triangle.
__global__ void instance_triangles_kernel(const float* positions, const mr_mesh_corner* corners,
                                          const DeviceInstance2* instances, uint32_t instance_count,
                                          uint32_t prims, unsigned* error, uint32_t* bounds) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    f3   mn = {INFINITY, INFINITY, INFINITY}, mx = {-INFINITY, -INFINITY, -INFINITY};
    if (p < prims) {
        const uint32_t         ii   = find_instance2(instances, instance_count, p);
        const DeviceInstance2& inst = instances[ii];
        const uint32_t         tri  = p - inst.first_prim;
        f3 v[3];
        for (int c = 0; c < 3; ++c) {
            const mr_mesh_corner& corner = corners[inst.corner_offset + 3 * tri + c];
            const float* q = positions + 3 * (static_cast<size_t>(inst.position_offset) + corner.position);
            v[c] = transform_point(inst.to_world, q[0], q[1], q[2]);
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
        mn = {fminf(fminf(v[0].x, v[1].x), v[2].x), fminf(fminf(v[0].y, v[1].y), v[2].y),
              fminf(fminf(v[0].z, v[1].z), v[2].z)};
        mx = {fmaxf(fmaxf(v[0].x, v[1].x), v[2].x), fmaxf(fmaxf(v[0].y, v[1].y), v[2].y),
              fmaxf(fmaxf(v[0].z, v[1].z), v[2].z)};
    }
    // Warp minima/maxima of the ordered bits, one atomic per value per warp.
    uint32_t o[6] = {ordered(mn.x), ordered(mn.y), ordered(mn.z), ordered(mx.x), ordered(mx.y), ordered(mx.z)};
    o[0] = __reduce_min_sync(0xffffffffu, o[0]);
    o[1] = __reduce_min_sync(0xffffffffu, o[1]);
    o[2] = __reduce_min_sync(0xffffffffu, o[2]);
    o[3] = __reduce_max_sync(0xffffffffu, o[3]);
    o[4] = __reduce_max_sync(0xffffffffu, o[4]);
    o[5] = __reduce_max_sync(0xffffffffu, o[5]);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(bounds + 0, o[0]);
        atomicMin(bounds + 1, o[1]);
        atomicMin(bounds + 2, o[2]);
        atomicMax(bounds + 3, o[3]);
        atomicMax(bounds + 4, o[4]);
        atomicMax(bounds + 5, o[5]);
    }
}

// Instance world boxes for the instance-level build: the eight corners of the mesh tree's root
// box transformed with the flattening's arithmetic, grown by 2^-18 of the magnitudes involved
// (the transform's absolute row sums) so that every world vertex of the instance lies inside.
__global__ void instance_boxes_kernel(DeviceInstance2* instances, uint32_t count, const float* mesh_boxes,
                                      const uint32_t* instance_mesh, float4* lo, float4* hi,
                                      float4* centroid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) {
        return;
    }
    DeviceInstance2& inst = instances[i];
    const float*     box  = mesh_boxes + 6 * instance_mesh[i];
    f3 mn = {INFINITY, INFINITY, INFINITY}, mx = {-INFINITY, -INFINITY, -INFINITY};
    f3 mag = {0, 0, 0};
    for (int c = 0; c < 8; ++c) {
        const float x = box[(c & 1) ? 3 : 0], y = box[(c & 2) ? 4 : 1], z = box[(c & 4) ? 5 : 2];
        const f3    w = transform_point(inst.to_world, x, y, z);
        mn = {fminf(mn.x, w.x), fminf(mn.y, w.y), fminf(mn.z, w.z)};
        mx = {fmaxf(mx.x, w.x), fmaxf(mx.y, w.y), fmaxf(mx.z, w.z)};
        const float* m = inst.to_world;
        for (int r = 0; r < 3; ++r) {
            const float s = fabsf(m[r] * x) + fabsf(m[4 + r] * y) + fabsf(m[8 + r] * z) + fabsf(m[12 + r]);
            if (r == 0) mag.x = fmaxf(mag.x, s);
            if (r == 1) mag.y = fmaxf(mag.y, s);
            if (r == 2) mag.z = fmaxf(mag.z, s);
        }
    }
    const f3 pad = {kBoxPadScale * (mag.x + (mx.x - mn.x)), kBoxPadScale * (mag.y + (mx.y - mn.y)),
                    kBoxPadScale * (mag.z + (mx.z - mn.z))};
    mn = mn - pad;
    mx = mx + pad;
    inst.lo[0] = mn.x, inst.lo[1] = mn.y, inst.lo[2] = mn.z;
    inst.hi[0] = mx.x, inst.hi[1] = mx.y, inst.hi[2] = mx.z;
    lo[i]       = f4(mn, 0.0f);
    hi[i]       = f4(mx, 0.0f);
    centroid[i] = f4((mn + mx) * 0.5f, 0.0f);
}

// Instance ids in instance-tree leaf order; bit 31 marks each leaf's last item (second kernel).
__global__ void tlas_items_kernel(const uint32_t* order, uint32_t count, uint32_t* items) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) {
        items[k] = order[k];
    }
}

__global__ void tlas_leaf_end_kernel(const mr_bvh_node* nodes, uint32_t node_count, uint32_t* items) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= node_count || nodes[i].count == 0) {
        return;
    }
    items[nodes[i].first + nodes[i].count - 1] |= 0x80000000u;
}

// Parent of every node of a binary tree (root: kNone).
__global__ void parents_kernel(const mr_bvh_node* nodes, uint32_t count, uint32_t* parent) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) {
        return;
    }
    if (i == 0) {
        parent[0] = kNone;
    }
    if (nodes[i].count == 0) {
        parent[nodes[i].first] = i;
        parent[nodes[i].right] = i;
    }
}

// Bottom-up refit of a binary tree over new primitive bounds: every leaf recomputes its box and
// walks up; at each interior node the second child to arrive (an atomic counter) recomputes the
// node's box from its two children. Topology and primitive order are unchanged.
__global__ void refit_kernel(mr_bvh_node* nodes, uint32_t count, const uint32_t* parent, const uint32_t* order,
                             const float4* lo, const float4* hi, uint32_t* arrivals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count || nodes[i].count == 0) {
        return;
    }
    mr_bvh_node& leaf = nodes[i];
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = 0; k < leaf.count; ++k) {
        const uint32_t p = order[leaf.first + k];
        const float4   a = lo[p], b = hi[p];
        mn[0] = fminf(mn[0], a.x), mn[1] = fminf(mn[1], a.y), mn[2] = fminf(mn[2], a.z);
        mx[0] = fmaxf(mx[0], b.x), mx[1] = fmaxf(mx[1], b.y), mx[2] = fmaxf(mx[2], b.z);
    }
    for (int a = 0; a < 3; ++a) {
        leaf.minimum[a] = mn[a];
        leaf.maximum[a] = mx[a];
    }
    uint32_t node = parent[i];
    while (node != kNone) {
        __threadfence();
        if (atomicAdd(arrivals + node, 1u) == 0) {
            return;  // the sibling's thread finishes this node
        }
        __threadfence();
        mr_bvh_node&       n = nodes[node];
        const mr_bvh_node& l = nodes[n.first];
        const mr_bvh_node& r = nodes[n.right];
        for (int a = 0; a < 3; ++a) {
            n.minimum[a] = fminf(*((volatile const float*)&l.minimum[a]), *((volatile const float*)&r.minimum[a]));
            n.maximum[a] = fmaxf(*((volatile const float*)&l.maximum[a]), *((volatile const float*)&r.maximum[a]));
        }
        node = parent[node];
    }
}

// Rows 0..5 of a mesh's wide nodes from the refit binary tree (children kept from the collapse).
__global__ void refit_wide_kernel(const mr_bvh_node* nodes, const int4* children, uint32_t count, float4* wide) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) {
        return;
    }
    const int4 c4   = children[k];
    const int  c[4] = {c4.x, c4.y, c4.z, c4.w};
    float      lo[3][4], hi[3][4];
    for (int i = 0; i < 4; ++i) {
        for (int a = 0; a < 3; ++a) {
            lo[a][i] = c[i] < 0 ? INFINITY : nodes[c[i]].minimum[a];
            hi[a][i] = c[i] < 0 ? -INFINITY : nodes[c[i]].maximum[a];
        }
    }
    float4* o = wide + 8 * static_cast<size_t>(k);
    for (int a = 0; a < 3; ++a) {
        o[2 * a]     = make_float4(lo[a][0], lo[a][1], lo[a][2], lo[a][3]);
        o[2 * a + 1] = make_float4(hi[a][0], hi[a][1], hi[a][2], hi[a][3]);
    }
}

unsigned grid(size_t n, unsigned block = 256) { return static_cast<unsigned>((n + block - 1) / block); }

// 3x3 inverse and infinity norms of an affine object_to_world (column-major 4x4), in double.
void inverse_affine(const float* m, float* to_object, float& a_norm, float& b_norm) {
    const double a[3][3] = {{m[0], m[4], m[8]}, {m[1], m[5], m[9]}, {m[2], m[6], m[10]}};
    const double t[3]    = {m[12], m[13], m[14]};
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                       a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                       a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    require(std::isfinite(det) && det != 0, "Instance transform is singular");
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    a_norm = 0;
    b_norm = 0;
    for (int r = 0; r < 3; ++r) {
        double b = 0, row = 0;
        for (int c = 0; c < 3; ++c) {
            to_object[4 * r + c] = static_cast<float>(inv[r][c]);
            b -= inv[r][c] * t[c];
            row += std::abs(inv[r][c]);
        }
        to_object[4 * r + 3] = static_cast<float>(b);
        a_norm = std::max(a_norm, static_cast<float>(row));
        b_norm = std::max(b_norm, static_cast<float>(std::abs(b)));
    }
}

// Object-space growth of an instance's mesh boxes that covers the FP32 rounding of its world
// vertices (at most a few unit roundoffs of the transform's absolute row sums), mapped back to
// object space by the inverse's norm, with a factor of 32 to spare; plus the same relative
// growth of the box itself.
float static_margin(const float* m, const float* box, float a_norm) {
    double world = 0, object = 0;
    for (int c = 0; c < 8; ++c) {
        const double x = box[(c & 1) ? 3 : 0], y = box[(c & 2) ? 4 : 1], z = box[(c & 4) ? 5 : 2];
        object = std::max({object, std::abs(x), std::abs(y), std::abs(z)});
        for (int r = 0; r < 3; ++r) {
            world = std::max(world, std::abs(double(m[r]) * x) + std::abs(double(m[4 + r]) * y) +
                                        std::abs(double(m[8 + r]) * z) + std::abs(double(m[12 + r])));
        }
    }
    return static_cast<float>(std::ldexp(double(a_norm) * world + object, -19));
}

}  // namespace

void fill_instance_transform(const mr_instance& in, DeviceInstance2& d) {
    std::memcpy(d.to_world, in.object_to_world, sizeof(d.to_world));
    std::memcpy(d.normal_to_world, in.normal_to_world, sizeof(d.normal_to_world));
    inverse_affine(in.object_to_world, d.to_object, d.a_norm, d.b_norm);
}

// Mesh trees: one binary build per mesh used by an instance, collapsed into wide nodes and
// appended to the shared node and slot arrays.
void build_mesh_trees(Scene& scene, const mr_scene_desc& desc, cudaStream_t stream) {
    auto&    t = *scene.two;
    uint32_t node_total = 0, slot_total = 0;
    std::vector<WideTree> wides(desc.mesh_count);
    t.mesh.resize(desc.mesh_count);
    for (uint32_t m = 0; m < desc.mesh_count; ++m) {
        MeshTree& mt   = t.mesh[m];
        mt.triangles   = desc.meshes[m].triangle_count;
        mt.positions   = desc.meshes[m].position_count;
        mt.slot_base   = slot_total;
        if (!t.used[m] || mt.triangles == 0) {
            continue;
        }
        DeviceBuffer<float4> lo, hi, centroid;
        lo.allocate(mt.triangles);
        hi.allocate(mt.triangles);
        centroid.allocate(mt.triangles);
        mesh_bounds_kernel<<<grid(mt.triangles), 256, 0, stream>>>(
            t.positions.ptr + 3ull * t.position_offset[m], t.corners.ptr + t.corner_offset[m], mt.triangles,
            lo.ptr, hi.ptr, centroid.ptr);
        MR_CUDA(cudaGetLastError());
        BuildResult built = build_bvh_device(lo.ptr, hi.ptr, centroid.ptr, mt.triangles, stream);
        scene.build_seconds += built.seconds;
        mt.nodes      = std::move(built.nodes);
        mt.order      = std::move(built.order);
        mt.node_count = built.node_count;
        mt.leaves     = built.leaves;
        mt.depth      = built.maximum_depth;
        wides[m]      = collapse_tree(mt.nodes.ptr, mt.node_count, stream);
        mt.wide_children = std::move(wides[m].children);
        mt.node_base  = node_total;
        mt.wide_count = wides[m].count;
        mt.root       = wides[m].root_count ? ~static_cast<int>(slot_total) : static_cast<int>(node_total);
        for (int a = 0; a < 3; ++a) {
            mt.box[a]     = wides[m].lo[a];
            mt.box[3 + a] = wides[m].hi[a];
        }
        node_total += wides[m].count;
        slot_total += mt.triangles;
    }
    t.blas_nodes.allocate(std::max<uint32_t>(1, node_total) * 8ull);
    t.blas_tris.allocate(std::max<uint32_t>(1, slot_total) * 3ull);
    for (uint32_t m = 0; m < desc.mesh_count; ++m) {
        MeshTree& mt = t.mesh[m];
        if (!t.used[m] || mt.triangles == 0) {
            continue;
        }
        write_mesh_tree(scene, m, wides[m], stream);
    }
}

void write_mesh_tree(Scene& scene, uint32_t m, const WideTree& wide, cudaStream_t stream) {
    auto&     t  = *scene.two;
    MeshTree& mt = t.mesh[m];
    if (wide.count) {
        rebase_nodes_kernel<<<grid(wide.count), 256, 0, stream>>>(wide.nodes.ptr, wide.count, mt.node_base,
                                                                   mt.slot_base,
                                                                   t.blas_nodes.ptr + 8ull * mt.node_base);
    }
    float4* slots = t.blas_tris.ptr + 3ull * mt.slot_base;
    mesh_slots_kernel<<<grid(mt.triangles), 256, 0, stream>>>(t.positions.ptr + 3ull * t.position_offset[m],
                                                               t.corners.ptr + t.corner_offset[m],
                                                               mt.order.ptr, mt.triangles, slots);
    mark_leaf_ends(mt.nodes.ptr, mt.node_count, slots, stream);
    MR_CUDA(cudaGetLastError());
}

// Instance boxes, the instance tree, the validation pass and the exact world bounds: everything
// that depends on the instances' transforms.
void build_instance_tree(Scene& scene, cudaStream_t stream) {
    auto&          t     = *scene.two;
    const uint32_t count = static_cast<uint32_t>(t.host_instances.size());
    std::vector<float>    boxes(6 * std::max<size_t>(1, t.mesh.size()));
    std::vector<uint32_t> instance_mesh(std::max<uint32_t>(1, count));
    for (size_t m = 0; m < t.mesh.size(); ++m) {
        std::memcpy(&boxes[6 * m], t.mesh[m].box, sizeof(t.mesh[m].box));
    }
    for (uint32_t i = 0; i < count; ++i) {
        DeviceInstance2& d = t.host_instances[i];
        const MeshTree&  mt = t.mesh[t.instance_mesh[i]];
        d.blas_root       = mt.root;
        d.margin_static   = static_margin(d.to_world, mt.box, d.a_norm);
        instance_mesh[i]  = t.instance_mesh[i];
    }
    t.instances.allocate(std::max<uint32_t>(1, count));
    DeviceBuffer<float>    d_boxes;
    DeviceBuffer<uint32_t> d_mesh;
    d_boxes.allocate(boxes.size());
    d_mesh.allocate(instance_mesh.size());
    MR_CUDA(cudaMemcpyAsync(d_boxes.ptr, boxes.data(), boxes.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
    MR_CUDA(cudaMemcpyAsync(d_mesh.ptr, instance_mesh.data(), instance_mesh.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, stream));
    if (count) {
        MR_CUDA(cudaMemcpyAsync(t.instances.ptr, t.host_instances.data(), count * sizeof(DeviceInstance2),
                                cudaMemcpyHostToDevice, stream));
    }
    // Validation and exact bounds over every instance triangle.
    const uint32_t prims = scene.d.primitive_count;
    DeviceBuffer<uint32_t> word;
    word.allocate(7);
    const uint32_t init[7] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u};
    MR_CUDA(cudaMemcpyAsync(word.ptr, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    if (prims) {
        instance_triangles_kernel<<<grid(prims), 256, 0, stream>>>(t.positions.ptr, t.corners.ptr, t.instances.ptr,
                                                                  count, prims, word.ptr + 6, word.ptr);
        MR_CUDA(cudaGetLastError());
    }
    uint32_t out[7];
    MR_CUDA(cudaMemcpyAsync(out, word.ptr, sizeof(out), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    require(!(out[6] & 1u), "Transformed triangle position is not finite");
    require(!(out[6] & 2u), "Transform collapses a triangle at float precision");
    for (int a = 0; a < 3; ++a) {
        t.world_lo[a] = unordered(out[a]);
        t.world_hi[a] = unordered(out[3 + a]);
    }
    // Instance world boxes and the instance-level tree.
    t.tlas_nodes.release();
    t.tlas_items.release();
    t.tlas_node_count = 0;
    scene.d.has_nodes = 0;
    if (count == 0 || prims == 0) {
        return;
    }
    DeviceBuffer<float4> lo, hi, centroid;
    lo.allocate(count);
    hi.allocate(count);
    centroid.allocate(count);
    instance_boxes_kernel<<<grid(count, 128), 128, 0, stream>>>(t.instances.ptr, count, d_boxes.ptr, d_mesh.ptr, lo.ptr,
                                                           hi.ptr, centroid.ptr);
    MR_CUDA(cudaGetLastError());
    BuildResult built = build_bvh_device(lo.ptr, hi.ptr, centroid.ptr, count, stream);
    scene.build_seconds += built.seconds;
    WideTree wide       = collapse_tree(built.nodes.ptr, built.node_count, stream);
    t.tlas_nodes        = std::move(wide.nodes);
    t.tlas_node_count   = built.node_count;
    t.tlas_depth        = built.maximum_depth;
    t.tlas_items.allocate(count);
    tlas_items_kernel<<<grid(count), 256, 0, stream>>>(built.order.ptr, count, t.tlas_items.ptr);
    tlas_leaf_end_kernel<<<grid(built.node_count), 256, 0, stream>>>(built.nodes.ptr, built.node_count,
                                                                    t.tlas_items.ptr);
    MR_CUDA(cudaGetLastError());
    // The instance records now hold their world boxes (written by instance_boxes_kernel).
    MR_CUDA(cudaMemcpyAsync(t.host_instances.data(), t.instances.ptr, count * sizeof(DeviceInstance2),
                            cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    scene.d.has_nodes  = 1;
    scene.d.root       = wide.root_count ? ~0 : 0;
    scene.d.root_count = wide.root_count;
    for (int a = 0; a < 3; ++a) {
        scene.d.root_lo[a] = wide.lo[a];
        scene.d.root_hi[a] = wide.hi[a];
    }
}

void publish_two_level(Scene& scene) {
    auto& t                  = *scene.two;
    scene.d.two_level        = 1;
    scene.d.slot_count       = scene.d.primitive_count;
    scene.d.instance_count   = static_cast<uint32_t>(t.host_instances.size());
    scene.d.instances        = t.instances.ptr;
    scene.d.tlas_items       = t.tlas_items.ptr;
    scene.d.nodes            = t.tlas_nodes.ptr;
    scene.d.node_count       = static_cast<uint32_t>(t.tlas_nodes.count / 8);
    scene.d.blas_nodes       = t.blas_nodes.ptr;
    scene.d.blas_tris        = t.blas_tris.ptr;
    scene.d.mesh_positions   = t.positions.ptr;
    scene.d.mesh_corners     = t.corners.ptr;
    uint64_t nodes = t.tlas_node_count, leaves = 0, depth = t.tlas_depth;
    for (const auto& m : t.mesh) {
        nodes += m.node_count;
        leaves += m.leaves;
        depth = std::max<uint64_t>(depth, t.tlas_depth + 1 + m.depth);
    }
    scene.statistics.nodes         = nodes;
    scene.statistics.leaves        = leaves;
    scene.statistics.maximum_depth = depth;
    scene.device_bytes = t.instances.bytes() + t.tlas_nodes.bytes() + t.tlas_items.bytes() + t.blas_nodes.bytes() +
                         t.blas_tris.bytes() + t.positions.bytes() + t.corners.bytes() +
                         scene.prim_emitter.bytes() + scene.materials.bytes() + scene.lights.bytes() +
                         scene.light_cdf.bytes() + scene.media.bytes() + scene.texels.bytes() +
                         scene.texture_table.bytes() + scene.env_row_cdf.bytes() + scene.env_col_cdf.bytes() +
                         scene.env_solid_angle.bytes();
    for (const auto& m : t.mesh) {
        scene.device_bytes += m.nodes.bytes() + m.order.bytes();
    }
}

void update_instances(Scene& scene, uint32_t first, uint32_t count, const mr_instance* instances) {
    require(scene.two != nullptr, "Refit needs a scene built with two levels");
    auto& t = *scene.two;
    require(instances != nullptr || count == 0, "Instance table is missing");
    require(first <= t.host_instances.size() && count <= t.host_instances.size() - first,
            "Instance range is outside the scene");
    const std::vector<DeviceInstance2> previous = t.host_instances;
    for (uint32_t k = 0; k < count; ++k) {
        const mr_instance& in = instances[k];
        const uint32_t     i  = first + k;
        require(in.mesh == t.instance_mesh[i] && in.material == t.instance_material[i],
                "An instance update keeps the instance's mesh and material");
        bool finite = true;
        for (int c = 0; c < 16; ++c) finite = finite && std::isfinite(in.object_to_world[c]);
        for (int c = 0; c < 9; ++c) finite = finite && std::isfinite(in.normal_to_world[c]);
        require(finite, "Transform must be finite");
        const DeviceInstance2& d = t.host_instances[i];
        if (d.flags & kTriEmissive) {
            require(std::memcmp(d.to_world, in.object_to_world, sizeof(d.to_world)) == 0 &&
                        std::memcmp(d.normal_to_world, in.normal_to_world, sizeof(d.normal_to_world)) == 0,
                    "Emissive instances are the scene's area lights and cannot move");
        }
    }
    try {
        for (uint32_t k = 0; k < count; ++k) {
            DeviceInstance2& d = t.host_instances[first + k];
            fill_instance_transform(instances[k], d);
            d.flags = (d.flags & ~kTriMirrored) | (determinant3(instances[k].object_to_world) < 0 ? kTriMirrored : 0u);
        }
        rebuild_after_refit(scene);
    } catch (...) {
        // A rejected update (a transform that collapses a triangle) leaves the scene as it was.
        t.host_instances = previous;
        rebuild_after_refit(scene);
        throw;
    }
}

namespace {

// Copies `count` positions (device) into mesh `mesh`'s range and refits its tree: the binary
// tree bottom-up, then the wide nodes it was collapsed into and the object-space slots.
void refit_mesh(Scene& scene, uint32_t mesh, const float* device_positions, cudaStream_t stream) {
    auto&     t  = *scene.two;
    MeshTree& mt = t.mesh[mesh];
    MR_CUDA(cudaMemcpyAsync(t.positions.ptr + 3ull * t.position_offset[mesh], device_positions,
                            3ull * mt.positions * sizeof(float), cudaMemcpyDeviceToDevice, stream));
    if (!t.used[mesh]) {
        return;
    }
    DeviceBuffer<float4>   lo, hi, centroid;
    DeviceBuffer<uint32_t> parent, arrivals;
    lo.allocate(mt.triangles);
    hi.allocate(mt.triangles);
    centroid.allocate(mt.triangles);
    parent.allocate(mt.node_count);
    arrivals.allocate(mt.node_count);
    mesh_bounds_kernel<<<grid(mt.triangles), 256, 0, stream>>>(
        t.positions.ptr + 3ull * t.position_offset[mesh], t.corners.ptr + t.corner_offset[mesh], mt.triangles,
        lo.ptr, hi.ptr, centroid.ptr);
    parents_kernel<<<grid(mt.node_count), 256, 0, stream>>>(mt.nodes.ptr, mt.node_count, parent.ptr);
    MR_CUDA(cudaMemsetAsync(arrivals.ptr, 0, mt.node_count * sizeof(uint32_t), stream));
    refit_kernel<<<grid(mt.node_count, 128), 128, 0, stream>>>(mt.nodes.ptr, mt.node_count, parent.ptr, mt.order.ptr,
                                                          lo.ptr, hi.ptr, arrivals.ptr);
    MR_CUDA(cudaGetLastError());
    // Same wide topology: each wide node takes its children's refit boxes.
    if (mt.wide_count) {
        refit_wide_kernel<<<grid(mt.wide_count, 128), 128, 0, stream>>>(mt.nodes.ptr, mt.wide_children.ptr,
                                                                   mt.wide_count,
                                                                   t.blas_nodes.ptr + 8ull * mt.node_base);
    }
    float4* slots = t.blas_tris.ptr + 3ull * mt.slot_base;
    mesh_slots_kernel<<<grid(mt.triangles), 256, 0, stream>>>(t.positions.ptr + 3ull * t.position_offset[mesh],
                                                               t.corners.ptr + t.corner_offset[mesh], mt.order.ptr,
                                                               mt.triangles, slots);
    mark_leaf_ends(mt.nodes.ptr, mt.node_count, slots, stream);
    MR_CUDA(cudaGetLastError());
    mr_bvh_node root{};
    MR_CUDA(cudaMemcpyAsync(&root, mt.nodes.ptr, sizeof(root), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    for (int a = 0; a < 3; ++a) {
        mt.box[a]     = root.minimum[a];
        mt.box[3 + a] = root.maximum[a];
    }
}

}  // namespace

void update_mesh(Scene& scene, uint32_t mesh, const float* positions, uint32_t position_count) {
    require(scene.two != nullptr, "Refit needs a scene built with two levels");
    auto& t = *scene.two;
    require(mesh < t.mesh.size(), "Mesh index is outside the scene");
    MeshTree& mt = t.mesh[mesh];
    require(positions != nullptr && position_count == mt.positions,
            "A mesh update keeps the mesh's position count");
    require(!t.emissive_mesh[mesh], "Meshes of emissive instances are area lights and cannot change");
    for (uint64_t k = 0; k < 3ull * position_count; ++k) {
        require(std::isfinite(positions[k]), "Mesh position must be finite");
    }
    struct OwnedStream {
        cudaStream_t stream = nullptr;
        OwnedStream() { MR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); }
        ~OwnedStream() { cudaStreamDestroy(stream); }
    } owned;
    cudaStream_t    stream = owned.stream;
    AllocationScope scope(stream);
    // The new positions pass MeshData::validate's degenerate-triangle check before anything
    // changes; the previous ones are kept to restore the scene if the world-space checks reject
    // the update.
    DeviceBuffer<float> fresh, previous;
    fresh.allocate(3ull * position_count);
    previous.allocate(3ull * position_count);
    MR_CUDA(cudaMemcpyAsync(fresh.ptr, positions, 3ull * position_count * sizeof(float), cudaMemcpyHostToDevice,
                            stream));
    MR_CUDA(cudaMemcpyAsync(previous.ptr, t.positions.ptr + 3ull * t.position_offset[mesh],
                            3ull * position_count * sizeof(float), cudaMemcpyDeviceToDevice, stream));
    {
        DeviceBuffer<float4>   lo, hi, centroid;
        DeviceBuffer<unsigned> error;
        lo.allocate(mt.triangles);
        hi.allocate(mt.triangles);
        centroid.allocate(mt.triangles);
        error.allocate(1);
        MR_CUDA(cudaMemsetAsync(error.ptr, 0, sizeof(unsigned), stream));
        mesh_bounds_kernel<<<grid(mt.triangles), 256, 0, stream>>>(fresh.ptr, t.corners.ptr + t.corner_offset[mesh],
                                                                  mt.triangles, lo.ptr, hi.ptr, centroid.ptr,
                                                                  error.ptr);
        unsigned bad = 0;
        MR_CUDA(cudaMemcpyAsync(&bad, error.ptr, sizeof(bad), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        require(!bad, "Degenerate mesh triangle");
    }
    try {
        refit_mesh(scene, mesh, fresh.ptr, stream);
        rebuild_after_refit(scene);
    } catch (...) {
        refit_mesh(scene, mesh, previous.ptr, stream);
        rebuild_after_refit(scene);
        throw;
    }
}

void rebuild_after_refit(Scene& scene) {
    struct OwnedStream {
        cudaStream_t stream = nullptr;
        OwnedStream() { MR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); }
        ~OwnedStream() { cudaStreamDestroy(stream); }
    } owned;
    cudaStream_t    stream = owned.stream;
    AllocationScope scope(stream);
    build_instance_tree(scene, stream);
    publish_two_level(scene);
    upload_light_table(scene, scene.two->world_lo, scene.two->world_hi, stream);
    MR_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace mr
