// traverse.cuh — FP32 ray queries over the BVH: slab test, watertight triangle test, nearest and
// any-hit traversal.
//
// Semantics follow the reference exactly (src/render/intersection.cpp, src/render/bvh.cpp:206-300):
// closed intervals, ties to the lower primitive id, single-sided culling by geometric winding,
// any-hit exit on the first accepted triangle, pruning of popped subtrees whose entry distance
// exceeds the current nearest hit. Differences are numeric only:
//  - slab distances are widened by 2^-20 relative instead of one double ulp, so the box test
//    stays conservative in FP32 (FP32 rounding of (b - o) * inv is at most a few ulps);
//  - the triangle test is the same permute/shear/difference-of-products algorithm in FP32 with
//    the error bound of the reference evaluated with FP32's unit roundoff.
#pragma once

#include "device_scene.cuh"

namespace mr {

// A wide node pushes <= 3 entries and sits at most 63 levels deep (built trees stop at 48,
// bvh.cpp:16; imported trees are refused beyond 64 levels), so at most 3 * 63 entries are
// stacked before any push: the check `sp > kStackSize - 3` never fires on an accepted tree.
constexpr int      kStackSize  = 195;
constexpr uint32_t kMaxVisits  = 1u << 16;  // node visits per ray before the query gives up

struct RayQuery {
    f3    o, d;
    float inv_lo[3];  // 1/d scaled down by 2^-20: near slab distances round toward the origin
    float inv_hi[3];  // 1/d scaled up by 2^-20: far slab distances round away
    bool  neg[3];     // direction sign per axis (the near slab is the max bound)
    int   kx, ky, kz;
    float sx, sy, sz;

    __device__ __forceinline__ void init(f3 origin, f3 direction) {
        o = origin;
        d = direction;
        const float lo = 0.99999904632568359375f;  // 1 - 2^-20
        const float hi = 1.00000095367431640625f;  // 1 + 2^-20
        for (int a = 0; a < 3; ++a) {
            const float c = comp(d, a);
            const float inv = 1.0f / c;  // +-inf for +-0: the slab then imposes no bound
            inv_lo[a] = inv * lo;
            inv_hi[a] = inv * hi;
            neg[a]    = signbit(c);
        }
        // Permutation and shear (src/render/intersection.cpp:62-74).
        const f3 ad = fabs3(d);
        kz          = ad.x > ad.y ? 0 : 1;
        if (ad.z > comp(ad, kz)) {
            kz = 2;
        }
        kx = kz == 2 ? 0 : kz + 1;
        ky = kx == 2 ? 0 : kx + 1;
        if (comp(d, kz) < 0) {
            const int t = kx;
            kx          = ky;
            ky          = t;
        }
        const float dz = comp(d, kz);
        sx             = comp(d, kx) / dz;
        sy             = comp(d, ky) / dz;
        sz             = 1.0f / dz;
    }
};

// Entry distance of one child box, or NaN when the slab intervals do not overlap within
// [tmin, tmax] (NaN compares false against every interval end, +inf would not for tmax = inf). `xy` = (lo.x, hi.x, lo.y, hi.y); (zlo, zhi) the z extent.
__device__ __forceinline__ float slab_enter(const RayQuery& q, float4 xy, float zlo, float zhi,
                                            float tmin, float tmax) {
    const float nx = ((q.neg[0] ? xy.y : xy.x) - q.o.x) * q.inv_lo[0];
    const float fx = ((q.neg[0] ? xy.x : xy.y) - q.o.x) * q.inv_hi[0];
    const float ny = ((q.neg[1] ? xy.w : xy.z) - q.o.y) * q.inv_lo[1];
    const float fy = ((q.neg[1] ? xy.z : xy.w) - q.o.y) * q.inv_hi[1];
    const float nz = ((q.neg[2] ? zhi : zlo) - q.o.z) * q.inv_lo[2];
    const float fz = ((q.neg[2] ? zlo : zhi) - q.o.z) * q.inv_hi[2];
    // fmaxf/fminf ignore the NaN of 0 * inf (origin on the slab plane of a zero component).
    const float enter = fmaxf(fmaxf(tmin, nx), fmaxf(ny, nz));
    const float leave = fminf(fminf(tmax, fx), fminf(fy, fz));
    return enter <= leave ? enter : __int_as_float(0x7fffffff);
}

// Slab test of one child of a wide node from its near and far planes per axis (already chosen by
// the ray's direction signs): the entry distance, or +inf when missed. A hit's entry is at most
// `tmax` (leave <= tmax), and +inf is also what an unbounded entry means, so interior traversal
// treats +inf as "no child" without a second comparison against the interval.
__device__ __forceinline__ float slab_near_far(const RayQuery& q, float nx, float fx, float ny, float fy,
                                               float nz, float fz, float tmin, float tmax) {
    const float tnx = (nx - q.o.x) * q.inv_lo[0];
    const float tfx = (fx - q.o.x) * q.inv_hi[0];
    const float tny = (ny - q.o.y) * q.inv_lo[1];
    const float tfy = (fy - q.o.y) * q.inv_hi[1];
    const float tnz = (nz - q.o.z) * q.inv_lo[2];
    const float tfz = (fz - q.o.z) * q.inv_hi[2];
    const float enter = fmaxf(fmaxf(tmin, tnx), fmaxf(tny, tnz));
    const float leave = fminf(fminf(tmax, tfx), fminf(tfy, tfz));
    return enter <= leave ? enter : __int_as_float(0x7f800000);
}

__device__ __forceinline__ void order2(float& ta, int& ra, float& tb, int& rb) {
    if (tb < ta) {
        const float t = ta;
        ta            = tb;
        tb            = t;
        const int r   = ra;
        ra            = rb;
        rb            = r;
    }
}

__device__ __forceinline__ float permuted(f3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Watertight triangle test (src/render/intersection.cpp:108-152) in FP32. On acceptance returns
// the distance and the three unnormalised edge functions plus their sum (the determinant).
__device__ __forceinline__ bool triangle_test(const RayQuery& q, f3 v0, f3 v1, f3 v2, float tmin,
                                              float tmax, float& t, float& ea, float& eb,
                                              float& ec, float& det) {
    const f3 t0 = v0 - q.o, t1 = v1 - q.o, t2 = v2 - q.o;
    const float z0 = permuted(t0, q.kz), z1 = permuted(t1, q.kz), z2 = permuted(t2, q.kz);
    const float p0x = fmaf(-q.sx, z0, permuted(t0, q.kx));
    const float p0y = fmaf(-q.sy, z0, permuted(t0, q.ky));
    const float p1x = fmaf(-q.sx, z1, permuted(t1, q.kx));
    const float p1y = fmaf(-q.sy, z1, permuted(t1, q.ky));
    const float p2x = fmaf(-q.sx, z2, permuted(t2, q.kx));
    const float p2y = fmaf(-q.sy, z2, permuted(t2, q.ky));
    const float a = difference_of_products(p1x, p2y, p1y, p2x);
    const float b = difference_of_products(p2x, p0y, p2y, p0x);
    const float c = difference_of_products(p0x, p1y, p0y, p1x);
    if ((a < 0 || b < 0 || c < 0) && (a > 0 || b > 0 || c > 0)) {
        return false;
    }
    const float determinant = a + b + c;
    if (determinant == 0) {
        return false;
    }
    const float pz0 = z0 * q.sz, pz1 = z1 * q.sz, pz2 = z2 * q.sz;
    const float distance = __fdiv_rn(a * pz0 + b * pz1 + c * pz2, determinant);
    if (!(distance >= tmin && distance <= tmax)) {
        return false;
    }
    // Error bound of PBRT 4 section 6.5.3 with FP32's unit roundoff u = 2^-24.
    constexpr float g2 = 2.0f * 5.9604644775390625e-08f / (1.0f - 2.0f * 5.9604644775390625e-08f);
    constexpr float g3 = 3.0f * 5.9604644775390625e-08f / (1.0f - 3.0f * 5.9604644775390625e-08f);
    constexpr float g5 = 5.0f * 5.9604644775390625e-08f / (1.0f - 5.0f * 5.9604644775390625e-08f);
    const float x = fmaxf(fmaxf(fabsf(p0x), fabsf(p1x)), fabsf(p2x));
    const float y = fmaxf(fmaxf(fabsf(p0y), fabsf(p1y)), fabsf(p2y));
    const float z = fmaxf(fmaxf(fabsf(pz0), fabsf(pz1)), fabsf(pz2));
    const float error_x    = g5 * (x + z);
    const float error_y    = g5 * (y + z);
    const float error_edge = 2.0f * (g2 * x * y + error_y * x + error_x * y);
    const float edge       = fmaxf(fmaxf(fabsf(a), fabsf(b)), fabsf(c));
    const float error_distance =
        3.0f * (g3 * edge * z + error_edge * z + g3 * z * edge) / fabsf(determinant);
    if (distance <= error_distance) {
        return false;
    }
    t   = distance;
    ea  = a;
    eb  = b;
    ec  = c;
    det = determinant;
    return true;
}

struct TraceResult {
    float    t;
    uint32_t slot;  // triangle slot in leaf order (two-level scenes: the primitive), kNone: miss
    uint32_t prim;
    float    a, b, c, det;
    uint32_t flags;  // two-level scenes: the hit instance's flags
};

struct TraceCounters {
    uint32_t bounds;
    uint32_t triangles;
};

// Nearest hit (ANY_HIT = false) or occlusion (ANY_HIT = true) in [tmin, tmax].
// Lanes of a warp traverse interior nodes together and postpone the first leaf they reach until
// every active lane holds one (or has finished), then test leaves together: interior and leaf
// work are not interleaved across lanes.
template <bool ANY_HIT>
__device__ __forceinline__ TraceResult trace(const DeviceScene& s, const RayQuery& q, float tmin,
                                             float tmax, TraceCounters& counters,
                                             unsigned& error) {
    TraceResult result;
    result.t    = tmax;
    result.slot = kNone;
    result.prim = kNone;
    if (!s.has_nodes) {
        return result;
    }
    if (!(finite3(q.o) && finite3(q.d))) {
        error |= kErrorRay;
        return result;
    }
    counters.bounds++;
    const float root_enter =
        slab_enter(q, make_float4(s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1]),
                   s.root_lo[2], s.root_hi[2], tmin, tmax);
    if (!(root_enter <= tmax)) {
        return result;
    }
    int2     stack[kStackSize];
    int      sp     = 0;
    int      node   = s.root;  // next node to visit (interior >= 0, leaf < 0)
    bool     alive  = true;    // `node` is valid
    int      leaf   = 0;
    bool     held   = false;   // a postponed leaf in `leaf`
    uint32_t visits = 0;
    const float inf = __int_as_float(0x7f800000);
    // Node rows 0..5 are lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of the four children: the near plane
    // of an axis is its hi row when the direction is negative there.
    const int near_x = q.neg[0] ? 1 : 0, near_y = q.neg[1] ? 3 : 2, near_z = q.neg[2] ? 5 : 4;
    // Next stacked subtree that can still contain a nearer hit, or none.
    const auto pop = [&]() {
        while (sp > 0) {
            const int2 e = stack[--sp];
            if (__int_as_float(e.y) <= result.t) {
                node = e.x;
                return;
            }
        }
        alive = false;
    };
    // Every pass of every loop below visits a node or tests a leaf, and both count against
    // kMaxVisits, so traversal ends on any input.
    while (alive || held) {
        if (alive && node < 0 && !held) {  // a leaf to test next (also a root that is a leaf)
            leaf = node;
            held = true;
            pop();
        }
        // Interior phase.
        while (alive && node >= 0) {
            if (++visits > kMaxVisits) {
                error |= kErrorVisits;
                return result;
            }
            const float4* n   = s.nodes + 8 * static_cast<size_t>(node);
            const float4  nx  = __ldg(n + near_x), fx = __ldg(n + (near_x ^ 1));
            const float4  ny  = __ldg(n + near_y), fy = __ldg(n + (near_y ^ 1));
            const float4  nz  = __ldg(n + near_z), fz = __ldg(n + (near_z ^ 1));
            const int4    ref = __ldg(reinterpret_cast<const int4*>(n + 6));
            counters.bounds += static_cast<uint32_t>(__ldg(reinterpret_cast<const int*>(n + 7)));
            float t0 = slab_near_far(q, nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, tmin, result.t);
            float t1 = slab_near_far(q, nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, tmin, result.t);
            float t2 = slab_near_far(q, nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, tmin, result.t);
            float t3 = slab_near_far(q, nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, tmin, result.t);
            int r0 = ref.x, r1 = ref.y, r2 = ref.z, r3 = ref.w;
            order2(t0, r0, t1, r1);
            order2(t2, r2, t3, r3);
            order2(t0, r0, t2, r2);
            order2(t1, r1, t3, r3);
            order2(t1, r1, t2, r2);
            if (t0 != inf) {
                if (sp > kStackSize - 3) {
                    error |= kErrorStack;
                    return result;
                }
                if (t3 != inf) {
                    stack[sp++] = make_int2(r3, __float_as_int(t3));
                }
                if (t2 != inf) {
                    stack[sp++] = make_int2(r2, __float_as_int(t2));
                }
                if (t1 != inf) {
                    stack[sp++] = make_int2(r1, __float_as_int(t1));
                }
                node = r0;
            } else {
                pop();
            }
            if (alive && node < 0 && !held) {  // postpone the first leaf and keep descending
                leaf = node;
                held = true;
                pop();
            }
            if (!__any_sync(__activemask(), !held)) {
                break;  // every lane here holds a leaf
            }
        }
        // Leaf phase: the postponed leaf, then any leaf the lane now points at.
        while (held) {
            if (++visits > kMaxVisits) {
                error |= kErrorVisits;
                return result;
            }
            for (uint32_t slot = static_cast<uint32_t>(~leaf);; ++slot) {
                const float4* tp = s.tris + 3 * static_cast<size_t>(slot);
                const float4  a4 = __ldg(tp + 0);
                const float4  b4 = __ldg(tp + 1);
                const float4  c4 = __ldg(tp + 2);
                const unsigned flags = __float_as_uint(b4.w);
                counters.triangles++;
                float t, ea, eb, ec, det;
                if (triangle_test(q, xyz(a4), xyz(b4), xyz(c4), tmin, result.t, t, ea, eb, ec,
                                  det)) {
                    bool visible = true;
                    if (flags & kTriSingleSided) {
                        const f3 outward = cross(xyz(b4) - xyz(a4), xyz(c4) - xyz(a4));
                        const float side = dot(q.d, outward);
                        visible = (flags & kTriMirrored) ? side > 0 : side < 0;
                    }
                    const uint32_t prim = __float_as_uint(a4.w);
                    if (visible && (t < result.t || (t == result.t && prim < result.prim) ||
                                    result.slot == kNone)) {
                        result.t    = t;
                        result.slot = slot;
                        result.prim = prim;
                        result.a    = ea;
                        result.b    = eb;
                        result.c    = ec;
                        result.det  = det;
                        if (ANY_HIT) {
                            return result;
                        }
                    }
                }
                if (flags & kTriLeafEnd) {
                    break;
                }
            }
            held = false;
            if (alive && node < 0) {
                leaf = node;
                held = true;
                pop();
            }
        }
    }
    return result;
}

// ---- two-level scenes ----

// The world ray mapped into an instance's object space (same parameter t: the direction is not
// renormalised), for slab tests against the instance's mesh boxes grown by `margin` on every
// side. The growth is folded into the origin per axis: o_near/o_far are the origins the near and
// far planes are measured from. It covers the rounding of this mapping and of the flattening's
// FP32 world vertices (whose world-space triangles are the ones tested), so a box that a
// world-space triangle of the instance hits is never culled.
struct ObjectRay {
    float o_near[3], o_far[3];
    float inv_lo[3], inv_hi[3];
    bool  neg[3];
};

constexpr float kInstanceMarginScale = 1.9073486328125e-06f;  // 2^-19 = 32 FP32 unit roundoffs

__device__ __forceinline__ void object_ray(const DeviceInstance2& inst, const RayQuery& qw,
                                           float t_exit, ObjectRay& r) {
    const float* m = inst.to_object;
    const f3 o = {fmaf(m[0], qw.o.x, fmaf(m[1], qw.o.y, fmaf(m[2], qw.o.z, m[3]))),
                  fmaf(m[4], qw.o.x, fmaf(m[5], qw.o.y, fmaf(m[6], qw.o.z, m[7]))),
                  fmaf(m[8], qw.o.x, fmaf(m[9], qw.o.y, fmaf(m[10], qw.o.z, m[11])))};
    const f3 d = {fmaf(m[0], qw.d.x, fmaf(m[1], qw.d.y, m[2] * qw.d.z)),
                  fmaf(m[4], qw.d.x, fmaf(m[5], qw.d.y, m[6] * qw.d.z)),
                  fmaf(m[8], qw.d.x, fmaf(m[9], qw.d.y, m[10] * qw.d.z))};
    const float reach  = max3(fabs3(qw.o)) + t_exit * max3(fabs3(qw.d));
    const float margin = inst.margin_static +
                         kInstanceMarginScale * (fmaf(inst.a_norm, reach, inst.b_norm));
    const float lo = 0.99999904632568359375f, hi = 1.00000095367431640625f;  // 1 -+ 2^-20
    for (int a = 0; a < 3; ++a) {
        const float c   = comp(d, a);
        const float inv = 1.0f / c;
        r.inv_lo[a]     = inv * lo;
        r.inv_hi[a]     = inv * hi;
        r.neg[a]        = signbit(c);
        const float oa  = comp(o, a);
        r.o_near[a]     = r.neg[a] ? oa - margin : oa + margin;
        r.o_far[a]      = r.neg[a] ? oa + margin : oa - margin;
    }
}

__device__ __forceinline__ float object_slab(const ObjectRay& r, float nx, float fx, float ny, float fy,
                                             float nz, float fz, float tmin, float tmax) {
    const float tnx = (nx - r.o_near[0]) * r.inv_lo[0];
    const float tfx = (fx - r.o_far[0]) * r.inv_hi[0];
    const float tny = (ny - r.o_near[1]) * r.inv_lo[1];
    const float tfy = (fy - r.o_far[1]) * r.inv_hi[1];
    const float tnz = (nz - r.o_near[2]) * r.inv_lo[2];
    const float tfz = (fz - r.o_far[2]) * r.inv_hi[2];
    const float enter = fmaxf(fmaxf(tmin, tnx), fmaxf(tny, tnz));
    const float leave = fminf(fminf(tmax, tfx), fminf(tfy, tfz));
    return enter <= leave ? enter : __int_as_float(0x7f800000);
}

// Entry and exit of a world box, or false when the ray misses it within [tmin, tmax].
__device__ __forceinline__ bool world_box(const RayQuery& q, const float* lo, const float* hi,
                                          float tmin, float tmax, float& enter, float& leave) {
    const float nx = ((q.neg[0] ? hi[0] : lo[0]) - q.o.x) * q.inv_lo[0];
    const float fx = ((q.neg[0] ? lo[0] : hi[0]) - q.o.x) * q.inv_hi[0];
    const float ny = ((q.neg[1] ? hi[1] : lo[1]) - q.o.y) * q.inv_lo[1];
    const float fy = ((q.neg[1] ? lo[1] : hi[1]) - q.o.y) * q.inv_hi[1];
    const float nz = ((q.neg[2] ? hi[2] : lo[2]) - q.o.z) * q.inv_lo[2];
    const float fz = ((q.neg[2] ? lo[2] : hi[2]) - q.o.z) * q.inv_hi[2];
    enter = fmaxf(fmaxf(tmin, nx), fmaxf(ny, nz));
    leave = fminf(fminf(tmax, fx), fminf(fy, fz));
    return enter <= leave;
}

// Wide-node children of `node` tested with `test(nx, fx, ny, fy, nz, fz)` (the near/far plane
// rows picked by `near`), ordered nearest first. Returns the child count hit (<= 4) with refs and
// entries in r[] / t[].
template <typename Test>
__device__ __forceinline__ void wide_children(const float4* nodes, int node, const int near[3],
                                              Test test, float t[4], int r[4], uint32_t& bounds) {
    const float4* n   = nodes + 8 * static_cast<size_t>(node);
    const float4  nx  = __ldg(n + near[0]), fx = __ldg(n + (near[0] ^ 1));
    const float4  ny  = __ldg(n + near[1]), fy = __ldg(n + (near[1] ^ 1));
    const float4  nz  = __ldg(n + near[2]), fz = __ldg(n + (near[2] ^ 1));
    const int4    ref = __ldg(reinterpret_cast<const int4*>(n + 6));
    bounds += static_cast<uint32_t>(__ldg(reinterpret_cast<const int*>(n + 7)));
    t[0] = test(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x);
    t[1] = test(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y);
    t[2] = test(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z);
    t[3] = test(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w);
    r[0] = ref.x, r[1] = ref.y, r[2] = ref.z, r[3] = ref.w;
    order2(t[0], r[0], t[1], r[1]);
    order2(t[2], r[2], t[3], r[3]);
    order2(t[0], r[0], t[2], r[2]);
    order2(t[1], r[1], t[3], r[3]);
    order2(t[1], r[1], t[2], r[2]);
}

// A wide node's or a lone leaf's stack discipline: a stack of (ref, entry) pairs shared by the
// two levels; entries beyond the current nearest hit are skipped when popped.
constexpr int kStackSize2 = 3 * 64 * 2 + 3;

// Nearest hit / occlusion in a two-level scene. The instance-level tree is traversed with the
// world ray; an instance whose world box the ray enters has its mesh tree traversed with the
// ray mapped into object space, and every candidate triangle is transformed to world space with
// the flattening's arithmetic (transform_point) and tested with the world ray: the same vertices,
// ray and test as the flattened scene, so the same hits (ties still go to the lower flat
// primitive id).
template <bool ANY_HIT>
__device__ __forceinline__ TraceResult trace2(const DeviceScene& s, const RayQuery& q, float tmin,
                                           float tmax, TraceCounters& counters, unsigned& error) {
    TraceResult result;
    result.t     = tmax;
    result.slot  = kNone;
    result.prim  = kNone;
    result.flags = 0;
    if (!s.has_nodes) {
        return result;
    }
    if (!(finite3(q.o) && finite3(q.d))) {
        error |= kErrorRay;
        return result;
    }
    counters.bounds++;
    float enter, leave;
    if (!world_box(q, s.root_lo, s.root_hi, tmin, tmax, enter, leave)) {
        return result;
    }
    int2     stack[kStackSize2];
    int      sp     = 0;
    uint32_t visits = 0;
    const float inf = __int_as_float(0x7f800000);
    const int near_w[3] = {q.neg[0] ? 1 : 0, q.neg[1] ? 3 : 2, q.neg[2] ? 5 : 4};
    stack[sp++] = make_int2(s.root, __float_as_int(enter));
    while (sp > 0) {
        const int2 top = stack[--sp];
        if (__int_as_float(top.y) > result.t) {
            continue;
        }
        if (++visits > kMaxVisits) {
            error |= kErrorVisits;
            return result;
        }
        const int node = top.x;
        if (node >= 0) {  // instance-level interior node
            float t[4];
            int   r[4];
            wide_children(s.nodes, node, near_w,
                          [&](float nx, float fx, float ny, float fy, float nz, float fz) {
                              return slab_near_far(q, nx, fx, ny, fy, nz, fz, tmin, result.t);
                          },
                          t, r, counters.bounds);
            if (sp > kStackSize2 - 4) {
                error |= kErrorStack;
                return result;
            }
            for (int k = 3; k >= 0; --k) {
                if (t[k] != inf) {
                    stack[sp++] = make_int2(r[k], __float_as_int(t[k]));
                }
            }
            continue;
        }
        // Instance-level leaf: its instances in order.
        for (uint32_t item = static_cast<uint32_t>(~node);; ++item) {
            const uint32_t         word = __ldg(s.tlas_items + item);
            const DeviceInstance2& inst = s.instances[word & 0x7fffffffu];
            counters.bounds++;
            float ienter, ileave;
            if (world_box(q, inst.lo, inst.hi, tmin, result.t, ienter, ileave)) {
                ObjectRay ro;
                object_ray(inst, q, ileave, ro);
                const int near_o[3] = {ro.neg[0] ? 1 : 0, ro.neg[1] ? 3 : 2, ro.neg[2] ? 5 : 4};
                const int base = sp;
                stack[sp++] = make_int2(inst.blas_root, __float_as_int(ienter));
                while (sp > base) {
                    const int2 e = stack[--sp];
                    if (__int_as_float(e.y) > result.t) {
                        continue;
                    }
                    if (++visits > kMaxVisits) {
                        error |= kErrorVisits;
                        return result;
                    }
                    if (e.x >= 0) {  // mesh-level interior node
                        float t[4];
                        int   r[4];
                        wide_children(s.blas_nodes, e.x, near_o,
                                      [&](float nx, float fx, float ny, float fy, float nz, float fz) {
                                          return object_slab(ro, nx, fx, ny, fy, nz, fz, tmin, result.t);
                                      },
                                      t, r, counters.bounds);
                        if (sp > kStackSize2 - 4) {
                            error |= kErrorStack;
                            return result;
                        }
                        for (int k = 3; k >= 0; --k) {
                            if (t[k] != inf) {
                                stack[sp++] = make_int2(r[k], __float_as_int(t[k]));
                            }
                        }
                        continue;
                    }
                    // Mesh-level leaf: its triangles, transformed to world space.
                    for (uint32_t slot = static_cast<uint32_t>(~e.x);; ++slot) {
                        const float4* tp = s.blas_tris + 3 * static_cast<size_t>(slot);
                        const float4  a4 = __ldg(tp + 0);
                        const float4  b4 = __ldg(tp + 1);
                        const float4  c4 = __ldg(tp + 2);
                        const f3 v0 = transform_point(inst.to_world, a4.x, a4.y, a4.z);
                        const f3 v1 = transform_point(inst.to_world, b4.x, b4.y, b4.z);
                        const f3 v2 = transform_point(inst.to_world, c4.x, c4.y, c4.z);
                        counters.triangles++;
                        float tt, ea, eb, ec, det;
                        if (triangle_test(q, v0, v1, v2, tmin, result.t, tt, ea, eb, ec, det)) {
                            bool visible = true;
                            if (inst.flags & kTriSingleSided) {
                                const float side = dot(q.d, cross(v1 - v0, v2 - v0));
                                visible = (inst.flags & kTriMirrored) ? side > 0 : side < 0;
                            }
                            const uint32_t prim = inst.first_prim + __float_as_uint(a4.w);
                            if (visible && (tt < result.t || (tt == result.t && prim < result.prim) ||
                                            result.slot == kNone)) {
                                result.t     = tt;
                                result.slot  = prim;
                                result.prim  = prim;
                                result.a     = ea;
                                result.b     = eb;
                                result.c     = ec;
                                result.det   = det;
                                result.flags = inst.flags;
                                if (ANY_HIT) {
                                    return result;
                                }
                            }
                        }
                        if (__float_as_uint(b4.w) & kTriLeafEnd) {
                            break;
                        }
                    }
                }
            }
            if (word & 0x80000000u) {
                break;
            }
        }
    }
    return result;
}

}  // namespace mr
