// split.cu — early split clipping of oversized triangles before the binned-SAH build.
//
// The reference's builder (src/render/bvh.cpp:101-196) bins whole triangles by centroid. In a
// scene of many small triangles and a few huge ones (the walls of a room around detailed
// objects) the huge triangles' centroids fall among the small ones, so every node above a huge
// triangle's leaf inherits its box, and rays test those large boxes again and again. Splitting
// references fixes the tree without changing any result: a triangle whose box is much larger
// than the scene's typical triangle box enters the build several times, each reference carrying
// the bounds of the triangle clipped to one cell of a grid laid over its box. Every reference
// points at the same triangle, so traversal tests the same triangle with the same arithmetic;
// nearest hits (ties broken by primitive id) and occlusion answers are those of the unsplit tree.
//
// Reference bounds are the clipped polygon's bounds widened by 2^-18 of the coordinate magnitude
// plus the triangle's extent (FP32 clipping error is far below that), then clamped to the
// triangle's exact box, so the references of a triangle always cover all of it.
#include <cmath>

#include "errors.hpp"
#include "scan.cuh"
#include "scene.cuh"

namespace mr {

namespace {

constexpr int kMaxCellsPerAxis     = 64;
constexpr int kMaxCellsPerTriangle = 4096;

__device__ __forceinline__ float axis_of(const f3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ void  set_axis(f3& v, int a, float x) {
    if (a == 0) {
        v.x = x;
    } else if (a == 1) {
        v.y = x;
    } else {
        v.z = x;
    }
}

__device__ __forceinline__ float box_area(float ex, float ey, float ez) {
    return 2.0f * (ex * ey + ey * ez + ez * ex);
}

// Grid over a triangle box whose cells have about `target` surface area each. Axes thinner than
// 1/64 of the longest are not divided.
__device__ void grid_dims(float4 lo, float4 hi, float target, int n[3]) {
    const float e[3] = {hi.x - lo.x, hi.y - lo.y, hi.z - lo.z};
    n[0] = n[1] = n[2] = 1;
    const float area = box_area(e[0], e[1], e[2]);
    if (!(area > target)) {
        return;
    }
    const float emax = fmaxf(e[0], fmaxf(e[1], e[2]));
    float       prod = 1.0f;
    int         d    = 0;
    for (int a = 0; a < 3; ++a) {
        if (e[a] >= emax * (1.0f / 64.0f)) {
            prod *= e[a];
            ++d;
        }
    }
    const float k    = fminf(ceilf(area / target), static_cast<float>(kMaxCellsPerTriangle));
    const float side = d == 1 ? prod / k : (d == 2 ? sqrtf(prod / k) : cbrtf(prod / k));
    int         total = 1;
    for (int a = 0; a < 3; ++a) {
        if (e[a] >= emax * (1.0f / 64.0f) && side > 0) {
            n[a] = max(1, min(kMaxCellsPerAxis, __float2int_rn(e[a] / side)));
        }
        total *= n[a];
    }
    while (total > kMaxCellsPerTriangle) {  // keep the product within the cap
        const int a = n[0] >= n[1] && n[0] >= n[2] ? 0 : (n[1] >= n[2] ? 1 : 2);
        n[a]        = (n[a] + 1) / 2;
        total       = n[0] * n[1] * n[2];
    }
}

// Boundary i of n cells over [lo, hi]: the same expression for both neighbours of a boundary,
// so the cells tile the box exactly.
__device__ __forceinline__ float boundary(float lo, float hi, int i, int n) {
    if (i <= 0) {
        return lo;
    }
    if (i >= n) {
        return hi;
    }
    return lo + (hi - lo) * (static_cast<float>(i) / static_cast<float>(n));
}

// Sutherland-Hodgman clip of a convex polygon against one axis-aligned half-space.
__device__ int clip(const f3* in, int count, f3* out, int axis, float plane, bool keep_above) {
    int m = 0;
    for (int i = 0; i < count; ++i) {
        const f3    p  = in[i];
        const f3    q  = in[i + 1 == count ? 0 : i + 1];
        const float dp = axis_of(p, axis) - plane;
        const float dq = axis_of(q, axis) - plane;
        const bool  ip = keep_above ? dp >= 0 : dp <= 0;
        const bool  iq = keep_above ? dq >= 0 : dq <= 0;
        if (ip) {
            out[m++] = p;
        }
        if (ip != iq) {
            const float t = dp / (dp - dq);
            f3          x = p + (q - p) * t;
            set_axis(x, axis, plane);
            out[m++] = x;
        }
    }
    return m;
}

__global__ void area_kernel(const float4* lo, const float4* hi, uint32_t count, double* sum, float* max_area) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float          a = 0;
    if (i < count) {
        const float4 l = lo[i], h = hi[i];
        a = box_area(h.x - l.x, h.y - l.y, h.z - l.z);
    }
    float s = a, m = a;
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sum, static_cast<double>(s));
        atomicMax(reinterpret_cast<int*>(max_area), __float_as_int(m));  // nonnegative floats
    }
}

__global__ void cell_count_kernel(const float4* lo, const float4* hi, uint32_t count, float target,
                                  uint32_t* cells) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        int n[3];
        grid_dims(lo[i], hi[i], target, n);
        cells[i] = static_cast<uint32_t>(n[0] * n[1] * n[2]);
    }
}

// One thread per cell: the clipped bounds of the cell's part of the triangle, or nothing.
__global__ void cell_write_kernel(const float4* world, const float4* lo, const float4* hi,
                                  const uint32_t* offsets, uint32_t prims, uint32_t cells, float target,
                                  float4* rlo, float4* rhi, uint32_t* rprim, uint32_t* valid) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) {
        return;
    }
    uint32_t a = 0, b = prims - 1;  // last prim with offsets[p] <= c
    while (a < b) {
        const uint32_t mid = (a + b + 1) >> 1;
        if (offsets[mid] <= c) {
            a = mid;
        } else {
            b = mid - 1;
        }
    }
    const uint32_t p  = a;
    const float4   tl = lo[p], th = hi[p];
    int            n[3];
    grid_dims(tl, th, target, n);
    const uint32_t k  = c - offsets[p];
    const int      ix = static_cast<int>(k % n[0]);
    const int      iy = static_cast<int>((k / n[0]) % n[1]);
    const int      iz = static_cast<int>(k / (n[0] * n[1]));
    rprim[c]          = p;
    if (n[0] * n[1] * n[2] == 1) {
        rlo[c]   = tl;
        rhi[c]   = th;
        valid[c] = 1;
        return;
    }
    f3 poly[9], tmp[9];
    poly[0] = xyz(world[3 * p + 0]);
    poly[1] = xyz(world[3 * p + 1]);
    poly[2] = xyz(world[3 * p + 2]);
    int         m     = 3;
    const int   idx[3] = {ix, iy, iz};
    const float blo[3] = {tl.x, tl.y, tl.z}, bhi[3] = {th.x, th.y, th.z};
    for (int axis = 0; axis < 3 && m > 0; ++axis) {
        if (n[axis] == 1) {
            continue;
        }
        if (idx[axis] > 0) {
            m = clip(poly, m, tmp, axis, boundary(blo[axis], bhi[axis], idx[axis], n[axis]), true);
            for (int v = 0; v < m; ++v) {
                poly[v] = tmp[v];
            }
        }
        if (m > 0 && idx[axis] < n[axis] - 1) {
            m = clip(poly, m, tmp, axis, boundary(blo[axis], bhi[axis], idx[axis] + 1, n[axis]), false);
            for (int v = 0; v < m; ++v) {
                poly[v] = tmp[v];
            }
        }
    }
    if (m == 0) {
        valid[c] = 0;
        return;
    }
    f3 l = poly[0], h = poly[0];
    for (int v = 1; v < m; ++v) {
        l = f3{fminf(l.x, poly[v].x), fminf(l.y, poly[v].y), fminf(l.z, poly[v].z)};
        h = f3{fmaxf(h.x, poly[v].x), fmaxf(h.y, poly[v].y), fmaxf(h.z, poly[v].z)};
    }
    const float ext = fmaxf(th.x - tl.x, fmaxf(th.y - tl.y, th.z - tl.z));
    const auto  widen_lo = [&](float v, float bound) {
        return fmaxf(bound, v - (fabsf(v) + ext) * 3.814697265625e-6f);  // 2^-18
    };
    const auto widen_hi = [&](float v, float bound) {
        return fminf(bound, v + (fabsf(v) + ext) * 3.814697265625e-6f);
    };
    rlo[c]   = make_float4(widen_lo(l.x, tl.x), widen_lo(l.y, tl.y), widen_lo(l.z, tl.z), 0.0f);
    rhi[c]   = make_float4(widen_hi(h.x, th.x), widen_hi(h.y, th.y), widen_hi(h.z, th.z), 0.0f);
    valid[c] = 1;
}

__global__ void compact_refs_kernel(const float4* rlo, const float4* rhi, const uint32_t* rprim,
                                    const uint32_t* valid, const uint32_t* slot, uint32_t cells,
                                    float4* lo, float4* hi, float4* centroid, uint32_t* prim) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < cells && valid[c]) {
        const uint32_t s = slot[c];
        const float4   l = rlo[c], h = rhi[c];
        lo[s]            = l;
        hi[s]            = h;
        centroid[s]      = make_float4(0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z), 0.0f);
        prim[s]          = rprim[c];
    }
}

__global__ void map_order_kernel(uint32_t* order, const uint32_t* prim, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        order[i] = prim[order[i]];
    }
}

}  // namespace

SplitReferences split_references(const float4* world, const float4* lo, const float4* hi, uint32_t prims,
                                  float factor, uint64_t max_references, cudaStream_t stream) {
    SplitReferences out;
    if (prims == 0) {
        return out;
    }
    const unsigned blocks = (prims + 255) / 256;
    DeviceBuffer<double> sum;
    DeviceBuffer<float>  max_area;
    sum.allocate(1);
    max_area.allocate(1);
    MR_CUDA(cudaMemsetAsync(sum.ptr, 0, sizeof(double), stream));
    MR_CUDA(cudaMemsetAsync(max_area.ptr, 0, sizeof(float), stream));
    area_kernel<<<blocks, 256, 0, stream>>>(lo, hi, prims, sum.ptr, max_area.ptr);
    double total_area = 0;
    float  largest    = 0;
    MR_CUDA(cudaMemcpyAsync(&total_area, sum.ptr, sizeof(double), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaMemcpyAsync(&largest, max_area.ptr, sizeof(float), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    // Cell area target: `factor` times the mean triangle box area, coarse enough that the largest
    // triangle needs at most the per-triangle cell cap, and doubled until the total fits.
    float target = static_cast<float>(std::max(static_cast<double>(factor) * total_area / prims,
                                               static_cast<double>(largest) / kMaxCellsPerTriangle));
    if (!(target > 0) || !std::isfinite(target)) {
        return out;  // degenerate boxes only: nothing to split
    }
    DeviceBuffer<uint32_t> cells, offsets, scratch, total;
    cells.allocate(prims);
    offsets.allocate(prims);
    scratch.allocate(scan_scratch_size(prims));
    total.allocate(1);
    uint32_t cell_total = 0;
    for (int round = 0; round < 40; ++round) {
        cell_count_kernel<<<blocks, 256, 0, stream>>>(lo, hi, prims, target, cells.ptr);
        exclusive_scan(cells.ptr, offsets.ptr, prims, scratch.ptr, total.ptr, stream);
        MR_CUDA(cudaMemcpyAsync(&cell_total, total.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        if (cell_total <= max_references) {
            break;
        }
        target *= 2.0f;
    }
    if (cell_total <= prims || cell_total > max_references) {
        return out;  // nothing worth splitting, or no target met the cap
    }
    DeviceBuffer<float4>   rlo, rhi;
    DeviceBuffer<uint32_t> rprim, valid, slot, slot_scratch;
    rlo.allocate(cell_total);
    rhi.allocate(cell_total);
    rprim.allocate(cell_total);
    valid.allocate(cell_total);
    slot.allocate(cell_total);
    slot_scratch.allocate(scan_scratch_size(cell_total));
    const unsigned cblocks = (cell_total + 255) / 256;
    cell_write_kernel<<<cblocks, 256, 0, stream>>>(world, lo, hi, offsets.ptr, prims, cell_total, target,
                                                   rlo.ptr, rhi.ptr, rprim.ptr, valid.ptr);
    exclusive_scan(valid.ptr, slot.ptr, cell_total, slot_scratch.ptr, total.ptr, stream);
    uint32_t refs = 0;
    MR_CUDA(cudaMemcpyAsync(&refs, total.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    out.lo.allocate(refs);
    out.hi.allocate(refs);
    out.centroid.allocate(refs);
    out.prim.allocate(refs);
    compact_refs_kernel<<<cblocks, 256, 0, stream>>>(rlo.ptr, rhi.ptr, rprim.ptr, valid.ptr, slot.ptr,
                                                     cell_total, out.lo.ptr, out.hi.ptr, out.centroid.ptr,
                                                     out.prim.ptr);
    MR_CUDA(cudaGetLastError());
    out.count = refs;
    return out;
}

void map_order_to_primitives(uint32_t* order, const uint32_t* prim, uint32_t count, cudaStream_t stream) {
    if (count) {
        map_order_kernel<<<(count + 255) / 256, 256, 0, stream>>>(order, prim, count);
        MR_CUDA(cudaGetLastError());
    }
}

}  // namespace mr
