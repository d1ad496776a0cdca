// builder.cu — GPU binned-SAH BVH builder.
//
// The algorithm is the reference's recursive builder (src/render/bvh.cpp:101-196) evaluated
// breadth-first on the GPU: 12 centroid bins per axis, C_T = C_I = 1, a leaf when a node holds at
// most 4 primitives, sits at depth 48, has no split with nonempty sides, or no split cheaper than
// the leaf cost (its primitive count). Ties keep the first axis and split in the reference's
// search order. Partitioning is stable (the reference's std::partition is not; the resulting
// primitive sets, and so the tree topology, are the same).
//
// Two regimes:
//  - nodes with more than kSmallTask primitives are processed one level at a time by the whole
//    GPU: fixed-size chunks of a node's primitive range reduce bounds and bin in shared memory
//    and merge with one atomic per value per chunk; splits are chosen one thread per node;
//    primitives are scattered with a chunk scan so the order is deterministic;
//  - smaller nodes are finished by one warp each, depth-first in shared memory, with node
//    indices taken from a range reserved per subtree (unused indices are squeezed out at the end).
// All arithmetic is FP32. Surface areas are evaluated on extents scaled by a power of two so the
// products cannot overflow (the reference uses double for the same reason, intersection.cpp:44-50).
#include <algorithm>
#include <vector>

#include "errors.hpp"
#include "scan.cuh"
#include "scene.cuh"

namespace mr {
namespace {

constexpr int      kBins         = 12;
constexpr uint32_t kMaxDepth     = 48;
constexpr uint32_t kLeafSize     = 4;
constexpr uint32_t kSmallTask    = 256;   // nodes at most this large are built by one warp
constexpr uint32_t kChunk        = 2048;  // primitives per block in the level-wide passes
constexpr int      kSmallWarps   = 4;     // warps per block in the small-task kernel
constexpr uint32_t kUnusedNode   = 0xffffffffu;

__device__ __forceinline__ uint32_t f2o(float f) {  // order-preserving float -> uint
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}
constexpr uint32_t kOrderedPosInf = 0xff800000u;  // f2o(+inf)
constexpr uint32_t kOrderedNegInf = 0x007fffffu;  // f2o(-inf)

// bin_index (src/render/bvh.cpp:23-27) in FP32.
__device__ __forceinline__ int bin_of(float c, float lo, float hi) {
    const float coordinate = (c - lo) / (hi - lo);
    const float scaled     = coordinate * static_cast<float>(kBins);
    return min(static_cast<int>(scaled), kBins - 1);
}

// Surface area of a box scaled by `s` (a power of two).
__device__ __forceinline__ float scaled_area(const float* lo, const float* hi, float s) {
    if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) {
        return 0.0f;
    }
    const float ex = (hi[0] - lo[0]) * s, ey = (hi[1] - lo[1]) * s, ez = (hi[2] - lo[2]) * s;
    return 2.0f * (ex * ey + ey * ez + ez * ex);
}

__device__ __forceinline__ float area_scale(const float* lo, const float* hi) {
    const float m = fmaxf(fmaxf(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
    if (!(m > 0) || !isfinite(m)) {
        return 1.0f;
    }
    int e;
    frexpf(m, &e);
    return ldexpf(1.0f, -e);  // exact power of two, brings the largest extent into [0.5, 1)
}

struct Task {  // a node still to be split
    uint32_t begin, end;
    uint32_t node;
    uint32_t depth;
    uint32_t range;  // small tasks: first node index reserved for descendants
};

struct TaskBounds {  // ordered-uint encoded: bounds lo/hi, centroid lo/hi
    uint32_t v[12];
};

struct TaskBins {  // per axis, per bin: count and bounds (ordered uints)
    uint32_t count[3][kBins];
    uint32_t box[3][kBins][6];
};

struct Chunk {
    uint32_t task;
    uint32_t begin, end;
};

struct Split {
    int      axis;       // -1: leaf
    int      bin;
    uint32_t left_count;
};

__global__ void init_task_state(TaskBounds* bounds, TaskBins* bins, uint32_t count) {
    const uint32_t t = blockIdx.x;
    if (t >= count) {
        return;
    }
    for (int i = threadIdx.x; i < 12; i += blockDim.x) {
        bounds[t].v[i] = (i % 6) < 3 ? kOrderedPosInf : kOrderedNegInf;
    }
    uint32_t* c = &bins[t].count[0][0];
    for (int i = threadIdx.x; i < 3 * kBins; i += blockDim.x) {
        c[i] = 0;
    }
    uint32_t* b = &bins[t].box[0][0][0];
    for (int i = threadIdx.x; i < 3 * kBins * 6; i += blockDim.x) {
        b[i] = (i % 6) < 3 ? kOrderedPosInf : kOrderedNegInf;
    }
}

// Pass 1: node bounds and centroid bounds.
__global__ void reduce_bounds_kernel(const Chunk* chunks, const uint32_t* order, const float4* plo,
                                     const float4* phi, const float4* pc, TaskBounds* bounds) {
    __shared__ uint32_t s[12];
    const Chunk ch = chunks[blockIdx.x];
    if (threadIdx.x < 12) {
        s[threadIdx.x] = (threadIdx.x % 6) < 3 ? kOrderedPosInf : kOrderedNegInf;
    }
    __syncthreads();
    float v[12];
    for (int i = 0; i < 12; ++i) {
        v[i] = (i % 6) < 3 ? INFINITY : -INFINITY;
    }
    for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const uint32_t p = order[i];
        const float4 a = __ldg(plo + p), b = __ldg(phi + p), c = __ldg(pc + p);
        v[0] = fminf(v[0], a.x), v[1] = fminf(v[1], a.y), v[2] = fminf(v[2], a.z);
        v[3] = fmaxf(v[3], b.x), v[4] = fmaxf(v[4], b.y), v[5] = fmaxf(v[5], b.z);
        v[6] = fminf(v[6], c.x), v[7] = fminf(v[7], c.y), v[8] = fminf(v[8], c.z);
        v[9] = fmaxf(v[9], c.x), v[10] = fmaxf(v[10], c.y), v[11] = fmaxf(v[11], c.z);
    }
    for (int i = 0; i < 12; ++i) {
        float x = v[i];
        for (int o = 16; o > 0; o >>= 1) {
            const float y = __shfl_xor_sync(0xffffffffu, x, o);
            x = (i % 6) < 3 ? fminf(x, y) : fmaxf(x, y);
        }
        if ((threadIdx.x & 31) == 0) {
            if ((i % 6) < 3) {
                atomicMin(&s[i], f2o(x));
            } else {
                atomicMax(&s[i], f2o(x));
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        if ((threadIdx.x % 6) < 3) {
            atomicMin(&bounds[ch.task].v[threadIdx.x], s[threadIdx.x]);
        } else {
            atomicMax(&bounds[ch.task].v[threadIdx.x], s[threadIdx.x]);
        }
    }
}

// Pass 2: 12 bins per axis.
__global__ void bin_kernel(const Chunk* chunks, const uint32_t* order, const float4* plo,
                           const float4* phi, const float4* pc, const TaskBounds* bounds,
                           TaskBins* bins) {
    __shared__ uint32_t count[3][kBins];
    __shared__ uint32_t box[3][kBins][6];
    const Chunk ch = chunks[blockIdx.x];
    for (int i = threadIdx.x; i < 3 * kBins; i += blockDim.x) {
        (&count[0][0])[i] = 0;
    }
    for (int i = threadIdx.x; i < 3 * kBins * 6; i += blockDim.x) {
        (&box[0][0][0])[i] = (i % 6) < 3 ? kOrderedPosInf : kOrderedNegInf;
    }
    __syncthreads();
    const TaskBounds& tb = bounds[ch.task];
    float clo[3], chi[3];
    for (int a = 0; a < 3; ++a) {
        clo[a] = o2f(tb.v[6 + a]);
        chi[a] = o2f(tb.v[9 + a]);
    }
    for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const uint32_t p = order[i];
        const float4 a = __ldg(plo + p), b = __ldg(phi + p), c = __ldg(pc + p);
        const float cc[3] = {c.x, c.y, c.z};
        for (int axis = 0; axis < 3; ++axis) {
            if (chi[axis] == clo[axis]) {
                continue;
            }
            const int k = bin_of(cc[axis], clo[axis], chi[axis]);
            atomicAdd(&count[axis][k], 1u);
            atomicMin(&box[axis][k][0], f2o(a.x));
            atomicMin(&box[axis][k][1], f2o(a.y));
            atomicMin(&box[axis][k][2], f2o(a.z));
            atomicMax(&box[axis][k][3], f2o(b.x));
            atomicMax(&box[axis][k][4], f2o(b.y));
            atomicMax(&box[axis][k][5], f2o(b.z));
        }
    }
    __syncthreads();
    TaskBins& out = bins[ch.task];
    for (int i = threadIdx.x; i < 3 * kBins; i += blockDim.x) {
        const uint32_t c = (&count[0][0])[i];
        if (c) {
            atomicAdd(&(&out.count[0][0])[i], c);
        }
    }
    for (int i = threadIdx.x; i < 3 * kBins * 6; i += blockDim.x) {
        const uint32_t v = (&box[0][0][0])[i];
        if ((i % 6) < 3) {
            if (v != kOrderedPosInf) atomicMin(&(&out.box[0][0][0])[i], v);
        } else {
            if (v != kOrderedNegInf) atomicMax(&(&out.box[0][0][0])[i], v);
        }
    }
}

// SAH sweep over the 12 bins of the three axes (src/render/bvh.cpp:131-183).
__device__ Split choose_split(const float* lo, const float* hi, const float* clo, const float* chi,
                              uint32_t count, const uint32_t (*bin_count)[kBins],
                              const float (*bin_lo)[kBins][3], const float (*bin_hi)[kBins][3]) {
    Split       best{-1, 0, 0};
    float       best_cost = static_cast<float>(count);
    const float s         = area_scale(lo, hi);
    const float parent    = scaled_area(lo, hi, s);
    for (int axis = 0; axis < 3; ++axis) {
        if (chi[axis] == clo[axis]) {
            continue;
        }
        float    rlo[kBins][3], rhi[kBins][3];
        uint32_t rcount[kBins];
        float    alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t acc    = 0;
        for (int k = kBins - 1; k >= 0; --k) {
            if (bin_count[axis][k]) {
                for (int d = 0; d < 3; ++d) {
                    alo[d] = fminf(alo[d], bin_lo[axis][k][d]);
                    ahi[d] = fmaxf(ahi[d], bin_hi[axis][k][d]);
                }
            }
            acc += bin_count[axis][k];
            for (int d = 0; d < 3; ++d) {
                rlo[k][d] = alo[d];
                rhi[k][d] = ahi[d];
            }
            rcount[k] = acc;
        }
        float    llo[3] = {INFINITY, INFINITY, INFINITY}, lhi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t lcount = 0;
        for (int split = 0; split + 1 < kBins; ++split) {
            if (bin_count[axis][split]) {
                for (int d = 0; d < 3; ++d) {
                    llo[d] = fminf(llo[d], bin_lo[axis][split][d]);
                    lhi[d] = fmaxf(lhi[d], bin_hi[axis][split][d]);
                }
            }
            lcount += bin_count[axis][split];
            if (lcount == 0 || rcount[split + 1] == 0) {
                continue;
            }
            const float cost =
                1.0f + (scaled_area(llo, lhi, s) * static_cast<float>(lcount) +
                        scaled_area(rlo[split + 1], rhi[split + 1], s) * static_cast<float>(rcount[split + 1])) /
                           parent;
            if (cost < best_cost) {
                best_cost = cost;
                best      = {axis, split, lcount};
            }
        }
    }
    return best;
}

__device__ __forceinline__ void write_node(mr_bvh_node& n, const float* lo, const float* hi,
                                           uint32_t first, uint32_t right, uint32_t count) {
    for (int a = 0; a < 3; ++a) {
        n.minimum[a] = lo[a];
        n.maximum[a] = hi[a];
    }
    n.first = first;
    n.right = right;
    n.count = count;
}

// Pass 3: one thread per large task decides leaf or split and writes leaves.
__global__ void split_kernel(const Task* tasks, uint32_t count, const TaskBounds* bounds,
                             const TaskBins* bins, Split* splits, uint32_t* child_counts,
                             mr_bvh_node* nodes, unsigned long long* leaves, unsigned* depth) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) {
        return;
    }
    const Task& task = tasks[t];
    float lo[3], hi[3], clo[3], chi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a]  = o2f(bounds[t].v[a]);
        hi[a]  = o2f(bounds[t].v[3 + a]);
        clo[a] = o2f(bounds[t].v[6 + a]);
        chi[a] = o2f(bounds[t].v[9 + a]);
    }
    atomicMax(depth, task.depth);
    const uint32_t n = task.end - task.begin;
    Split          s{-1, 0, 0};
    if (n > kLeafSize && task.depth < kMaxDepth) {
        float blo[3][kBins][3], bhi[3][kBins][3];
        for (int a = 0; a < 3; ++a) {
            for (int k = 0; k < kBins; ++k) {
                for (int d = 0; d < 3; ++d) {
                    blo[a][k][d] = o2f(bins[t].box[a][k][d]);
                    bhi[a][k][d] = o2f(bins[t].box[a][k][3 + d]);
                }
            }
        }
        s = choose_split(lo, hi, clo, chi, n, bins[t].count, blo, bhi);
    }
    splits[t]       = s;
    child_counts[t] = s.axis < 0 ? 0u : 2u;
    if (s.axis < 0) {
        write_node(nodes[task.node], lo, hi, task.begin, 0, n);
        atomicAdd(leaves, 1ull);
    } else {
        write_node(nodes[task.node], lo, hi, 0, 0, 0);  // children filled by emit_children
    }
}

// Pass 4: per chunk, how many primitives go left.
__global__ void count_left_kernel(const Chunk* chunks, const uint32_t* order, const float4* pc,
                                  const TaskBounds* bounds, const Split* splits, uint32_t* left) {
    __shared__ uint32_t total;
    const Chunk ch = chunks[blockIdx.x];
    const Split s  = splits[ch.task];
    if (threadIdx.x == 0) {
        total = 0;
    }
    __syncthreads();
    if (s.axis >= 0) {
        const float lo = o2f(bounds[ch.task].v[6 + s.axis]);
        const float hi = o2f(bounds[ch.task].v[9 + s.axis]);
        uint32_t    mine = 0;
        for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
            const float4 c  = __ldg(pc + order[i]);
            const float  cc = s.axis == 0 ? c.x : (s.axis == 1 ? c.y : c.z);
            mine += bin_of(cc, lo, hi) <= s.bin ? 1u : 0u;
        }
        for (int o = 16; o > 0; o >>= 1) {
            mine += __shfl_xor_sync(0xffffffffu, mine, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&total, mine);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        left[blockIdx.x] = total;
    }
}

// Pass 5: stable scatter into `out` (chunks of split tasks only; others copy through).
__global__ void scatter_kernel(const Chunk* chunks, const uint32_t* chunk_left_offset,
                               const uint32_t* task_first_chunk, const Task* tasks,
                               const uint32_t* order, const float4* pc, const TaskBounds* bounds,
                               const Split* splits, uint32_t* out) {
    const Chunk    ch   = chunks[blockIdx.x];
    const Split    s    = splits[ch.task];
    const Task     task = tasks[ch.task];
    if (s.axis < 0) {
        for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
            out[i] = order[i];
        }
        return;
    }
    const float    lo      = o2f(bounds[ch.task].v[6 + s.axis]);
    const float    hi      = o2f(bounds[ch.task].v[9 + s.axis]);
    const uint32_t base_l  = chunk_left_offset[blockIdx.x] - chunk_left_offset[task_first_chunk[ch.task]];
    const uint32_t before  = ch.begin - task.begin;  // primitives of this task in earlier chunks
    uint32_t       left_so_far = 0;
    for (uint32_t start = ch.begin; start < ch.end; start += blockDim.x) {
        const uint32_t i    = start + threadIdx.x;
        bool           goes = false;
        uint32_t       p    = 0;
        if (i < ch.end) {
            p = order[i];
            const float4 c  = __ldg(pc + p);
            const float  cc = s.axis == 0 ? c.x : (s.axis == 1 ? c.y : c.z);
            goes            = bin_of(cc, lo, hi) <= s.bin;
        }
        uint32_t total;
        const uint32_t rank = block_exclusive_scan(goes ? 1u : 0u, total);
        if (i < ch.end) {
            const uint32_t local = i - ch.begin;
            if (goes) {
                out[task.begin + base_l + left_so_far + rank] = p;
            } else {
                const uint32_t right_rank = (before + local) - (base_l + left_so_far + rank);
                out[task.begin + s.left_count + right_rank] = p;
            }
        }
        left_so_far += total;
    }
}

__global__ void copy_kernel(const Chunk* chunks, const uint32_t* in, uint32_t* out) {
    const Chunk ch = chunks[blockIdx.x];
    for (uint32_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        out[i] = in[i];
    }
}

// Pass 6: link children, enqueue them as large or small tasks.
__global__ void emit_children_kernel(const Task* tasks, uint32_t count, const Split* splits,
                                     const uint32_t* child_offsets, uint32_t node_base,
                                     mr_bvh_node* nodes, Task* next_large, uint32_t* next_large_count,
                                     Task* small, uint32_t* small_count) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count || splits[t].axis < 0) {
        return;
    }
    const Task&    task  = tasks[t];
    const uint32_t left  = node_base + child_offsets[t];
    const uint32_t right = left + 1;
    nodes[task.node].first = left;
    nodes[task.node].right = right;
    const uint32_t mid     = task.begin + splits[t].left_count;
    const Task     children[2] = {{task.begin, mid, left, task.depth + 1, 0},
                                  {mid, task.end, right, task.depth + 1, 0}};
    for (int c = 0; c < 2; ++c) {
        const uint32_t n = children[c].end - children[c].begin;
        if (n > kSmallTask) {  // at depth 48 the split pass turns it into a leaf
            next_large[atomicAdd(next_large_count, 1u)] = children[c];
        } else {
            small[atomicAdd(small_count, 1u)] = children[c];
        }
    }
}

// Chunk descriptors for a level.
__global__ void make_chunks_kernel(const Task* tasks, uint32_t count, const uint32_t* chunk_offsets,
                                   Chunk* chunks, uint32_t* task_first_chunk) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) {
        return;
    }
    const Task&    task  = tasks[t];
    const uint32_t first = chunk_offsets[t];
    task_first_chunk[t]  = first;
    uint32_t k           = first;
    for (uint32_t b = task.begin; b < task.end; b += kChunk, ++k) {
        chunks[k] = {t, b, min(b + kChunk, task.end)};
    }
}

__global__ void chunk_count_kernel(const Task* tasks, uint32_t count, uint32_t* out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) {
        out[t] = (tasks[t].end - tasks[t].begin + kChunk - 1) / kChunk;
    }
}

__global__ void small_reserve_kernel(const Task* small, uint32_t count, uint32_t* sizes) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) {
        const uint32_t n = small[t].end - small[t].begin;
        sizes[t]         = 2 * n - 2;  // descendants of a subtree over n primitives
    }
}

// Small subtrees: one warp per task, depth-first in shared memory. Node indices are assigned in
// pre-order from the task's reserved range (the reference's emplacement order, bvh.cpp:104-105).
__global__ void __launch_bounds__(32 * kSmallWarps)
small_build_kernel(const Task* small, uint32_t count, const uint32_t* ranges, uint32_t range_base,
                   uint32_t* order, const float4* plo, const float4* phi, const float4* pc,
                   mr_bvh_node* nodes, unsigned long long* leaves, unsigned* max_depth) {
    struct Entry {
        uint32_t begin, end, depth, parent_slot;  // parent_slot: node index*2 + side, or ~0
    };
    __shared__ uint32_t s_idx[kSmallWarps][kSmallTask];
    __shared__ uint32_t s_tmp[kSmallWarps][kSmallTask];
    __shared__ uint32_t s_count[kSmallWarps][3][kBins];
    __shared__ uint32_t s_box[kSmallWarps][3][kBins][6];
    __shared__ Entry    s_stack[kSmallWarps][kMaxDepth + 2];
    const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t t    = blockIdx.x * kSmallWarps + warp;
    if (t >= count) {
        return;
    }
    const Task task = small[t];
    const uint32_t n = task.end - task.begin;
    for (uint32_t i = lane; i < n; i += 32) {
        s_idx[warp][i] = order[task.begin + i];
    }
    __syncwarp();
    uint32_t next_node = range_base + ranges[t];
    int      sp        = 0;
    if (lane == 0) {
        s_stack[warp][0] = {0, n, task.depth, kUnusedNode};
    }
    sp = 1;
    bool first = true;
    uint32_t local_leaves = 0, local_depth = 0;
    while (sp > 0) {
        __syncwarp();
        const Entry e = s_stack[warp][--sp];
        __syncwarp();
        const uint32_t node = first ? task.node : next_node++;
        first               = false;
        if (lane == 0 && e.parent_slot != kUnusedNode) {
            mr_bvh_node& parent = nodes[e.parent_slot >> 1];
            if (e.parent_slot & 1u) {
                parent.right = node;
            } else {
                parent.first = node;
            }
        }
        local_depth = max(local_depth, e.depth);
        // Bounds and centroid bounds (warp reduction).
        float v[12];
        for (int i = 0; i < 12; ++i) {
            v[i] = (i % 6) < 3 ? INFINITY : -INFINITY;
        }
        for (uint32_t i = e.begin + lane; i < e.end; i += 32) {
            const uint32_t p = s_idx[warp][i];
            const float4 a = __ldg(plo + p), b = __ldg(phi + p), c = __ldg(pc + p);
            v[0] = fminf(v[0], a.x), v[1] = fminf(v[1], a.y), v[2] = fminf(v[2], a.z);
            v[3] = fmaxf(v[3], b.x), v[4] = fmaxf(v[4], b.y), v[5] = fmaxf(v[5], b.z);
            v[6] = fminf(v[6], c.x), v[7] = fminf(v[7], c.y), v[8] = fminf(v[8], c.z);
            v[9] = fmaxf(v[9], c.x), v[10] = fmaxf(v[10], c.y), v[11] = fmaxf(v[11], c.z);
        }
        for (int i = 0; i < 12; ++i) {
            for (int o = 16; o > 0; o >>= 1) {
                const float y = __shfl_xor_sync(0xffffffffu, v[i], o);
                v[i]          = (i % 6) < 3 ? fminf(v[i], y) : fmaxf(v[i], y);
            }
        }
        const float* lo = v;
        const float* hi = v + 3;
        const float* clo = v + 6;
        const float* chi = v + 9;
        const uint32_t m = e.end - e.begin;
        Split s{-1, 0, 0};
        if (m > kLeafSize && e.depth < kMaxDepth) {
            for (int i = lane; i < 3 * kBins; i += 32) {
                (&s_count[warp][0][0])[i] = 0;
            }
            for (int i = lane; i < 3 * kBins * 6; i += 32) {
                (&s_box[warp][0][0][0])[i] = (i % 6) < 3 ? kOrderedPosInf : kOrderedNegInf;
            }
            __syncwarp();
            for (uint32_t i = e.begin + lane; i < e.end; i += 32) {
                const uint32_t p = s_idx[warp][i];
                const float4 a = __ldg(plo + p), b = __ldg(phi + p), c = __ldg(pc + p);
                const float cc[3] = {c.x, c.y, c.z};
                for (int axis = 0; axis < 3; ++axis) {
                    if (chi[axis] == clo[axis]) {
                        continue;
                    }
                    const int k = bin_of(cc[axis], clo[axis], chi[axis]);
                    atomicAdd(&s_count[warp][axis][k], 1u);
                    atomicMin(&s_box[warp][axis][k][0], f2o(a.x));
                    atomicMin(&s_box[warp][axis][k][1], f2o(a.y));
                    atomicMin(&s_box[warp][axis][k][2], f2o(a.z));
                    atomicMax(&s_box[warp][axis][k][3], f2o(b.x));
                    atomicMax(&s_box[warp][axis][k][4], f2o(b.y));
                    atomicMax(&s_box[warp][axis][k][5], f2o(b.z));
                }
            }
            __syncwarp();
            if (lane == 0) {
                float blo[3][kBins][3], bhi[3][kBins][3];
                for (int a = 0; a < 3; ++a) {
                    for (int k = 0; k < kBins; ++k) {
                        for (int d = 0; d < 3; ++d) {
                            blo[a][k][d] = o2f(s_box[warp][a][k][d]);
                            bhi[a][k][d] = o2f(s_box[warp][a][k][3 + d]);
                        }
                    }
                }
                s = choose_split(lo, hi, clo, chi, m, s_count[warp], blo, bhi);
            }
            s.axis       = __shfl_sync(0xffffffffu, s.axis, 0);
            s.bin        = __shfl_sync(0xffffffffu, s.bin, 0);
            s.left_count = __shfl_sync(0xffffffffu, s.left_count, 0);
        }
        if (s.axis < 0) {
            if (lane == 0) {
                write_node(nodes[node], lo, hi, task.begin + e.begin, 0, m);
            }
            ++local_leaves;
            continue;
        }
        // Stable partition in shared memory.
        uint32_t left_so_far = 0;
        const float plo_axis = clo[s.axis], phi_axis = chi[s.axis];
        for (uint32_t start = e.begin; start < e.end; start += 32) {
            const uint32_t i    = start + lane;
            bool           goes = false;
            uint32_t       p    = 0;
            if (i < e.end) {
                p = s_idx[warp][i];
                const float4 c  = __ldg(pc + p);
                const float  cc = s.axis == 0 ? c.x : (s.axis == 1 ? c.y : c.z);
                goes            = bin_of(cc, plo_axis, phi_axis) <= s.bin;
            }
            const unsigned mask = __ballot_sync(0xffffffffu, goes);
            const uint32_t rank = __popc(mask & ((1u << lane) - 1u));
            if (i < e.end) {
                if (goes) {
                    s_tmp[warp][e.begin + left_so_far + rank] = p;
                } else {
                    const uint32_t right_rank = (i - e.begin) - (left_so_far + rank);
                    s_tmp[warp][e.begin + s.left_count + right_rank] = p;
                }
            }
            left_so_far += __popc(mask);
        }
        __syncwarp();
        for (uint32_t i = e.begin + lane; i < e.end; i += 32) {
            s_idx[warp][i] = s_tmp[warp][i];
        }
        if (lane == 0) {
            write_node(nodes[node], lo, hi, 0, 0, 0);
            const uint32_t mid = e.begin + s.left_count;
            s_stack[warp][sp]     = {mid, e.end, e.depth + 1, node * 2 + 1};
            s_stack[warp][sp + 1] = {e.begin, mid, e.depth + 1, node * 2};
        }
        sp += 2;
    }
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) {
        order[task.begin + i] = s_idx[warp][i];
    }
    if (lane == 0) {
        atomicAdd(leaves, static_cast<unsigned long long>(local_leaves));
        atomicMax(max_depth, local_depth);
    }
    // Mark the unused tail of the reserved range.
    const uint32_t reserved_end = range_base + ranges[t] + (2 * n - 2);
    for (uint32_t k = next_node + lane; k < reserved_end; k += 32) {
        nodes[k].count = kUnusedNode;
        nodes[k].first = 0;
        nodes[k].right = 0;
    }
}

__global__ void valid_flag_kernel(const mr_bvh_node* nodes, uint32_t count, uint32_t* flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        flags[i] = nodes[i].count == kUnusedNode ? 0u : 1u;
    }
}

__global__ void compact_nodes_kernel(const mr_bvh_node* in, uint32_t count, const uint32_t* index,
                                     mr_bvh_node* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count || in[i].count == kUnusedNode) {
        return;
    }
    mr_bvh_node n = in[i];
    if (n.count == 0) {
        n.first = index[n.first];
        n.right = index[n.right];
    }
    out[index[i]] = n;
}

__global__ void iota_kernel(uint32_t* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        out[i] = i;
    }
}

inline unsigned blocks_for(size_t n, unsigned per = 256) {
    return static_cast<unsigned>((n + per - 1) / per);
}

}  // namespace

BuildResult build_bvh_device(const float4* lo, const float4* hi, const float4* centroid,
                             uint32_t count, cudaStream_t stream) {
    BuildResult result;
    if (count == 0) {
        return result;
    }
    cudaEvent_t start, stop;
    MR_CUDA(cudaEventCreate(&start));
    MR_CUDA(cudaEventCreate(&stop));
    MR_CUDA(cudaEventRecord(start, stream));

    const size_t node_capacity = 2ull * count - 1;
    DeviceBuffer<mr_bvh_node> nodes;
    DeviceBuffer<uint32_t>    order, scratch_order;
    nodes.allocate(node_capacity);
    order.allocate(count);
    scratch_order.allocate(count);
    iota_kernel<<<blocks_for(count), 256, 0, stream>>>(order.ptr, count);

    // Task storage: a level never holds more than count / (kSmallTask + 1) large tasks, the
    // small list never more than count tasks... bounded by count.
    const size_t max_tasks  = std::max<size_t>(1, count / (kSmallTask / 2) + 2);
    const size_t max_chunks = count / kChunk + max_tasks + 1;
    DeviceBuffer<uint8_t> raw;
    const size_t bytes =
        2 * max_tasks * sizeof(Task) + max_tasks * (sizeof(TaskBounds) + sizeof(TaskBins) + sizeof(Split)) +
        6 * max_tasks * sizeof(uint32_t) + max_chunks * (sizeof(Chunk) + 2 * sizeof(uint32_t)) +
        static_cast<size_t>(count) * (sizeof(Task) + 2 * sizeof(uint32_t)) + 64 * 16 +
        (scan_scratch_size(std::max(max_chunks, static_cast<size_t>(count))) + 8) * sizeof(uint32_t);
    raw.allocate(bytes);
    uint8_t* cursor = raw.ptr;
    const auto take = [&](size_t b) {
        uint8_t* p = cursor;
        cursor += (b + 15) & ~size_t(15);
        return p;
    };
    Task*       tasks[2]      = {reinterpret_cast<Task*>(take(max_tasks * sizeof(Task))),
                                 reinterpret_cast<Task*>(take(max_tasks * sizeof(Task)))};
    TaskBounds* task_bounds   = reinterpret_cast<TaskBounds*>(take(max_tasks * sizeof(TaskBounds)));
    TaskBins*   task_bins     = reinterpret_cast<TaskBins*>(take(max_tasks * sizeof(TaskBins)));
    Split*      splits        = reinterpret_cast<Split*>(take(max_tasks * sizeof(Split)));
    uint32_t*   child_counts  = reinterpret_cast<uint32_t*>(take(max_tasks * sizeof(uint32_t)));
    uint32_t*   child_offsets = reinterpret_cast<uint32_t*>(take(max_tasks * sizeof(uint32_t)));
    uint32_t*   chunk_counts  = reinterpret_cast<uint32_t*>(take(max_tasks * sizeof(uint32_t)));
    uint32_t*   chunk_offsets = reinterpret_cast<uint32_t*>(take(max_tasks * sizeof(uint32_t)));
    uint32_t*   task_first    = reinterpret_cast<uint32_t*>(take(max_tasks * sizeof(uint32_t)));
    Chunk*      chunks        = reinterpret_cast<Chunk*>(take(max_chunks * sizeof(Chunk)));
    uint32_t*   chunk_left    = reinterpret_cast<uint32_t*>(take(max_chunks * sizeof(uint32_t)));
    uint32_t*   chunk_left_off = reinterpret_cast<uint32_t*>(take(max_chunks * sizeof(uint32_t)));
    Task*       small         = reinterpret_cast<Task*>(take(static_cast<size_t>(count) * sizeof(Task)));
    uint32_t*   small_sizes   = reinterpret_cast<uint32_t*>(take(static_cast<size_t>(count) * sizeof(uint32_t)));
    uint32_t*   small_ranges  = reinterpret_cast<uint32_t*>(take(static_cast<size_t>(count) * sizeof(uint32_t)));
    uint32_t*   counters      = reinterpret_cast<uint32_t*>(take(16 * sizeof(uint32_t)));
    unsigned long long* leaves = reinterpret_cast<unsigned long long*>(take(sizeof(unsigned long long)));
    uint32_t*   scratch       = reinterpret_cast<uint32_t*>(
        take((scan_scratch_size(std::max(max_chunks, static_cast<size_t>(count))) + 8) * sizeof(uint32_t)));
    // counters: [0] next large count, [1] small count, [2] child total, [3] chunk total,
    //           [4] max depth, [5] small range total
    MR_CUDA(cudaMemsetAsync(counters, 0, 16 * sizeof(uint32_t), stream));
    MR_CUDA(cudaMemsetAsync(leaves, 0, sizeof(unsigned long long), stream));

    uint32_t node_base = 1;  // node 0 is the root
    uint32_t level_count = 0;
    uint32_t small_total = 0;
    // Root task: large unless it is small enough for one warp.
    const Task root{0, count, 0, 0, 0};
    int        cur = 0;
    if (count > kSmallTask) {
        MR_CUDA(cudaMemcpyAsync(tasks[0], &root, sizeof(Task), cudaMemcpyHostToDevice, stream));
        level_count = 1;
    } else {
        MR_CUDA(cudaMemcpyAsync(small, &root, sizeof(Task), cudaMemcpyHostToDevice, stream));
        small_total = 1;
        const uint32_t one = 1;
        MR_CUDA(cudaMemcpyAsync(counters + 1, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    }

    while (level_count > 0) {
        Task* level = tasks[cur];
        Task* next  = tasks[cur ^ 1];
        // Chunk list of this level.
        chunk_count_kernel<<<blocks_for(level_count), 256, 0, stream>>>(level, level_count, chunk_counts);
        exclusive_scan(chunk_counts, chunk_offsets, level_count, scratch, counters + 3, stream);
        make_chunks_kernel<<<blocks_for(level_count), 256, 0, stream>>>(level, level_count, chunk_offsets,
                                                                          chunks, task_first);
        uint32_t chunk_total = 0;
        MR_CUDA(cudaMemcpyAsync(&chunk_total, counters + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        init_task_state<<<level_count, 128, 0, stream>>>(task_bounds, task_bins, level_count);
        reduce_bounds_kernel<<<chunk_total, 256, 0, stream>>>(chunks, order.ptr, lo, hi, centroid, task_bounds);
        bin_kernel<<<chunk_total, 256, 0, stream>>>(chunks, order.ptr, lo, hi, centroid, task_bounds, task_bins);
        split_kernel<<<blocks_for(level_count, 64), 64, 0, stream>>>(level, level_count, task_bounds, task_bins,
                                                                       splits, child_counts, nodes.ptr, leaves,
                                                                       counters + 4);
        count_left_kernel<<<chunk_total, 256, 0, stream>>>(chunks, order.ptr, centroid, task_bounds, splits,
                                                            chunk_left);
        exclusive_scan(chunk_left, chunk_left_off, chunk_total, scratch, nullptr, stream);
        scatter_kernel<<<chunk_total, 256, 0, stream>>>(chunks, chunk_left_off, task_first, level, order.ptr,
                                                         centroid, task_bounds, splits, scratch_order.ptr);
        copy_kernel<<<chunk_total, 256, 0, stream>>>(chunks, scratch_order.ptr, order.ptr);
        exclusive_scan(child_counts, child_offsets, level_count, scratch, counters + 2, stream);
        MR_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t), stream));
        emit_children_kernel<<<blocks_for(level_count), 256, 0, stream>>>(level, level_count, splits,
                                                                           child_offsets, node_base, nodes.ptr,
                                                                           next, counters, small, counters + 1);
        MR_CUDA(cudaGetLastError());
        uint32_t host_counters[3];
        MR_CUDA(cudaMemcpyAsync(host_counters, counters, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        node_base += host_counters[2];
        level_count = host_counters[0];
        small_total = host_counters[1];
        // Deterministic task order for the next level and the small list: by range begin.
        if (level_count > 1) {
            std::vector<Task> h(level_count);
            MR_CUDA(cudaMemcpyAsync(h.data(), next, level_count * sizeof(Task), cudaMemcpyDeviceToHost, stream));
            MR_CUDA(cudaStreamSynchronize(stream));
            std::sort(h.begin(), h.end(), [](const Task& a, const Task& b) { return a.begin < b.begin; });
            MR_CUDA(cudaMemcpyAsync(next, h.data(), level_count * sizeof(Task), cudaMemcpyHostToDevice, stream));
        }
        cur ^= 1;
    }

    if (small_total > 0) {
        std::vector<Task> h(small_total);
        MR_CUDA(cudaMemcpyAsync(h.data(), small, small_total * sizeof(Task), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        std::sort(h.begin(), h.end(), [](const Task& a, const Task& b) { return a.begin < b.begin; });
        MR_CUDA(cudaMemcpyAsync(small, h.data(), small_total * sizeof(Task), cudaMemcpyHostToDevice, stream));
        small_reserve_kernel<<<blocks_for(small_total), 256, 0, stream>>>(small, small_total, small_sizes);
        exclusive_scan(small_sizes, small_ranges, small_total, scratch, counters + 5, stream);
        const unsigned blocks = (small_total + kSmallWarps - 1) / kSmallWarps;
        small_build_kernel<<<blocks, 32 * kSmallWarps, 0, stream>>>(small, small_total, small_ranges, node_base,
                                                                     order.ptr, lo, hi, centroid, nodes.ptr,
                                                                     leaves, counters + 4);
        MR_CUDA(cudaGetLastError());
        uint32_t reserved = 0;
        MR_CUDA(cudaMemcpyAsync(&reserved, counters + 5, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        node_base += reserved;
    }

    // Squeeze out unused node indices.
    const uint32_t used_capacity = node_base;
    DeviceBuffer<uint32_t> valid, index;
    valid.allocate(used_capacity);
    index.allocate(used_capacity);
    valid_flag_kernel<<<blocks_for(used_capacity), 256, 0, stream>>>(nodes.ptr, used_capacity, valid.ptr);
    exclusive_scan(valid.ptr, index.ptr, used_capacity, scratch, counters + 6, stream);
    uint32_t compact = 0;
    MR_CUDA(cudaMemcpyAsync(&compact, counters + 6, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    result.nodes.allocate(compact);
    compact_nodes_kernel<<<blocks_for(used_capacity), 256, 0, stream>>>(nodes.ptr, used_capacity, index.ptr,
                                                                         result.nodes.ptr);
    MR_CUDA(cudaGetLastError());
    unsigned long long host_leaves = 0;
    uint32_t           host_depth  = 0;
    MR_CUDA(cudaMemcpyAsync(&host_leaves, leaves, sizeof(host_leaves), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaMemcpyAsync(&host_depth, counters + 4, sizeof(host_depth), cudaMemcpyDeviceToHost, stream));
    MR_CUDA(cudaEventRecord(stop, stream));
    MR_CUDA(cudaStreamSynchronize(stream));
    float ms = 0;
    MR_CUDA(cudaEventElapsedTime(&ms, start, stop));
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    result.order         = std::move(order);
    result.node_count    = compact;
    result.leaves        = host_leaves;
    result.maximum_depth = host_depth;
    result.seconds       = ms * 1e-3;
    return result;
}

}  // namespace mr
