// scan.cuh — device-wide exclusive prefix sum of uint32 (reduce-then-scan, three launches).
#pragma once

#include "common.cuh"

namespace mr {

constexpr int kScanBlock = 1024;  // items per block (256 threads x 4)

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) {
            v += n;
        }
    }
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024); returns the total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t& total) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t block_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t inclusive = warp_inclusive_scan(v);
    if (lane == 31) {
        warp_sums[warp] = inclusive;
    }
    __syncthreads();
    if (warp == 0) {
        const int      nw = (blockDim.x + 31) >> 5;
        const uint32_t s  = lane < nw ? warp_sums[lane] : 0;
        const uint32_t is = warp_inclusive_scan(s);
        if (lane < nw) {
            warp_sums[lane] = is - s;
        }
        if (lane == nw - 1) {
            block_total = is;
        }
    }
    __syncthreads();
    const uint32_t result = warp_sums[warp] + inclusive - v;
    total                 = block_total;
    __syncthreads();
    return result;
}

// Exclusive scan of n values; `scratch` needs scan_scratch_size(n) uint32s. Writes the grand
// total to *total_device when non-null. `out` may alias `in`.
inline size_t scan_scratch_size(size_t n) {
    size_t blocks = (n + kScanBlock - 1) / kScanBlock;
    size_t total  = 0;
    while (blocks > 1) {
        total += 2 * blocks;
        blocks = (blocks + kScanBlock - 1) / kScanBlock;
    }
    return total + 2;
}

void exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, uint32_t* scratch,
                    uint32_t* total_device, cudaStream_t stream);

}  // namespace mr
