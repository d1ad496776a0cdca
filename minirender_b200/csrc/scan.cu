// scan.cu — host driver of the device-wide exclusive scan (scan.cuh).
#include "scan.cuh"

namespace mr {

__global__ void scan_block_kernel(const uint32_t* in, uint32_t* out, uint32_t* block_sums,
                                  size_t n) {
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x * 4;
    uint32_t     v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
    }
    const uint32_t local = v[0] + v[1] + v[2] + v[3];
    uint32_t       total;
    uint32_t       prefix = block_exclusive_scan(local, total);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (base + i < n) {
            out[base + i] = prefix;
        }
        prefix += v[i];
    }
    if (threadIdx.x == 0) {
        block_sums[blockIdx.x] = total;
    }
}

__global__ void scan_add_kernel(uint32_t* out, const uint32_t* block_offsets, size_t n) {
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x * 4;
    const uint32_t add = block_offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (base + i < n) {
            out[base + i] += add;
        }
    }
}


void exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, uint32_t* scratch,
                    uint32_t* total_device, cudaStream_t stream) {
    if (n == 0) {
        if (total_device) {
            cudaMemsetAsync(total_device, 0, sizeof(uint32_t), stream);
        }
        return;
    }
    const size_t blocks = (n + kScanBlock - 1) / kScanBlock;
    uint32_t*    sums   = scratch;
    scan_block_kernel<<<static_cast<unsigned>(blocks), kScanBlock / 4, 0, stream>>>(in, out, sums, n);
    if (blocks == 1) {
        if (total_device) {
            cudaMemcpyAsync(total_device, sums, sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
        }
        return;
    }
    uint32_t* offsets = scratch + blocks;
    exclusive_scan(sums, offsets, blocks, scratch + 2 * blocks, total_device, stream);
    scan_add_kernel<<<static_cast<unsigned>(blocks), kScanBlock / 4, 0, stream>>>(out, offsets, n);
}

}  // namespace mr
