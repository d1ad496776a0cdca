// rng.cuh — the reference's per-(seed, pixel, sample) PCG32 streams on the GPU.
//
// Integer-exact restatement of src/core/sampling.cpp:28-65: SplitMix64 seeding, PCG32
// XSH-RR output, two 32-bit outputs per 1-D sample. The reference forms a 53-bit double from
// (u32 >> 5, u32 >> 6); here the same 53-bit integer is rounded once to FP32 (round to nearest)
// and clamped below 1, so every sample is the FP32 rounding of the reference's double and the
// stream consumes exactly the same u32s in the same order.
#pragma once

#include "common.cuh"

namespace mr {

MR_HD uint64_t splitmix_finalize(uint64_t value) {
    value = (value ^ (value >> 30)) * 0xbf58476d1ce4e5b9ULL;
    value = (value ^ (value >> 27)) * 0x94d049bb133111ebULL;
    return value ^ (value >> 31);
}

struct Pcg32 {
    uint64_t state;
    uint64_t increment;

    MR_HD uint32_t next_u32() {
        const uint64_t previous = state;
        state                   = previous * 6364136223846793005ULL + increment;
        const uint32_t shifted  = static_cast<uint32_t>(((previous >> 18) ^ previous) >> 27);
        const uint32_t rotation = static_cast<uint32_t>(previous >> 59);
        return (shifted >> rotation) | (shifted << ((0u - rotation) & 31u));
    }

    // FP32 rounding of the reference's 53-bit next_1d, clamped to [0, 1).
    __device__ __forceinline__ float next_1d() {
        const uint64_t high = next_u32() >> 5;
        const uint64_t low  = next_u32() >> 6;
        const float    v    = __ull2float_rn((high << 26) | low) * 1.1102230246251565e-16f;  // 2^-53
        return fminf(v, kOneBelow);
    }

    MR_HD static Pcg32 seeded(uint64_t seed, uint64_t sequence) {
        Pcg32 p{0, (sequence << 1) | 1};
        p.next_u32();
        p.state += seed;
        p.next_u32();
        return p;
    }

    // Sampler::for_sample (src/core/sampling.cpp:43-46).
    MR_HD static Pcg32 for_sample(uint64_t seed, uint64_t pixel, uint64_t sample) {
        return seeded(splitmix_finalize(seed ^ splitmix_finalize(pixel + 0x9e3779b97f4a7c15ULL)),
                      splitmix_finalize(sample + 0xd1b54a32d192ed03ULL) ^ splitmix_finalize(pixel));
    }
};

}  // namespace mr
