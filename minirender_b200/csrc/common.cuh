// common.cuh — FP32 vector helpers, device constants and status plumbing shared by all kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "minirender_b200.h"

#ifndef MR_HD
#define MR_HD __host__ __device__ __forceinline__
#endif

namespace mr {

constexpr float kPi      = 3.14159265358979323846f;
constexpr float kInvPi   = 0.318309886183790671538f;
constexpr float kFltEps  = 1.1920928955078125e-07f;  // FLT_EPSILON (2^-23)
constexpr float kFltMin  = 1.17549435082228750797e-38f;
constexpr float kFltMax  = 3.40282346638528859812e+38f;
constexpr float kOneBelow = 0.99999994039535522461f;  // nextafter(1, 0)
constexpr unsigned kNone  = 0xffffffffu;

// Device-side error bits, OR-ed into a status word and mapped to mr_status by the host.
enum ErrorBits : unsigned {
    kErrorRadiance = 1u,  // nonfinite or negative path contribution (std::runtime_error)
    kErrorOverflow = 2u,  // pixel above FLT_MAX (std::overflow_error)
    kErrorStack    = 4u,  // traversal stack exhausted (never for trees of depth <= 48)
    kErrorMedium   = 8u,  // zero mixture probability in free-flight sampling
    kErrorVisits   = 16u, // a ray visited more nodes than any well-formed tree allows
    kErrorRay      = 32u, // a ray with a nonfinite origin or direction reached traversal
};

struct f3 {
    float x, y, z;
};

MR_HD f3 make(float x, float y, float z) { return {x, y, z}; }
MR_HD f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
MR_HD f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
MR_HD f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
MR_HD f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
MR_HD f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
MR_HD f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
MR_HD f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
MR_HD f3& operator+=(f3& a, f3 b) { return a = a + b; }
MR_HD f3& operator*=(f3& a, f3 b) { return a = a * b; }
MR_HD float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
MR_HD f3 cross(f3 a, f3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
MR_HD float length(f3 a) { return sqrtf(dot(a, a)); }
MR_HD f3 normalize(f3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
MR_HD f3 fabs3(f3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
MR_HD float max3(f3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
MR_HD float comp(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
MR_HD bool finite3(f3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
MR_HD f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
MR_HD float4 f4(f3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// Kahan's difference of products a*b - c*d with one FMA-recovered rounding error
// (the same structure as src/render/intersection.cpp:14-18, in FP32).
__device__ __forceinline__ float difference_of_products(float a, float b, float c, float d) {
    const float cd         = c * d;
    const float correction = fmaf(-c, d, cd);
    return fmaf(a, b, -cd) + correction;
}

}  // namespace mr
