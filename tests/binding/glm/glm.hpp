// A stand-in for the vector and matrix types of GLM 1.x, written for this project: only what the
// reference's scene headers declare with (vec2/vec3/vec4, dvec2/dvec3, mat3/mat4: component
// names and their colour aliases, scalar and per-component constructors, column access, equality).
// No arithmetic: the binding compiled against it only copies fields. Storage matches GLM's
// (tightly packed components, column-major matrices), which the binding relies on.
#pragma once

#include <cstddef>

namespace glm {

template <typename T>
struct tvec2 {
    union { T x, r, s; };
    union { T y, g, t; };
    constexpr tvec2() : x(0), y(0) {}
    constexpr explicit tvec2(T v) : x(v), y(v) {}
    constexpr tvec2(T a, T b) : x(a), y(b) {}
    constexpr T&       operator[](std::size_t i) { return i == 0 ? x : y; }
    constexpr const T& operator[](std::size_t i) const { return i == 0 ? x : y; }
    friend constexpr bool operator==(const tvec2& a, const tvec2& b) { return a.x == b.x && a.y == b.y; }
};

template <typename T>
struct tvec3 {
    union { T x, r, s; };
    union { T y, g, t; };
    union { T z, b, p; };
    constexpr tvec3() : x(0), y(0), z(0) {}
    constexpr explicit tvec3(T v) : x(v), y(v), z(v) {}
    constexpr tvec3(T a, T b, T c) : x(a), y(b), z(c) {}
    constexpr T&       operator[](std::size_t i) { return i == 0 ? x : (i == 1 ? y : z); }
    constexpr const T& operator[](std::size_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
    friend constexpr bool operator==(const tvec3& a, const tvec3& b) {
        return a.x == b.x && a.y == b.y && a.z == b.z;
    }
};

template <typename T>
struct tvec4 {
    union { T x, r, s; };
    union { T y, g, t; };
    union { T z, b, p; };
    union { T w, a, q; };
    constexpr tvec4() : x(0), y(0), z(0), w(0) {}
    constexpr explicit tvec4(T v) : x(v), y(v), z(v), w(v) {}
    constexpr tvec4(T a_, T b_, T c_, T d_) : x(a_), y(b_), z(c_), w(d_) {}
    constexpr T&       operator[](std::size_t i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    constexpr const T& operator[](std::size_t i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    friend constexpr bool operator==(const tvec4& a, const tvec4& b) {
        return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
    }
};

// N x N column-major matrix; the scalar constructor fills the diagonal.
template <typename T, std::size_t N, typename Column>
struct tmat {
    Column value[N];
    constexpr tmat() : tmat(T(1)) {}
    constexpr explicit tmat(T d) : value{} {
        for (std::size_t c = 0; c < N; ++c) {
            value[c] = Column(T(0));
            value[c][c] = d;
        }
    }
    constexpr Column&       operator[](std::size_t c) { return value[c]; }
    constexpr const Column& operator[](std::size_t c) const { return value[c]; }
    friend constexpr bool operator==(const tmat& a, const tmat& b) {
        for (std::size_t c = 0; c < N; ++c) {
            if (!(a.value[c] == b.value[c])) return false;
        }
        return true;
    }
};

using vec2  = tvec2<float>;
using vec3  = tvec3<float>;
using vec4  = tvec4<float>;
using dvec2 = tvec2<double>;
using dvec3 = tvec3<double>;
using dvec4 = tvec4<double>;
using mat3  = tmat<float, 3, vec3>;
using mat4  = tmat<float, 4, vec4>;

static_assert(sizeof(vec3) == 12 && sizeof(vec2) == 8 && sizeof(mat4) == 64 && sizeof(mat3) == 36,
              "GLM's packed layout");

}  // namespace glm
