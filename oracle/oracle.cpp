// oracle.cpp — CPU oracle of MiniRender's offline path tracer. TEST INFRASTRUCTURE ONLY.
//
// This file restates, in FP64 C++ with no third-party code, the reference algorithm of the path
// the B200 library accelerates. It exists to check the GPU product, never to be the product:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it. Each function
// cites the reference file:line it follows (paths inside the MiniRender source tree).
//
// The reference itself cannot be compiled here (it needs GLM, which is absent), so this is a
// restatement ("port"). It is pinned by the reference's own golden vectors and known-answer
// tests (tests/test_oracle_golden.py).
//
// GLM semantics restated where they change rounding: normalize(v) = v * (1/sqrt(dot(v,v))),
// dot(a,b) = (ax*bx + ay*by) + az*bz, mat4*vec4 = (m0*x + m1*y) + (m2*z + m3*w).

#include "minirender_b200.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numbers>
#include <optional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace oracle {

constexpr double pi       = std::numbers::pi;
constexpr double infinity = std::numeric_limits<double>::infinity();
constexpr double dbl_eps  = std::numeric_limits<double>::epsilon();
// The unit of the position error bounds that offset spawned rays and shadow-segment ends
// (path_tracer.cpp:87-105): double's epsilon, as the reference computes them. Built with
// ORACLE_FP32_OFFSETS it is float's epsilon, the size of the FP32 device's bounds; the tests use
// that build only to show which image differences come from the larger FP32 offsets.
#ifdef ORACLE_FP32_OFFSETS
constexpr double offset_eps = std::numeric_limits<float>::epsilon();
#else
constexpr double offset_eps = dbl_eps;
#endif

// ---- vector helpers (GLM operation order) --------------------------------------------------

struct dvec2 {
    double x = 0, y = 0;
};
struct dvec3 {
    double x = 0, y = 0, z = 0;
    double&       operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    double        operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct fvec3 {
    float  x = 0, y = 0, z = 0;
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float  operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

inline dvec3 operator+(dvec3 a, dvec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline dvec3 operator-(dvec3 a, dvec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline dvec3 operator-(dvec3 a) { return {-a.x, -a.y, -a.z}; }
inline dvec3 operator*(dvec3 a, dvec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline dvec3 operator*(dvec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline dvec3 operator*(double s, dvec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline dvec3 operator/(dvec3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline dvec3 operator/(dvec3 a, dvec3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline dvec3& operator+=(dvec3& a, dvec3 b) { return a = a + b; }
inline dvec3& operator*=(dvec3& a, dvec3 b) { return a = a * b; }
inline dvec3& operator/=(dvec3& a, double s) { return a = a / s; }
inline double dot(dvec3 a, dvec3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double dot2(dvec2 a, dvec2 b) { return a.x * b.x + a.y * b.y; }
inline dvec3 cross(dvec3 a, dvec3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline double length(dvec3 a) { return std::sqrt(dot(a, a)); }
inline dvec3 normalize(dvec3 a) { return a * (1.0 / std::sqrt(dot(a, a))); }
inline dvec3 dabs(dvec3 a) { return {std::abs(a.x), std::abs(a.y), std::abs(a.z)}; }
inline double max3(dvec3 a) { return std::max({a.x, a.y, a.z}); }
inline bool finite3(dvec3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline bool finite3(fvec3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline dvec3 widen(fvec3 a) { return {a.x, a.y, a.z}; }
inline fvec3 narrow(dvec3 a) {
    return {static_cast<float>(a.x), static_cast<float>(a.y), static_cast<float>(a.z)};
}
inline dvec3 from(const float* p) { return {p[0], p[1], p[2]}; }
inline dvec3 from(const double* p) { return {p[0], p[1], p[2]}; }

void require(bool condition, const char* message) {
    if (!condition) {
        throw std::invalid_argument(message);
    }
}

// ---- sampling (src/core/sampling.cpp) ----------------------------------------------------

void check_unit(double u) {  // sampling.cpp:16-20
    if (!(u >= 0 && u < 1)) {
        throw std::invalid_argument("Sample coordinate must be in [0,1)");
    }
}
void check_unit(dvec2 u) {
    check_unit(u.x);
    check_unit(u.y);
}

std::uint64_t mix(std::uint64_t value) {  // sampling.cpp:28-32 (SplitMix64 finaliser)
    value = (value ^ (value >> 30U)) * 0xbf58476d1ce4e5b9ULL;
    value = (value ^ (value >> 27U)) * 0x94d049bb133111ebULL;
    return value ^ (value >> 31U);
}

class Sampler {  // sampling.cpp:36-65, PCG32 XSH-RR
  public:
    explicit Sampler(std::uint64_t seed = 0, std::uint64_t sequence = 1)
        : increment_((sequence << 1U) | 1U) {
        next_u32();
        state_ += seed;
        next_u32();
    }
    static Sampler for_sample(std::uint64_t seed, std::uint64_t pixel, std::uint64_t sample) {
        return Sampler(mix(seed ^ mix(pixel + 0x9e3779b97f4a7c15ULL)),
                       mix(sample + 0xd1b54a32d192ed03ULL) ^ mix(pixel));
    }
    std::uint32_t next_u32() {
        const auto previous = state_;
        state_              = previous * 6364136223846793005ULL + increment_;
        const auto shifted  = static_cast<std::uint32_t>(((previous >> 18U) ^ previous) >> 27U);
        const auto rotation = static_cast<std::uint32_t>(previous >> 59U);
        return (shifted >> rotation) | (shifted << ((0U - rotation) & 31U));
    }
    double next_1d() {
        const auto high = next_u32() >> 5U;
        const auto low  = next_u32() >> 6U;
        return (static_cast<double>(high) * 67108864.0 + low) / 9007199254740992.0;
    }
    dvec2 next_2d() {
        const double x = next_1d();
        return {x, next_1d()};
    }
    std::uint64_t state() const { return state_; }
    std::uint64_t increment() const { return increment_; }

  private:
    std::uint64_t state_     = 0;
    std::uint64_t increment_ = 1;
};

dvec2 sample_disk(dvec2 u) {  // sampling.cpp:67-79, Shirley-Chiu concentric map
    check_unit(u);
    const dvec2 square{2.0 * u.x - 1.0, 2.0 * u.y - 1.0};
    if (square.x == 0 && square.y == 0) {
        return {0, 0};
    }
    const bool   horizontal = std::abs(square.x) > std::abs(square.y);
    const double radius     = horizontal ? square.x : square.y;
    const double angle =
        horizontal ? (pi / 4) * (square.y / square.x) : pi / 2 - (pi / 4) * (square.x / square.y);
    return {radius * std::cos(angle), radius * std::sin(angle)};
}

dvec3 sample_sphere(dvec2 u) {  // sampling.cpp:81-86
    check_unit(u);
    const double z      = 1 - 2 * u.x;
    const double radius = std::sqrt(std::max(0.0, 1 - z * z));
    return {radius * std::cos(2 * pi * u.y), radius * std::sin(2 * pi * u.y), z};
}

dvec3 sample_hemisphere(dvec2 u) {  // sampling.cpp:88-92
    check_unit(u);
    const double radius = std::sqrt(std::max(0.0, 1 - u.x * u.x));
    return {radius * std::cos(2 * pi * u.y), radius * std::sin(2 * pi * u.y), u.x};
}

dvec3 sample_cosine_hemisphere(dvec2 u) {  // sampling.cpp:94-97
    const auto disk = sample_disk(u);
    return {disk.x, disk.y, std::sqrt(std::max(0.0, 1 - dot2(disk, disk)))};
}

dvec3 sample_triangle(dvec2 u) {  // sampling.cpp:99-103
    check_unit(u);
    const double root = std::sqrt(u.x);
    return {1 - root, root * (1 - u.y), root * u.y};
}

double cosine_hemisphere_pdf(dvec3 direction) {  // sampling.cpp:105-107
    return std::max(0.0, direction.z) / pi;
}

struct DiscreteSample {
    std::size_t index       = 0;
    double      probability = 0;
    double      remapped    = 0;
};

class DiscreteDistribution {  // sampling.cpp:109-150
  public:
    DiscreteDistribution() : cdf_(1, 0) {}
    explicit DiscreteDistribution(const std::vector<double>& weights)
        : cdf_(weights.size() + 1, 0) {
        double maximum = 0;
        for (const auto weight : weights) {
            if (!std::isfinite(weight) || weight < 0) {
                throw std::invalid_argument("Distribution weights must be finite and nonnegative");
            }
            maximum = std::max(maximum, weight);
        }
        for (std::size_t index = 0; index < weights.size(); ++index) {
            cdf_[index + 1] = cdf_[index] + (maximum > 0 ? weights[index] / maximum : 1);
        }
        if (!weights.empty()) {
            const double integral = cdf_.back();
            for (auto& value : cdf_) {
                value /= integral;
            }
        }
    }
    std::optional<DiscreteSample> sample(double u) const {
        check_unit(u);
        if (size() == 0) {
            return std::nullopt;
        }
        const auto   upper    = std::upper_bound(cdf_.begin(), cdf_.end(), u);
        const auto   index    = static_cast<std::size_t>(upper - cdf_.begin() - 1);
        const double mass     = probability(index);
        const double remapped = std::min((u - cdf_[index]) / mass, std::nextafter(1.0, 0.0));
        return DiscreteSample{index, mass, remapped};
    }
    double probability(std::size_t index) const {
        if (index >= size()) {
            throw std::out_of_range("Distribution index is out of range");
        }
        return cdf_[index + 1] - cdf_[index];
    }
    std::size_t size() const noexcept { return cdf_.size() - 1; }
    const std::vector<double>& cdf() const { return cdf_; }

  private:
    std::vector<double> cdf_;
};

// ---- intersection (src/render/intersection.cpp) ------------------------------------------

double difference_of_products(double a, double b, double c, double d) {  // intersection.cpp:14-18
    const double cd         = c * d;
    const double correction = std::fma(-c, d, cd);
    return std::fma(a, b, -cd) + correction;
}

struct RayInterval {  // intersection.hpp:15-20
    double minimum = 1e-5;
    double maximum = infinity;
    void   validate() const {  // intersection.cpp:22-26
        if (!std::isfinite(minimum) || minimum < 0 || std::isnan(maximum) || maximum < minimum) {
            throw std::invalid_argument("Ray interval must satisfy 0 <= minimum <= maximum");
        }
    }
};

struct Bounds3 {  // intersection.hpp:24-35, intersection.cpp:28-50
    fvec3 minimum{infinityf(), infinityf(), infinityf()};
    fvec3 maximum{-infinityf(), -infinityf(), -infinityf()};
    static constexpr float infinityf() { return std::numeric_limits<float>::infinity(); }
    bool empty() const noexcept {
        return minimum.x > maximum.x || minimum.y > maximum.y || minimum.z > maximum.z;
    }
    void expand(fvec3 p) {
        minimum = {std::min(minimum.x, p.x), std::min(minimum.y, p.y), std::min(minimum.z, p.z)};
        maximum = {std::max(maximum.x, p.x), std::max(maximum.y, p.y), std::max(maximum.z, p.z)};
    }
    void expand(const Bounds3& b) {
        if (!b.empty()) {
            expand(b.minimum);
            expand(b.maximum);
        }
    }
    double surface_area() const noexcept {
        if (empty()) {
            return 0;
        }
        const auto e = widen(maximum) - widen(minimum);
        return 2 * (e.x * e.y + e.y * e.z + e.z * e.x);
    }
};

struct Ray {  // scene.hpp:27-30
    dvec3 origin{0, 0, 0};
    dvec3 direction{0, 0, -1};
};

struct TriangleHit {
    double distance = 0;
    dvec3  barycentric;
};

class RayQuery {  // intersection.cpp:52-152
  public:
    explicit RayQuery(const Ray& ray) : origin_(ray.origin), direction_(ray.direction) {
        for (int axis = 0; axis < 3; ++axis) {
            if (!std::isfinite(origin_[axis]) || !std::isfinite(direction_[axis])) {
                throw std::invalid_argument("Ray origin and direction must be finite");
            }
            inverse_[axis] = direction_[axis] == 0 ? 0 : 1 / direction_[axis];
        }
        if (std::abs(dot(direction_, direction_) - 1) > 1e-4) {
            throw std::invalid_argument("Ray direction must have unit length");
        }
        const auto absolute = dabs(direction_);
        z_                  = absolute.x > absolute.y ? 0 : 1;
        if (absolute.z > absolute[z_]) {
            z_ = 2;
        }
        x_ = (z_ + 1) % 3;
        y_ = (x_ + 1) % 3;
        if (direction_[z_] < 0) {
            std::swap(x_, y_);
        }
        shear_x_ = direction_[x_] / direction_[z_];
        shear_y_ = direction_[y_] / direction_[z_];
        scale_z_ = 1 / direction_[z_];
    }

    std::optional<double> intersect(const Bounds3& bounds, RayInterval interval) const {
        interval.validate();
        if (bounds.empty()) {
            return std::nullopt;
        }
        double enter = interval.minimum;
        double leave = interval.maximum;
        for (int axis = 0; axis < 3; ++axis) {
            if (direction_[axis] == 0) {
                if (origin_[axis] < bounds.minimum[axis] || origin_[axis] > bounds.maximum[axis]) {
                    return std::nullopt;
                }
                continue;
            }
            double near = (static_cast<double>(bounds.minimum[axis]) - origin_[axis]) * inverse_[axis];
            double far  = (static_cast<double>(bounds.maximum[axis]) - origin_[axis]) * inverse_[axis];
            if (near > far) {
                std::swap(near, far);
            }
            near  = std::nextafter(near, -infinity);
            far   = std::nextafter(far, infinity);
            enter = std::max(enter, near);
            leave = std::min(leave, far);
            if (enter > leave) {
                return std::nullopt;
            }
        }
        return enter;
    }

    std::optional<TriangleHit> intersect(const std::array<fvec3, 3>& vertices,
                                         RayInterval                 interval) const {
        interval.validate();
        std::array<dvec3, 3> p;
        for (std::size_t index = 0; index < 3; ++index) {
            const auto t = widen(vertices[index]) - origin_;
            p[index] = {t[x_] - shear_x_ * t[z_], t[y_] - shear_y_ * t[z_], t[z_] * scale_z_};
        }
        const double a = difference_of_products(p[1].x, p[2].y, p[1].y, p[2].x);
        const double b = difference_of_products(p[2].x, p[0].y, p[2].y, p[0].x);
        const double c = difference_of_products(p[0].x, p[1].y, p[0].y, p[1].x);
        if ((a < 0 || b < 0 || c < 0) && (a > 0 || b > 0 || c > 0)) {
            return std::nullopt;
        }
        const double determinant = a + b + c;
        if (determinant == 0) {
            return std::nullopt;
        }
        const double distance = (a * p[0].z + b * p[1].z + c * p[2].z) / determinant;
        if (distance < interval.minimum || distance > interval.maximum) {
            return std::nullopt;
        }
        const auto gamma = [](double operations) {
            const double error = operations * (dbl_eps * 0.5);
            return error / (1 - error);
        };
        const double x          = std::max({std::abs(p[0].x), std::abs(p[1].x), std::abs(p[2].x)});
        const double y          = std::max({std::abs(p[0].y), std::abs(p[1].y), std::abs(p[2].y)});
        const double z          = std::max({std::abs(p[0].z), std::abs(p[1].z), std::abs(p[2].z)});
        const double error_x    = gamma(5) * (x + z);
        const double error_y    = gamma(5) * (y + z);
        const double error_edge = 2 * (gamma(2) * x * y + error_y * x + error_x * y);
        const double edge       = std::max({std::abs(a), std::abs(b), std::abs(c)});
        const double error_distance =
            3 * (gamma(3) * edge * z + error_edge * z + gamma(3) * z * edge) / std::abs(determinant);
        if (distance <= error_distance) {
            return std::nullopt;
        }
        return TriangleHit{distance, dvec3{a, b, c} / determinant};
    }

  private:
    dvec3  origin_;
    dvec3  direction_;
    dvec3  inverse_;
    int    x_ = 0, y_ = 1, z_ = 2;
    double shear_x_ = 0, shear_y_ = 0, scale_z_ = 1;
};

// ---- textures (src/core/texture.cpp) -------------------------------------------------------

struct fvec2 {
    float x = 0, y = 0;
};

struct Image {  // linear RGB, origin top-left
    std::size_t        width = 0, height = 0;
    std::vector<fvec3> pixels;
    const fvec3& at(std::size_t x, std::size_t y) const { return pixels[y * width + x]; }
};

int wrap(int coordinate, int extent) {  // texture.cpp:13-15
    return (coordinate % extent + extent) % extent;
}

fvec2 image_uv(fvec2 uv) {  // texture.cpp:17-22
    if (!std::isfinite(uv.x) || !std::isfinite(uv.y)) {
        throw std::invalid_argument("Texture coordinates must be finite");
    }
    return {uv.x - std::floor(uv.x), 1.0F - (uv.y - std::floor(uv.y))};
}

// glm::mix of float vectors: x * (1 - a) + y * a.
fvec3 mixf(fvec3 x, fvec3 y, float a) {
    const float b = 1.0F - a;
    return {x.x * b + y.x * a, x.y * b + y.y * a, x.z * b + y.z * a};
}

Image downsample(const Image& source) {  // texture.cpp:25-50
    Image target;
    target.width  = std::max(std::size_t(1), source.width / 2);
    target.height = std::max(std::size_t(1), source.height / 2);
    target.pixels.resize(target.width * target.height);
    for (std::size_t y = 0; y < target.height; ++y) {
        for (std::size_t x = 0; x < target.width; ++x) {
            const double left   = double(x) * double(source.width) / double(target.width);
            const double right  = double(x + 1) * double(source.width) / double(target.width);
            const double top    = double(y) * double(source.height) / double(target.height);
            const double bottom = double(y + 1) * double(source.height) / double(target.height);
            dvec3        sum;
            double       weight_sum = 0;
            for (std::size_t sy = static_cast<std::size_t>(top); sy < static_cast<std::size_t>(std::ceil(bottom));
                 ++sy) {
                for (std::size_t sx = static_cast<std::size_t>(left);
                     sx < static_cast<std::size_t>(std::ceil(right)); ++sx) {
                    const double weight = (std::min(right, double(sx + 1)) - std::max(left, double(sx))) *
                                          (std::min(bottom, double(sy + 1)) - std::max(top, double(sy)));
                    sum += widen(source.at(sx, sy)) * weight;
                    weight_sum += weight;
                }
            }
            target.pixels[y * target.width + x] = narrow(sum / weight_sum);
        }
    }
    return target;
}

class Texture {  // texture.cpp:54-139
  public:
    explicit Texture(Image image) {
        if (image.width > 16384 || image.height > 16384 || image.width * image.height > 64u * 1024u * 1024u) {
            throw std::invalid_argument("Texture exceeds the 64-megapixel budget");
        }
        for (const auto& p : image.pixels) {
            if (!finite3(p)) {
                throw std::invalid_argument("Texture contains nonfinite samples");
            }
        }
        levels_.push_back(std::move(image));
        while (levels_.back().width > 1 || levels_.back().height > 1) {
            levels_.push_back(downsample(levels_.back()));
        }
    }
    const Image& level(std::size_t index) const { return levels_.at(index); }
    std::size_t  level_count() const noexcept { return levels_.size(); }

    fvec3 sample(fvec2 uv, float lod, std::uint32_t filter) const {
        if (!std::isfinite(lod)) {
            throw std::invalid_argument("Texture LOD must be finite");
        }
        if (filter == MR_FILTER_NEAREST) {
            const auto   coordinate = image_uv(uv);
            const auto&  image      = levels_.front();
            const int    x          = static_cast<int>(std::floor(coordinate.x * static_cast<float>(image.width)));
            const int    y          = static_cast<int>(std::floor(coordinate.y * static_cast<float>(image.height)));
            return image.at(static_cast<std::size_t>(wrap(x, static_cast<int>(image.width))),
                            static_cast<std::size_t>(wrap(y, static_cast<int>(image.height))));
        }
        if (filter == MR_FILTER_BILINEAR) {
            return bilinear(uv, 0);
        }
        const float clamped = std::clamp(lod, 0.0F, static_cast<float>(levels_.size() - 1));
        const auto  lower   = static_cast<std::size_t>(std::floor(clamped));
        const auto  upper   = std::min(lower + 1, levels_.size() - 1);
        return mixf(bilinear(uv, lower), bilinear(uv, upper), clamped - static_cast<float>(lower));
    }

  private:
    fvec3 bilinear(fvec2 uv, std::size_t level_index) const {
        const auto& image      = levels_.at(level_index);
        const auto  coordinate = image_uv(uv);
        const float x          = coordinate.x * static_cast<float>(image.width) - 0.5F;
        const float y          = coordinate.y * static_cast<float>(image.height) - 0.5F;
        const int   ix         = static_cast<int>(std::floor(x));
        const int   iy         = static_cast<int>(std::floor(y));
        const float tx         = x - std::floor(x);
        const float ty         = y - std::floor(y);
        const auto  texel      = [&](int px, int py) {
            return image.at(static_cast<std::size_t>(wrap(px, static_cast<int>(image.width))),
                            static_cast<std::size_t>(wrap(py, static_cast<int>(image.height))));
        };
        return mixf(mixf(texel(ix, iy), texel(ix + 1, iy), tx), mixf(texel(ix, iy + 1), texel(ix + 1, iy + 1), tx),
                    ty);
    }
    std::vector<Image> levels_;
};

// ---- scene snapshot ---------------------------------------------------------------------

struct Material {
    std::uint32_t kind = MR_MATERIAL_DIFFUSE;
    fvec3         base_color{0.7F, 0.7F, 0.7F};
    fvec3         emission{0, 0, 0};
    float         roughness    = 0.35F;
    float         ior          = 1.5F;
    bool          double_sided = true;
    std::uint32_t texture_filter = MR_FILTER_TRILINEAR;
    float         normal_scale   = 1;
    bool          normal_flip_y  = false;
    // RenderInstance's resolved textures (include/minirender/scene/scene.hpp:201-209).
    std::shared_ptr<const Texture> base_color_texture, normal_texture;
};

struct Corner {
    std::uint32_t position;
    fvec3         normal;
    fvec2         uv;
};

struct Mesh {
    std::vector<fvec3>                 positions;
    std::vector<std::array<Corner, 3>> triangles;
};

struct Instance {
    std::shared_ptr<const Mesh> mesh;
    Material                    material;
    float                       object_to_world[16];  // column-major
    float                       normal_to_world[9];   // column-major
};

struct MediumRegion {
    dvec3  minimum, maximum;
    dvec3  absorption, scattering;
    double anisotropy = 0;
    bool   enabled    = true;
    dvec3  extinction() const { return absorption + scattering; }
};

struct DirectionalLightDesc {
    fvec3 direction, color;
    float intensity;
};

struct Snapshot {
    mr_camera                         camera{};
    fvec3                             environment;
    std::vector<Instance>             instances;
    std::vector<DirectionalLightDesc> directional_lights;
    std::vector<MediumRegion>         media;
    std::shared_ptr<const Texture>    environment_texture;
    float                             environment_strength         = 1;
    float                             environment_rotation_degrees = 0;
};

// glm::vec3(object_to_world * glm::vec4(p, 1)) in float (bvh.cpp:68-69).
fvec3 transform_point(const float* m, fvec3 p) {
    fvec3 r;
    for (int row = 0; row < 3; ++row) {
        const float a = m[0 + row] * p.x;
        const float b = m[4 + row] * p.y;
        const float c = m[8 + row] * p.z;
        const float d = m[12 + row] * 1.0F;
        r[row]        = (a + b) + (c + d);
    }
    return r;
}

// glm::determinant(glm::dmat3(object_to_world)) (bvh.cpp:56).
double determinant3(const float* m) {
    const auto e = [m](int c, int r) { return static_cast<double>(m[4 * c + r]); };
    return +e(0, 0) * (e(1, 1) * e(2, 2) - e(2, 1) * e(1, 2)) -
           e(1, 0) * (e(0, 1) * e(2, 2) - e(2, 1) * e(0, 2)) +
           e(2, 0) * (e(0, 1) * e(1, 2) - e(1, 1) * e(0, 2));
}

// glm::dmat3(normal_to_world) * dvec3(n) (bvh.cpp:319-320).
dvec3 transform_normal(const float* m, fvec3 n) {
    dvec3 r;
    for (int row = 0; row < 3; ++row) {
        r[row] = (static_cast<double>(m[row]) * n.x + static_cast<double>(m[3 + row]) * n.y) +
                 static_cast<double>(m[6 + row]) * n.z;
    }
    return r;
}

void validate_camera(const mr_camera& c) {  // scene.cpp:141-155
    const fvec3 position = narrow(from(c.position)), target = narrow(from(c.target)),
                up = narrow(from(c.up));
    require(finite3(position) && finite3(target) && finite3(up), "Camera vectors must be finite");
    const fvec3 view{target.x - position.x, target.y - position.y, target.z - position.z};
    const float view_length = std::sqrt(view.x * view.x + view.y * view.y + view.z * view.z);
    require(view_length > 1e-6F, "Camera position and target must differ");
    const fvec3 side{view.y * up.z - up.y * view.z, view.z * up.x - up.z * view.x,
                     view.x * up.y - up.x * view.y};
    require(std::sqrt(side.x * side.x + side.y * side.y + side.z * side.z) > 1e-6F,
            "Camera up must not be parallel to view direction");
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

std::shared_ptr<Snapshot> make_snapshot(const mr_scene_desc& d) {
    auto s    = std::make_shared<Snapshot>();
    s->camera = d.camera;
    validate_camera(d.camera);
    s->environment = narrow(from(d.environment));
    require(finite3(s->environment) && s->environment.x >= 0 && s->environment.y >= 0 &&
                s->environment.z >= 0,
            "Environment must be finite and nonnegative");
    std::vector<std::shared_ptr<const Texture>> textures;
    for (std::uint32_t i = 0; i < d.texture_count; ++i) {
        const auto& src = d.textures[i];
        require(src.width > 0 && src.height > 0 && src.rgb, "Texture data is missing");
        Image image;
        image.width  = src.width;
        image.height = src.height;
        image.pixels.resize(static_cast<std::size_t>(src.width) * src.height);
        for (std::size_t k = 0; k < image.pixels.size(); ++k) {
            image.pixels[k] = {src.rgb[3 * k], src.rgb[3 * k + 1], src.rgb[3 * k + 2]};
        }
        textures.push_back(std::make_shared<const Texture>(std::move(image)));
    }
    const auto texture = [&](std::uint32_t one_based) -> std::shared_ptr<const Texture> {
        if (one_based == 0) {
            return nullptr;
        }
        require(one_based <= textures.size(), "Material references missing texture");
        return textures[one_based - 1];
    };
    s->environment_texture          = texture(d.environment_texture);
    s->environment_strength         = d.environment_strength;
    s->environment_rotation_degrees = d.environment_rotation_degrees;
    std::vector<std::shared_ptr<const Mesh>> meshes;
    for (std::uint32_t i = 0; i < d.mesh_count; ++i) {
        const auto& src = d.meshes[i];
        auto        m   = std::make_shared<Mesh>();
        require(src.position_count > 0 && src.triangle_count > 0,
                "Mesh must contain positions and triangles");
        m->positions.resize(src.position_count);
        for (std::uint32_t p = 0; p < src.position_count; ++p) {
            m->positions[p] = {src.positions[3 * p], src.positions[3 * p + 1],
                               src.positions[3 * p + 2]};
            require(finite3(m->positions[p]), "Mesh position must be finite");
        }
        m->triangles.resize(src.triangle_count);
        for (std::uint32_t t = 0; t < src.triangle_count; ++t) {
            for (int c = 0; c < 3; ++c) {
                const auto& corner = src.corners[3 * t + c];
                require(corner.position < src.position_count, "Mesh position index is out of range");
                m->triangles[t][c] = {corner.position,
                                      fvec3{corner.normal[0], corner.normal[1], corner.normal[2]},
                                      fvec2{corner.uv[0], corner.uv[1]}};
            }
        }
        meshes.push_back(m);
    }
    std::vector<Material> materials;
    for (std::uint32_t i = 0; i < d.material_count; ++i) {
        const auto& src = d.materials[i];
        Material    m;
        m.kind         = src.kind;
        m.base_color   = narrow(from(src.base_color));
        m.emission     = narrow(from(src.emission));
        m.roughness    = src.roughness;
        m.ior          = src.ior;
        m.double_sided = src.double_sided != 0;
        m.texture_filter     = src.texture_filter;
        m.normal_scale       = src.normal_scale;
        m.normal_flip_y      = src.normal_flip_y != 0;
        m.base_color_texture = texture(src.base_color_texture);
        m.normal_texture     = texture(src.normal_texture);
        require(m.texture_filter <= MR_FILTER_TRILINEAR, "Unknown texture filter");
        require(std::isfinite(m.normal_scale), "Normal scale must be finite");
        require(finite3(m.base_color) && m.base_color.x >= 0 && m.base_color.y >= 0 &&
                    m.base_color.z >= 0 && m.base_color.x <= 1 && m.base_color.y <= 1 &&
                    m.base_color.z <= 1,
                "Material base color must be in [0,1]");
        require(finite3(m.emission) && m.emission.x >= 0 && m.emission.y >= 0 && m.emission.z >= 0,
                "Material emission must be nonnegative");
        require(std::isfinite(m.roughness) && m.roughness >= 0 && m.roughness <= 1,
                "Roughness must be in [0,1]");
        require(std::isfinite(m.ior) && m.ior > 0, "IOR must be positive");
        require(m.kind <= MR_MATERIAL_DIELECTRIC, "Material kind is not supported");
        materials.push_back(m);
    }
    for (std::uint32_t i = 0; i < d.instance_count; ++i) {
        const auto& src = d.instances[i];
        require(src.mesh < d.mesh_count, "Object references missing mesh");
        require(src.material < d.material_count, "Object references missing material");
        Instance inst;
        inst.mesh     = meshes[src.mesh];
        inst.material = materials[src.material];
        std::memcpy(inst.object_to_world, src.object_to_world, sizeof(inst.object_to_world));
        std::memcpy(inst.normal_to_world, src.normal_to_world, sizeof(inst.normal_to_world));
        s->instances.push_back(std::move(inst));
    }
    for (std::uint32_t i = 0; i < d.directional_light_count; ++i) {
        const auto&          src = d.directional_lights[i];
        DirectionalLightDesc l{narrow(from(src.direction)), narrow(from(src.color)), src.intensity};
        s->directional_lights.push_back(l);
    }
    require(d.medium_count <= 32, "Scene supports at most 32 medium regions");
    for (std::uint32_t i = 0; i < d.medium_count; ++i) {
        const auto&  src = d.media[i];
        MediumRegion r;
        r.minimum    = from(src.minimum);
        r.maximum    = from(src.maximum);
        r.absorption = from(src.absorption);
        r.scattering = from(src.scattering);
        r.anisotropy = src.anisotropy;
        r.enabled    = src.enabled != 0;
        require(finite3(r.absorption) && finite3(r.scattering) && finite3(r.extinction()) &&
                    r.absorption.x >= 0 && r.absorption.y >= 0 && r.absorption.z >= 0 &&
                    r.scattering.x >= 0 && r.scattering.y >= 0 && r.scattering.z >= 0 &&
                    std::isfinite(r.anisotropy) && std::abs(r.anisotropy) < 1,
                "Medium coefficients must be finite/nonnegative and |g| < 1");
        require(finite3(r.minimum) && finite3(r.maximum) && r.minimum.x < r.maximum.x &&
                    r.minimum.y < r.maximum.y && r.minimum.z < r.maximum.z,
                "Medium region requires an ID and a finite positive box");
        s->media.push_back(r);
    }
    return s;
}

// ---- BVH (src/render/bvh.cpp) ------------------------------------------------------------

constexpr std::uint32_t bin_count           = 12;  // bvh.cpp:15
constexpr std::size_t   maximum_build_depth = 48;  // bvh.cpp:16

std::uint32_t bin_index(float centroid, float low, float high) {  // bvh.cpp:23-27
    const double coordinate =
        (static_cast<double>(centroid) - low) / (static_cast<double>(high) - low);
    return std::min(static_cast<std::uint32_t>(coordinate * bin_count), bin_count - 1);
}

struct TraceStatistics {
    std::uint64_t bounds_tests   = 0;
    std::uint64_t triangle_tests = 0;
};

struct SurfaceHit {
    double        distance = 0;
    dvec3         position;
    fvec3         geometric_normal;
    fvec3         shading_normal;
    fvec2         uv;
    dvec3         barycentric;
    std::uint32_t instance_index = 0;
    std::uint32_t triangle_index = 0;
    std::uint32_t primitive      = 0;
    bool          front_face     = true;
    dvec3         position_error;
};

// uv_tangents (src/geometry/uv_tangents.cpp:12-36): the triangle's unit dP/du and dP/dv.
bool uv_tangents(const std::array<fvec3, 3>& positions, const std::array<fvec2, 3>& coordinates, dvec3& u_axis,
                 dvec3& v_axis) {
    const auto a = widen(positions[1]) - widen(positions[0]);
    const auto b = widen(positions[2]) - widen(positions[0]);
    dvec2 s{double(coordinates[1].x) - double(coordinates[0].x), double(coordinates[1].y) - double(coordinates[0].y)};
    dvec2 t{double(coordinates[2].x) - double(coordinates[0].x), double(coordinates[2].y) - double(coordinates[0].y)};
    const double scale = std::max({std::abs(s.x), std::abs(s.y), std::abs(t.x), std::abs(t.y)});
    if (!std::isfinite(scale) || scale == 0) {
        return false;
    }
    s.x /= scale, s.y /= scale;
    t.x /= scale, t.y /= scale;
    const double determinant = s.x * t.y - s.y * t.x;
    if (!std::isfinite(determinant) || std::abs(determinant) < 1e-12) {
        return false;
    }
    const auto   u  = (t.y * a - s.y * b) / determinant;
    const auto   v  = (-t.x * a + s.x * b) / determinant;
    const double lu = length(u);
    const double lv = length(v);
    if (!std::isfinite(lu) || !std::isfinite(lv) || lu == 0 || lv == 0) {
        return false;
    }
    u_axis = u / lu;
    v_axis = v / lv;
    return true;
}

struct BvhStatistics {
    std::size_t triangles = 0, nodes = 0, leaves = 0, maximum_depth = 0;
};

class SceneBvh {
  public:
    struct Primitive {
        std::array<fvec3, 3> vertices;
        std::uint32_t        instance;
        std::uint32_t        triangle;
    };
    struct BuildPrimitive {
        Bounds3 bounds;
        fvec3   centroid;
    };
    struct Node {
        Bounds3       bounds;
        std::uint32_t first = 0, right = 0, count = 0;
    };
    struct PrimitiveHit {
        std::uint32_t primitive;
        TriangleHit   hit;
    };

    // bvh.cpp:31-99 (world-space flattening + build); `imported` replaces the build.
    SceneBvh(std::shared_ptr<const Snapshot> scene, const mr_bvh_desc* imported = nullptr)
        : scene_(std::move(scene)) {
        std::size_t total = 0;
        for (const auto& instance : scene_->instances) {
            total += instance.mesh->triangles.size();
        }
        if (total > std::numeric_limits<std::uint32_t>::max() / 2) {
            throw std::length_error("Scene triangle count exceeds BVH index range");
        }
        primitives_.reserve(total);
        std::vector<BuildPrimitive> build_primitives;
        build_primitives.reserve(total);
        for (std::size_t ii = 0; ii < scene_->instances.size(); ++ii) {
            const auto& instance = scene_->instances[ii];
            mirrored_.push_back(determinant3(instance.object_to_world) < 0);
            for (std::size_t index = 0; index < instance.mesh->triangles.size(); ++index) {
                const auto&    triangle = instance.mesh->triangles[index];
                Primitive      primitive{};
                BuildPrimitive bp{};
                primitive.instance = static_cast<std::uint32_t>(ii);
                primitive.triangle = static_cast<std::uint32_t>(index);
                dvec3 center;
                for (int corner = 0; corner < 3; ++corner) {
                    const auto world = transform_point(
                        instance.object_to_world,
                        instance.mesh->positions[triangle[corner].position]);
                    if (!finite3(world)) {
                        throw std::invalid_argument("Transformed triangle position is not finite");
                    }
                    primitive.vertices[corner] = world;
                    bp.bounds.expand(world);
                    center += widen(world) / 3.0;
                }
                const auto edge1  = widen(primitive.vertices[1]) - widen(primitive.vertices[0]);
                const auto edge2  = widen(primitive.vertices[2]) - widen(primitive.vertices[0]);
                const auto normal = cross(edge1, edge2);
                if (dot(normal, normal) == 0) {
                    throw std::invalid_argument(
                        "Transform collapses a triangle at float precision");
                }
                bp.centroid = narrow(center);
                primitives_.push_back(primitive);
                build_primitives.push_back(bp);
            }
        }
        statistics_.triangles = primitives_.size();
        order_.resize(primitives_.size());
        for (std::uint32_t i = 0; i < order_.size(); ++i) {
            order_[i] = i;
        }
        if (imported) {
            import(*imported);
        } else if (!primitives_.empty()) {
            nodes_.reserve(primitives_.size() * 2 - 1);
            build(0, static_cast<std::uint32_t>(primitives_.size()), 0, build_primitives);
        }
        statistics_.nodes = nodes_.size();
    }

    void import(const mr_bvh_desc& d) {
        require(d.primitive_count == primitives_.size(), "Imported BVH primitive count differs");
        nodes_.resize(d.node_count);
        for (std::uint32_t i = 0; i < d.node_count; ++i) {
            const auto& n = d.nodes[i];
            nodes_[i].bounds.minimum = {n.minimum[0], n.minimum[1], n.minimum[2]};
            nodes_[i].bounds.maximum = {n.maximum[0], n.maximum[1], n.maximum[2]};
            nodes_[i].first          = n.first;
            nodes_[i].right          = n.right;
            nodes_[i].count          = n.count;
            statistics_.leaves += n.count > 0;
        }
        for (std::uint32_t i = 0; i < d.primitive_count; ++i) {
            order_[i] = d.order[i];
        }
    }

    // bvh.cpp:101-196, recursive 12-bin SAH build in DFS pre-order.
    std::uint32_t build(std::uint32_t begin, std::uint32_t end, std::size_t depth,
                        const std::vector<BuildPrimitive>& primitives) {
        const auto node_index = static_cast<std::uint32_t>(nodes_.size());
        nodes_.emplace_back();
        Bounds3 bounds;
        Bounds3 centroids;
        for (auto index = begin; index < end; ++index) {
            bounds.expand(primitives[order_[index]].bounds);
            centroids.expand(primitives[order_[index]].centroid);
        }
        const auto count          = end - begin;
        statistics_.maximum_depth = std::max(statistics_.maximum_depth, depth);
        const auto leaf           = [&] {
            nodes_[node_index] = {bounds, begin, 0, count};
            ++statistics_.leaves;
            return node_index;
        };
        if (count <= 4 || depth >= maximum_build_depth) {
            return leaf();
        }
        struct Bin {
            Bounds3       bounds;
            std::uint32_t count = 0;
        };
        double        best_cost   = static_cast<double>(count);
        int           best_axis   = -1;
        std::uint32_t best_split  = 0;
        const double  parent_area = bounds.surface_area();
        for (int axis = 0; axis < 3; ++axis) {
            if (centroids.maximum[axis] == centroids.minimum[axis]) {
                continue;
            }
            std::array<Bin, bin_count> bins{};
            for (auto index = begin; index < end; ++index) {
                const auto& primitive = primitives[order_[index]];
                auto&       bin       = bins[bin_index(primitive.centroid[axis],
                                                       centroids.minimum[axis],
                                                       centroids.maximum[axis])];
                ++bin.count;
                bin.bounds.expand(primitive.bounds);
            }
            std::array<Bounds3, bin_count>       right_bounds;
            std::array<std::uint32_t, bin_count> right_counts{};
            Bounds3                              right;
            std::uint32_t                        right_count = 0;
            for (std::uint32_t index = bin_count; index-- > 0;) {
                right.expand(bins[index].bounds);
                right_count += bins[index].count;
                right_bounds[index] = right;
                right_counts[index] = right_count;
            }
            Bounds3       left;
            std::uint32_t left_count = 0;
            for (std::uint32_t split = 0; split + 1 < bin_count; ++split) {
                left.expand(bins[split].bounds);
                left_count += bins[split].count;
                if (left_count == 0 || right_counts[split + 1] == 0) {
                    continue;
                }
                const double cost =
                    1 + (left.surface_area() * left_count +
                         right_bounds[split + 1].surface_area() * right_counts[split + 1]) /
                            parent_area;
                if (cost < best_cost) {
                    best_cost  = cost;
                    best_axis  = axis;
                    best_split = split;
                }
            }
        }
        if (best_axis < 0) {
            return leaf();
        }
        const auto first  = order_.begin() + begin;
        const auto last   = order_.begin() + end;
        const auto middle = std::partition(first, last, [&](std::uint32_t index) {
            return bin_index(primitives[index].centroid[best_axis], centroids.minimum[best_axis],
                             centroids.maximum[best_axis]) <= best_split;
        });
        const auto split  = static_cast<std::uint32_t>(middle - order_.begin());
        const auto left   = build(begin, split, depth + 1, primitives);
        const auto right  = build(split, end, depth + 1, primitives);
        nodes_[node_index] = {bounds, left, right, 0};
        return node_index;
    }

    // bvh.cpp:206-300, ordered DFS with closed intervals and the lower-id tie rule.
    std::optional<PrimitiveHit> trace(const Ray& ray, RayInterval interval, bool any_hit,
                                      TraceStatistics* statistics) const {
        interval.validate();
        const RayQuery query(ray);
        if (nodes_.empty()) {
            return std::nullopt;
        }
        const auto box_hit = [&](const Bounds3& bounds) {
            if (statistics) {
                ++statistics->bounds_tests;
            }
            return query.intersect(bounds, interval);
        };
        const auto root = box_hit(nodes_[0].bounds);
        if (!root) {
            return std::nullopt;
        }
        struct Entry {
            std::uint32_t node;
            double        enter;
        };
        std::array<Entry, maximum_build_depth + 2> stack{};
        std::size_t                                pending = 0;
        stack[pending++]                                   = {0, *root};
        std::optional<PrimitiveHit>                result;
        while (pending) {
            const auto entry = stack[--pending];
            if (entry.enter > interval.maximum) {
                continue;
            }
            const auto& node = nodes_[entry.node];
            if (node.count) {
                for (std::uint32_t offset = 0; offset < node.count; ++offset) {
                    const auto primitive = order_[node.first + offset];
                    if (statistics) {
                        ++statistics->triangle_tests;
                    }
                    const auto hit = query.intersect(primitives_[primitive].vertices, interval);
                    if (hit) {
                        const auto& candidate = primitives_[primitive];
                        const auto& instance  = scene_->instances[candidate.instance];
                        if (!instance.material.double_sided) {
                            const auto edge1 =
                                widen(candidate.vertices[1]) - widen(candidate.vertices[0]);
                            const auto edge2 =
                                widen(candidate.vertices[2]) - widen(candidate.vertices[0]);
                            const auto outward =
                                cross(edge1, edge2) * (mirrored_[candidate.instance] ? -1.0 : 1.0);
                            if (dot(ray.direction, outward) >= 0) {
                                continue;
                            }
                        }
                    }
                    if (hit && (!result || hit->distance < result->hit.distance ||
                                (hit->distance == result->hit.distance &&
                                 primitive < result->primitive))) {
                        result = PrimitiveHit{primitive, *hit};
                        if (any_hit) {
                            return result;
                        }
                        interval.maximum = hit->distance;
                    }
                }
            } else {
                const auto left  = box_hit(nodes_[node.first].bounds);
                const auto right = box_hit(nodes_[node.right].bounds);
                if (left && right) {
                    const bool left_nearer = *left <= *right;
                    stack[pending++] =
                        left_nearer ? Entry{node.right, *right} : Entry{node.first, *left};
                    stack[pending++] =
                        left_nearer ? Entry{node.first, *left} : Entry{node.right, *right};
                } else if (left) {
                    stack[pending++] = {node.first, *left};
                } else if (right) {
                    stack[pending++] = {node.right, *right};
                }
            }
        }
        return result;
    }

    // bvh.cpp:302-370, normal maps decoded in the triangle's UV tangent frame.
    SurfaceHit surface_hit(const Ray& ray, const PrimitiveHit& hit) const {
        const auto& primitive = primitives_[hit.primitive];
        const auto& instance  = scene_->instances[primitive.instance];
        const auto& triangle  = instance.mesh->triangles[primitive.triangle];
        const auto  edge1     = widen(primitive.vertices[1]) - widen(primitive.vertices[0]);
        const auto  edge2     = widen(primitive.vertices[2]) - widen(primitive.vertices[0]);
        auto        geometric = normalize(cross(edge1, edge2));
        if (mirrored_[primitive.instance]) {
            geometric = -geometric;
        }
        dvec3  shading, position, absolute_position;
        dvec2  uv;
        for (int corner = 0; corner < 3; ++corner) {
            const double weight = hit.hit.barycentric[corner];
            shading += weight * normalize(transform_normal(instance.normal_to_world,
                                                           triangle[corner].normal));
            uv.x += weight * static_cast<double>(triangle[corner].uv.x);
            uv.y += weight * static_cast<double>(triangle[corner].uv.y);
            const auto term = weight * widen(primitive.vertices[corner]);
            position += term;
            absolute_position += dabs(term);
        }
        if (dot(shading, shading) < 1e-24) {
            shading = geometric;
        } else {
            shading = normalize(shading);
            if (dot(shading, geometric) < 0) {
                shading = -shading;
            }
        }
        const fvec2 uv_f{static_cast<float>(uv.x), static_cast<float>(uv.y)};
        const auto& material = instance.material;
        if (material.normal_texture && material.normal_scale > 0) {
            const std::array<fvec2, 3> coords{triangle[0].uv, triangle[1].uv, triangle[2].uv};
            dvec3 axis_u, axis_v;
            if (uv_tangents(primitive.vertices, coords, axis_u, axis_v)) {
                const auto t0 = axis_u - shading * dot(axis_u, shading);
                if (dot(t0, t0) > 1e-12) {
                    const auto t = normalize(t0);
                    auto       b = cross(shading, t);
                    if (dot(b, axis_v) < 0) {
                        b = -b;
                    }
                    // glm::dvec3(sample) * 2. - 1.
                    auto sample = widen(material.normal_texture->sample(uv_f, 0, material.texture_filter)) * 2.0 -
                                  dvec3{1, 1, 1};
                    sample.x *= material.normal_scale;
                    sample.y *= material.normal_scale * (material.normal_flip_y ? -1. : 1.);
                    const auto mapped = t * sample.x + b * sample.y + shading * sample.z;
                    if (dot(mapped, geometric) > 1e-8) {
                        shading = normalize(mapped);
                    }
                }
            }
        }
        SurfaceHit result;
        result.distance         = hit.hit.distance;
        result.position         = position;
        result.geometric_normal = narrow(geometric);
        result.shading_normal   = narrow(shading);
        result.uv               = uv_f;
        result.barycentric      = hit.hit.barycentric;
        result.instance_index   = primitive.instance;
        result.triangle_index   = primitive.triangle;
        result.primitive        = hit.primitive;
        result.front_face       = dot(ray.direction, geometric) < 0;
        result.position_error   = absolute_position * (7 * offset_eps);
        return result;
    }

    std::optional<SurfaceHit> intersect(const Ray& ray, RayInterval interval,
                                        TraceStatistics* statistics) const {
        const auto hit = trace(ray, interval, false, statistics);
        return hit ? std::optional(surface_hit(ray, *hit)) : std::nullopt;
    }
    bool occluded(const Ray& ray, RayInterval interval, TraceStatistics* statistics) const {
        return trace(ray, interval, true, statistics).has_value();
    }

    // Whole-tree SAH cost with C_T = C_I = 1 (the constants of bvh.cpp:134-135).
    double sah_cost() const {
        if (nodes_.empty()) {
            return 0;
        }
        const double root = nodes_[0].bounds.surface_area();
        double       cost = 0;
        for (const auto& n : nodes_) {
            const double a = n.bounds.surface_area() / root;
            cost += n.count ? a * n.count : a;
        }
        return cost;
    }

    const std::vector<Node>&          nodes() const { return nodes_; }
    const std::vector<std::uint32_t>& order() const { return order_; }
    const std::vector<Primitive>&     primitives() const { return primitives_; }
    const BvhStatistics&              statistics() const { return statistics_; }

  private:
    std::shared_ptr<const Snapshot> scene_;
    std::vector<Primitive>          primitives_;
    std::vector<std::uint32_t>      order_;
    std::vector<Node>               nodes_;
    std::vector<bool>               mirrored_;
    BvhStatistics                   statistics_;
};

// ---- BSDF (src/render/bsdf.cpp) -----------------------------------------------------------

constexpr double delta_alpha = 1e-6;  // bsdf.cpp:17

dvec3 unit_direction(dvec3 value) {  // bsdf.cpp:23-28
    if (!finite3(value) || std::abs(dot(value, value) - 1) > 1e-4) {
        throw std::invalid_argument("BSDF direction must be finite and have unit length");
    }
    return normalize(value);
}

void check_bsdf_sample(double value) {  // bsdf.cpp:30-34
    if (!(value >= 0 && value < 1)) {
        throw std::invalid_argument("BSDF sample coordinate must be in [0,1)");
    }
}

double distribution(dvec3 m, double alpha) {  // bsdf.cpp:36-41, GGX D
    const double a2          = alpha * alpha;
    const double denominator = m.x * m.x + m.y * m.y + a2 * m.z * m.z;
    return m.z > 0 ? a2 / (pi * denominator * denominator) : 0;
}

double smith_g1_over_cosine(dvec3 v, double alpha) {  // bsdf.cpp:43-48
    if (v.z <= 0) {
        return 0;
    }
    return 2 / (v.z + std::sqrt(v.z * v.z + alpha * alpha * (v.x * v.x + v.y * v.y)));
}

double fresnel_from_transmission(double cosine, double sin2, double eta_i,
                                 double eta_t) {  // bsdf.cpp:51-64
    if (eta_i == eta_t) {
        return 0;
    }
    if (sin2 >= 1) {
        return 1;
    }
    const double transmitted_cosine = std::sqrt(1 - sin2);
    const double parallel           = (eta_t * cosine - eta_i * transmitted_cosine) /
                            (eta_t * cosine + eta_i * transmitted_cosine);
    const double perpendicular = (eta_i * cosine - eta_t * transmitted_cosine) /
                                 (eta_i * cosine + eta_t * transmitted_cosine);
    return 0.5 * (parallel * parallel + perpendicular * perpendicular);
}

dvec3 schlick(dvec3 f0, double cosine) {  // bsdf.cpp:66-69
    const double t  = 1 - std::clamp(cosine, 0.0, 1.0);
    const double t5 = t * t * t * t * t;
    return f0 + (dvec3{1, 1, 1} - f0) * t5;
}

dvec3 sample_visible_normal(dvec3 wo, dvec2 u, double alpha) {  // bsdf.cpp:72-85, Heitz 2018
    const auto   view  = normalize(dvec3{alpha * wo.x, alpha * wo.y, wo.z});
    const double lensq = view.x * view.x + view.y * view.y;
    const auto t1 = lensq > 0 ? dvec3{-view.y, view.x, 0} / std::sqrt(lensq) : dvec3{1, 0, 0};
    const auto t2 = cross(view, t1);
    const double radius = std::sqrt(u.x);
    const double x      = radius * std::cos(2 * pi * u.y);
    const double blend  = 0.5 * (1 + view.z);
    const double y =
        (1 - blend) * std::sqrt(std::max(0.0, 1 - x * x)) + blend * radius * std::sin(2 * pi * u.y);
    const auto normal = x * t1 + y * t2 + std::sqrt(std::max(0.0, 1 - x * x - y * y)) * view;
    return normalize(dvec3{alpha * normal.x, alpha * normal.y, std::max(0.0, normal.z)});
}

class ShadingFrame {  // bsdf.cpp:89-110
  public:
    explicit ShadingFrame(dvec3 normal) {
        const double maximum = std::max({std::abs(normal.x), std::abs(normal.y), std::abs(normal.z)});
        if (!finite3(normal) || maximum == 0) {
            throw std::invalid_argument("Shading normal must be finite and nonzero");
        }
        normal_           = normalize(normal / maximum);
        const auto helper = std::abs(normal_.z) < 0.999 ? dvec3{0, 0, 1} : dvec3{0, 1, 0};
        tangent_          = normalize(cross(helper, normal_));
        bitangent_        = cross(normal_, tangent_);
    }
    dvec3 to_local(dvec3 w) const { return {dot(w, tangent_), dot(w, bitangent_), dot(w, normal_)}; }
    dvec3 to_world(dvec3 l) const { return l.x * tangent_ + l.y * bitangent_ + l.z * normal_; }
    const dvec3& normal() const { return normal_; }

  private:
    dvec3 tangent_, bitangent_, normal_;
};

double fresnel_dielectric(double cosine, double eta_i, double eta_t) {  // bsdf.cpp:112-120
    if (!std::isfinite(cosine) || cosine < 0 || cosine > 1 || !std::isfinite(eta_i) ||
        !std::isfinite(eta_t) || eta_i <= 0 || eta_t <= 0) {
        throw std::invalid_argument("Fresnel requires cosine in [0,1] and positive finite IORs");
    }
    const double ratio = eta_i / eta_t;
    const double sin2  = ratio * ratio * std::max(0.0, 1 - cosine * cosine);
    return fresnel_from_transmission(cosine, sin2, eta_i, eta_t);
}

enum class Event { diffuse, glossy, specular_reflection, specular_transmission };

struct BsdfSample {
    dvec3  direction;
    dvec3  weight;
    double probability = 0;
    bool   discrete    = false;
    Event  event       = Event::diffuse;
    double eta         = 1;
};

class Bsdf {  // bsdf.cpp:122-277 without cloth and energy compensation
  public:
    // color = base_color * clamp(texture colour, 0, 1) (bsdf.cpp:122-141).
    Bsdf(const Material& material, bool front_face, bool importance = false,
         fvec3 texture_color = fvec3{1, 1, 1})
        : kind_(material.kind),
          color_(widen(material.base_color) * dvec3{std::clamp(double(texture_color.x), 0.0, 1.0),
                                                    std::clamp(double(texture_color.y), 0.0, 1.0),
                                                    std::clamp(double(texture_color.z), 0.0, 1.0)}),
          alpha_(static_cast<double>(material.roughness) * material.roughness),
          eta_i_(front_face ? 1 : material.ior), eta_t_(front_face ? material.ior : 1),
          importance_(importance) {}

    bool is_delta() const noexcept {
        return kind_ == MR_MATERIAL_MIRROR || kind_ == MR_MATERIAL_DIELECTRIC ||
               (kind_ == MR_MATERIAL_CONDUCTOR && alpha_ <= delta_alpha);
    }
    dvec3 evaluate_normalized(dvec3 wo, dvec3 wi) const {
        if (wo.z <= 0 || wi.z <= 0 || is_delta()) {
            return {0, 0, 0};
        }
        if (kind_ == MR_MATERIAL_DIFFUSE) {
            return color_ / pi;
        }
        const auto m = normalize(wo + wi);
        return schlick(color_, dot(wo, m)) * distribution(m, alpha_) *
               smith_g1_over_cosine(wo, alpha_) * smith_g1_over_cosine(wi, alpha_) / 4.0;
    }
    double pdf_normalized(dvec3 wo, dvec3 wi) const {
        if (wo.z <= 0 || wi.z <= 0 || is_delta()) {
            return 0;
        }
        if (kind_ == MR_MATERIAL_DIFFUSE) {
            return cosine_hemisphere_pdf(wi);
        }
        const auto m = normalize(wo + wi);
        return distribution(m, alpha_) * smith_g1_over_cosine(wo, alpha_) / 4;
    }
    dvec3  evaluate(dvec3 wo, dvec3 wi) const { return evaluate_normalized(unit_direction(wo), unit_direction(wi)); }
    double pdf(dvec3 wo, dvec3 wi) const { return pdf_normalized(unit_direction(wo), unit_direction(wi)); }

    std::optional<BsdfSample> sample(dvec3 wo, double component, dvec2 u) const {
        wo = unit_direction(wo);
        check_bsdf_sample(component);
        check_bsdf_sample(u.x);
        check_bsdf_sample(u.y);
        if (wo.z <= 0) {
            return std::nullopt;
        }
        const dvec3 reflected{-wo.x, -wo.y, wo.z};
        if (kind_ == MR_MATERIAL_DIELECTRIC) {
            const double ratio = eta_i_ / eta_t_;
            const double sin2  = ratio * ratio * (wo.x * wo.x + wo.y * wo.y);
            const double reflectance =
                fresnel_from_transmission(std::clamp(wo.z, 0.0, 1.0), sin2, eta_i_, eta_t_);
            if (component < reflectance) {
                return BsdfSample{reflected, {1, 1, 1}, reflectance, true,
                                  Event::specular_reflection, 1};
            }
            const dvec3  transmitted{-ratio * wo.x, -ratio * wo.y, -std::sqrt(std::max(0.0, 1 - sin2))};
            const double scale = importance_ ? 1 : ratio * ratio;
            return BsdfSample{transmitted, color_ * scale, 1 - reflectance, true,
                              Event::specular_transmission, eta_t_ / eta_i_};
        }
        if (is_delta()) {
            const auto weight = kind_ == MR_MATERIAL_MIRROR ? color_ : schlick(color_, wo.z);
            return BsdfSample{reflected, weight, 1, true, Event::specular_reflection, 1};
        }
        dvec3 wi;
        if (kind_ == MR_MATERIAL_DIFFUSE) {
            wi = sample_cosine_hemisphere(u);
        } else {
            const auto m = sample_visible_normal(wo, u, alpha_);
            wi           = normalize(2 * dot(wo, m) * m - wo);
        }
        if (wi.z <= 0) {
            return std::nullopt;
        }
        const auto   evaluated_wi = unit_direction(wi);
        const double density      = pdf_normalized(wo, evaluated_wi);
        const auto   weight       = evaluate_normalized(wo, evaluated_wi) * wi.z / density;
        return BsdfSample{wi, weight, density, false,
                          kind_ == MR_MATERIAL_DIFFUSE ? Event::diffuse : Event::glossy, 1};
    }

  private:
    std::uint32_t kind_;
    dvec3         color_;
    double        alpha_;
    double        eta_i_;
    double        eta_t_;
    bool          importance_;
};

// ---- lights (src/render/light.cpp) --------------------------------------------------------

double luminance(dvec3 c) {  // light.cpp:21-23
    return dot(c, dvec3{0.2126, 0.7152, 0.0722});
}

double area_density(dvec3 reference, dvec3 point, dvec3 normal, double area) {  // light.cpp:49-57
    const auto   difference       = point - reference;
    const double squared_distance = dot(difference, difference);
    if (squared_distance == 0) {
        return 0;
    }
    const double cosine = std::abs(dot(normal, -difference / std::sqrt(squared_distance)));
    return cosine > 0 ? squared_distance / (area * cosine) : 0;
}

dvec3 positive(dvec3 c) { return {std::max(c.x, 0.0), std::max(c.y, 0.0), std::max(c.z, 0.0)}; }  // light.cpp:25-27

dvec3 unit_light_direction(dvec3 direction) {  // light.cpp:35-40
    if (!finite3(direction) || std::abs(dot(direction, direction) - 1) > 1e-4) {
        throw std::invalid_argument("Light direction must be finite and have unit length");
    }
    return normalize(direction);
}

// glm::mix of double vectors: x * (1 - a) + y * a.
dvec3 mixd(dvec3 x, dvec3 y, double a) { return x * (1 - a) + y * a; }

constexpr double uniform_fraction = 0.05;  // light.cpp:15

// EnvironmentLight (light.cpp:61-195): constant radiance plus an optional lat-long map (origin at
// the image's top left, +Y north, longitude 0 along +X increasing towards +Z), importance-sampled
// over a grid of at most 1024x512 texels (a mip level) weighted by luminance and solid angle,
// mixed with 5% uniform sphere density.
class EnvironmentLight {
  public:
    explicit EnvironmentLight(const Snapshot& scene)
        : constant_(widen(scene.environment)), texture_(scene.environment_texture),
          strength_(scene.environment_strength),
          rotation_(std::remainder(static_cast<double>(scene.environment_rotation_degrees), 360.0) * pi / 180),
          integral_(4 * pi * luminance(constant_)) {
        if (!texture_ || strength_ == 0) {
            return;
        }
        while (texture_->level(grid_level_).width > 1024 || texture_->level(grid_level_).height > 512) {
            ++grid_level_;
        }
        const auto&         image = texture_->level(grid_level_);
        std::vector<double> weights;
        weights.reserve(image.width * image.height);
        double map_integral = 0;
        for (std::size_t y = 0; y < image.height; ++y) {
            const double theta0 = pi * static_cast<double>(y) / static_cast<double>(image.height);
            const double theta1 = pi * static_cast<double>(y + 1) / static_cast<double>(image.height);
            const double angle  = (2 * pi / static_cast<double>(image.width)) * 2 *
                                 std::sin((theta0 + theta1) * 0.5) * std::sin((theta1 - theta0) * 0.5);
            solid_angles_.push_back(angle);
            for (std::size_t x = 0; x < image.width; ++x) {
                const double weight = luminance(positive(widen(image.at(x, y)))) * angle;
                weights.push_back(weight);
                map_integral += weight;
            }
        }
        pixels_  = DiscreteDistribution(weights);
        uniform_ = map_integral == 0;
        double      full_integral = 0;
        const auto& full          = texture_->level(0);
        for (std::size_t y = 0; y < full.height; ++y) {
            const double theta0 = pi * static_cast<double>(y) / static_cast<double>(full.height);
            const double theta1 = pi * static_cast<double>(y + 1) / static_cast<double>(full.height);
            const double angle  = (2 * pi / static_cast<double>(full.width)) * 2 *
                                 std::sin((theta0 + theta1) * 0.5) * std::sin((theta1 - theta0) * 0.5);
            for (std::size_t x = 0; x < full.width; ++x) {
                full_integral += luminance(positive(widen(full.at(x, y)))) * angle;
            }
        }
        integral_ += strength_ * full_integral;
    }

    dvec2 coordinates(dvec3 direction) const {  // light.cpp:112-119
        direction = unit_light_direction(direction);
        double u  = (std::atan2(direction.z, direction.x) + rotation_) / (2 * pi);
        u -= std::floor(u);
        const double v = std::atan2(std::hypot(direction.x, direction.z), direction.y) / pi;
        return {u, v};
    }

    dvec3 lookup(dvec2 uv) const {  // light.cpp:121-138
        const auto&  image = texture_->level(0);
        const double x     = uv.x * static_cast<double>(image.width) - 0.5;
        const double y     = uv.y * static_cast<double>(image.height) - 0.5;
        const int    ix    = static_cast<int>(std::floor(x));
        const int    iy    = static_cast<int>(std::floor(y));
        const double tx    = x - std::floor(x);
        const double ty    = y - std::floor(y);
        const auto   texel = [&](int column, int row) {
            const int width = static_cast<int>(image.width), height = static_cast<int>(image.height);
            const auto wrapped = static_cast<std::size_t>((column % width + width) % width);
            return positive(widen(image.at(wrapped, static_cast<std::size_t>(std::clamp(row, 0, height - 1)))));
        };
        return mixd(mixd(texel(ix, iy), texel(ix + 1, iy), tx), mixd(texel(ix, iy + 1), texel(ix + 1, iy + 1), tx),
                    ty);
    }

    dvec3 evaluate(dvec3 direction) const {  // light.cpp:140-143
        const auto uv = coordinates(direction);
        return constant_ + (texture_ ? strength_ * lookup(uv) : dvec3{0, 0, 0});
    }

    double pdf(dvec3 direction) const {  // light.cpp:145-157
        const auto uv = coordinates(direction);
        if (uniform_) {
            return 1 / (4 * pi);
        }
        const auto& grid = texture_->level(grid_level_);
        const auto  x    = std::min(static_cast<std::size_t>(uv.x * static_cast<double>(grid.width)), grid.width - 1);
        const auto  y    = std::min(static_cast<std::size_t>(uv.y * static_cast<double>(grid.height)), grid.height - 1);
        return uniform_fraction / (4 * pi) +
               (1 - uniform_fraction) * pixels_.probability(y * grid.width + x) / solid_angles_[y];
    }

    // light.cpp:159-191: direction, radiance, density.
    void sample(dvec2 u, dvec3& direction, dvec3& radiance, double& density) const {
        check_unit(u);
        if (uniform_ || u.x < uniform_fraction) {
            direction = sample_sphere({uniform_ ? u.x : u.x / uniform_fraction, u.y});
        } else {
            const auto   selected = pixels_.sample((u.x - uniform_fraction) / (1 - uniform_fraction));
            const auto&  grid     = texture_->level(grid_level_);
            const auto   x = selected->index % grid.width, y = selected->index / grid.width;
            const double theta0 = pi * static_cast<double>(y) / static_cast<double>(grid.height);
            const double theta1 = pi * static_cast<double>(y + 1) / static_cast<double>(grid.height);
            const double difference = 2 * std::sin((theta0 + theta1) * 0.5) * std::sin((theta1 - theta0) * 0.5);
            const double v = std::clamp(u.y, dbl_eps * 0.5, std::nextafter(1.0, 0.0));
            double       cosine, sine;
            if (y < grid.height / 2) {
                const double h = 1 - std::cos(theta0) + v * difference;
                cosine         = 1 - h;
                sine           = std::sqrt(std::max(0.0, h * (2 - h)));
            } else {
                const double h = 1 + std::cos(theta1) + (1 - v) * difference;
                cosine         = -1 + h;
                sine           = std::sqrt(std::max(0.0, h * (2 - h)));
            }
            const double phi = 2 * pi * (static_cast<double>(x) + selected->remapped) / static_cast<double>(grid.width) -
                               rotation_;
            direction = {sine * std::cos(phi), cosine, sine * std::sin(phi)};
        }
        radiance = evaluate(direction);
        density  = pdf(direction);
    }

    double luminance_integral() const noexcept { return integral_; }

  private:
    dvec3                          constant_;
    std::shared_ptr<const Texture> texture_;
    double                         strength_ = 1;
    double                         rotation_ = 0;
    double                         integral_ = 0;
    bool                           uniform_  = true;
    std::size_t                    grid_level_ = 0;
    std::vector<double>            solid_angles_;
    DiscreteDistribution           pixels_;
};

enum class LightKind { area, directional, environment };

struct LightSample {
    dvec3       direction;
    dvec3       radiance;
    double      distance    = infinity;
    double      probability = 0;
    bool        discrete    = false;
    LightKind   kind        = LightKind::area;
    std::size_t emitter     = 0;
    dvec3       position, normal, position_error;
};

class LightSampler {  // light.cpp:197-352
  public:
    explicit LightSampler(const Snapshot& scene) : environment_(scene) {
        integral_ = environment_.luminance_integral();
        Bounds3             bounds;
        std::vector<double> weights;
        for (std::size_t index = 0; index < scene.instances.size(); ++index) {
            const auto& instance = scene.instances[index];
            const auto  radiance = widen(instance.material.emission);
            for (std::size_t face = 0; face < instance.mesh->triangles.size(); ++face) {
                std::array<dvec3, 3> vertices;
                for (int corner = 0; corner < 3; ++corner) {
                    const auto world = transform_point(
                        instance.object_to_world,
                        instance.mesh->positions[instance.mesh->triangles[face][corner].position]);
                    if (!finite3(world)) {
                        throw std::invalid_argument("Transformed light scene position is not finite");
                    }
                    bounds.expand(world);
                    vertices[corner] = widen(world);
                }
                if (luminance(radiance) == 0) {
                    continue;
                }
                const auto   c    = cross(vertices[1] - vertices[0], vertices[2] - vertices[0]);
                const double area = length(c) * 0.5;
                if (area == 0) {
                    continue;
                }
                area_choices_[{static_cast<std::uint32_t>(index), static_cast<std::uint32_t>(face)}] =
                    choices_.size();
                choices_.push_back({LightKind::area, areas_.size()});
                const double orientation = determinant3(instance.object_to_world) < 0 ? -1 : 1;
                areas_.push_back({vertices, c * orientation / (2 * area), radiance, area,
                                  instance.material.double_sided});
                weights.push_back((instance.material.double_sided ? 2 : 1) * pi * area *
                                  luminance(radiance));
            }
        }
        const auto   extent = widen(bounds.maximum) - widen(bounds.minimum);
        const double projected_area =
            pi * (bounds.empty() ? 1 : std::max(dot(extent, extent) * 0.25, 1e-12));
        for (const auto& light : scene.directional_lights) {
            const auto radiance = widen(light.color) * static_cast<double>(light.intensity);
            if (luminance(radiance) > 0) {
                choices_.push_back({LightKind::directional, directional_.size()});
                directional_.push_back({-normalize(widen(light.direction)), radiance});
                weights.push_back(projected_area * luminance(radiance));
            }
        }
        if (integral_ > 0) {
            environment_choice_ = choices_.size();
            choices_.push_back({LightKind::environment, 0});
            weights.push_back(projected_area * integral_);
        }
        selection_ = DiscreteDistribution(weights);
    }

    dvec3  environment_evaluate(dvec3 direction) const { return environment_.evaluate(direction); }
    double environment_density(dvec3 direction) const { return environment_.pdf(direction); }

    std::optional<LightSample> sample(dvec3 reference, double light_u, dvec2 surface_u) const {
        if (!finite3(reference)) {
            throw std::invalid_argument("Light reference point must be finite");
        }
        check_unit(surface_u);
        const auto selected = selection_.sample(light_u);
        if (!selected) {
            return std::nullopt;
        }
        const auto& choice = choices_[selected->index];
        if (choice.kind == LightKind::directional) {
            const auto& light = directional_[choice.index];
            LightSample s;
            s.direction   = light.direction;
            s.radiance    = light.radiance;
            s.probability = selected->probability;
            s.discrete    = true;
            s.kind        = choice.kind;
            s.emitter     = selected->index;
            return s;
        }
        if (choice.kind == LightKind::environment) {
            LightSample s;
            double      density = 0;
            environment_.sample(surface_u, s.direction, s.radiance, density);
            s.probability = selected->probability * density;
            s.kind        = choice.kind;
            s.emitter     = selected->index;
            return s;
        }
        const auto& light       = areas_[choice.index];
        const auto  barycentric = sample_triangle(surface_u);
        const auto  point       = barycentric.x * light.vertices[0] + barycentric.y * light.vertices[1] +
                           barycentric.z * light.vertices[2];
        if (!light.double_sided && dot(light.normal, reference - point) <= 0) {
            return std::nullopt;
        }
        const double density = area_density(reference, point, light.normal, light.area);
        if (density == 0) {
            return std::nullopt;
        }
        const auto   direction = point - reference;
        const double distance  = length(direction);
        const auto   error = (dabs(barycentric.x * light.vertices[0]) + dabs(barycentric.y * light.vertices[1]) +
                            dabs(barycentric.z * light.vertices[2])) *
                           (7 * offset_eps);
        LightSample s;
        s.direction      = direction / distance;
        s.radiance       = light.radiance;
        s.distance       = distance;
        s.probability    = selected->probability * density;
        s.kind           = choice.kind;
        s.emitter        = selected->index;
        s.position       = point;
        s.normal         = light.normal;
        s.position_error = error;
        return s;
    }

    double area_pdf(dvec3 reference, const SurfaceHit& hit) const {  // light.cpp:323-334
        const auto choice = area_choices_.find({hit.instance_index, hit.triangle_index});
        if (choice == area_choices_.end()) {
            return 0;
        }
        const auto& light = areas_[choices_[choice->second].index];
        if (!light.double_sided && dot(light.normal, reference - hit.position) <= 0) {
            return 0;
        }
        return selection_.probability(choice->second) *
               area_density(reference, hit.position, light.normal, light.area);
    }

    double environment_pdf(dvec3 direction) const {  // light.cpp:336-340
        return environment_choice_
                   ? selection_.probability(*environment_choice_) * environment_density(direction)
                   : 0;
    }

    std::size_t size() const { return choices_.size(); }
    double      selection_probability(std::size_t i) const { return selection_.probability(i); }
    double      luminance_integral() const { return integral_; }

  private:
    struct Area {
        std::array<dvec3, 3> vertices;
        dvec3                normal, radiance;
        double               area;
        bool                 double_sided;
    };
    struct Directional {
        dvec3 direction, radiance;
    };
    struct Choice {
        LightKind   kind;
        std::size_t index;
    };
    EnvironmentLight                                                environment_;
    double                                                          integral_ = 0;
    std::vector<Area>                                               areas_;
    std::vector<Directional>                                        directional_;
    std::vector<Choice>                                             choices_;
    std::map<std::pair<std::uint32_t, std::uint32_t>, std::size_t> area_choices_;
    std::optional<std::size_t>                                      environment_choice_;
    DiscreteDistribution                                            selection_;
};

// ---- media (src/render/medium.cpp) -------------------------------------------------------

double phase_value(double cosine, double g) {  // medium.cpp:41-46
    const double a           = std::abs(g);
    const double denominator = (1 - a) * (1 - a) + 2 * a * (1 + std::copysign(1.0, g) * cosine);
    return ((1 - g) * (1 + g)) / (4 * pi * denominator * std::sqrt(denominator));
}

double henyey_greenstein(dvec3 wo, dvec3 wi, double g) {  // medium.cpp:89-94
    return phase_value(std::clamp(dot(wo, wi), -1.0, 1.0), g);
}

struct PhaseSample {
    dvec3  direction;
    double probability = 0;
};

PhaseSample sample_henyey_greenstein(dvec3 wo, double g, dvec2 u) {  // medium.cpp:96-117
    double c;
    if (g >= 0) {
        const double denominator = (1 - g) + 2 * g * u.x;
        c = 1 - 2 * (1 - g) * (1 - g) * (1 - u.x) * (1 + g * u.x) / (denominator * denominator);
    } else {
        const double denominator = (1 + g) - 2 * g * (1 - u.x);
        c = -1 + 2 * (1 + g) * (1 + g) * u.x * (1 - g * (1 - u.x)) / (denominator * denominator);
    }
    c                 = std::clamp(c, -1.0, 1.0);
    const double sine = std::sqrt(std::max(0.0, (1 - c) * (1 + c)));
    const double phi  = 2 * pi * u.y;
    const auto   direction =
        normalize(ShadingFrame(-wo).to_world({sine * std::cos(phi), sine * std::sin(phi), c}));
    return {direction, henyey_greenstein(wo, direction, g)};
}

double optical_depth(double extinction, double distance) {  // medium.cpp:48-50
    return extinction == 0 ? 0 : extinction * distance;
}

dvec3 medium_transmittance(const MediumRegion& m, double distance) {  // medium.cpp:119-128
    if (std::isnan(distance) || distance < 0) {
        throw std::invalid_argument("Medium distance must be nonnegative");
    }
    const auto e = m.extinction();
    return {std::exp(-optical_depth(e.x, distance)), std::exp(-optical_depth(e.y, distance)),
            std::exp(-optical_depth(e.z, distance))};
}

dvec3 mixture_weight(const MediumRegion& m, double distance, bool scattered) {  // medium.cpp:53-86
    const auto e = m.extinction();
    dvec3      log_density{-infinity, -infinity, -infinity};
    dvec3      log_numerator{-infinity, -infinity, -infinity};
    for (int c = 0; c < 3; ++c) {
        const double attenuation = -optical_depth(e[c], distance);
        if (!scattered) {
            log_density[c]   = attenuation;
            log_numerator[c] = attenuation;
        } else {
            if (e[c] > 0) {
                log_density[c] = std::log(e[c]) + attenuation;
            }
            if (m.scattering[c] > 0) {
                log_numerator[c] = std::log(m.scattering[c]) + attenuation;
            }
        }
    }
    const double largest = max3(log_density);
    if (!std::isfinite(largest)) {
        throw std::runtime_error("Medium sample has zero mixture probability");
    }
    double sum = 0;
    for (int c = 0; c < 3; ++c) {
        sum += std::exp(log_density[c] - largest);
    }
    const double log_probability = largest + std::log(sum / 3);
    dvec3        result;
    for (int c = 0; c < 3; ++c) {
        result[c] = std::exp(log_numerator[c] - log_probability);
    }
    return result;
}

struct DistanceSample {
    bool   scattered = false;
    double distance  = 0;
    dvec3  weight{1, 1, 1};
};

DistanceSample sample_medium_distance(const MediumRegion& m, double length, double channel_u,
                                      double distance_u) {  // medium.cpp:130-143
    const auto   e       = m.extinction();
    const auto   channel = std::min(static_cast<int>(channel_u * 3), 2);
    const double distance =
        e[channel] == 0 ? infinity : -std::log1p(-distance_u) / e[channel];
    const bool   scattered = distance < length;
    const double actual    = scattered ? distance : length;
    return {scattered, actual, mixture_weight(m, actual, scattered)};
}

struct Segment {
    std::size_t region;
    double      minimum, maximum;
};

struct MediumInteraction {
    dvec3  position;
    double distance   = 0;
    double anisotropy = 0;
};

struct MediumSample {
    dvec3                            weight{1, 1, 1};
    std::optional<MediumInteraction> interaction;
};

class MediumField {  // medium.cpp:145-229
  public:
    explicit MediumField(const std::vector<MediumRegion>& regions) : regions_(regions) {}

    std::vector<Segment> segments(const Ray& ray, RayInterval interval) const {
        interval.validate();
        static_cast<void>(RayQuery(ray));
        std::vector<Segment> result;
        for (std::size_t index = 0; index < regions_.size(); ++index) {
            const auto& region = regions_[index];
            if (!region.enabled) {
                continue;
            }
            double enter = interval.minimum;
            double leave = interval.maximum;
            for (int axis = 0; axis < 3; ++axis) {
                if (ray.direction[axis] == 0) {
                    if (ray.origin[axis] <= region.minimum[axis] ||
                        ray.origin[axis] >= region.maximum[axis]) {
                        leave = enter;
                        break;
                    }
                    continue;
                }
                double near = (region.minimum[axis] - ray.origin[axis]) / ray.direction[axis];
                double far  = (region.maximum[axis] - ray.origin[axis]) / ray.direction[axis];
                if (near > far) {
                    std::swap(near, far);
                }
                enter = std::max(enter, near);
                leave = std::min(leave, far);
            }
            if (leave > enter) {
                result.push_back({index, enter, leave});
            }
        }
        std::sort(result.begin(), result.end(),
                  [](const auto& a, const auto& b) { return a.minimum < b.minimum; });
        return result;
    }

    dvec3 transmittance(const Ray& ray, RayInterval interval) const {
        dvec3 result{1, 1, 1};
        if (regions_.empty()) {
            return result;
        }
        for (const auto& part : segments(ray, interval)) {
            result *= medium_transmittance(regions_[part.region], part.maximum - part.minimum);
        }
        return result;
    }

    MediumSample sample(const Ray& ray, RayInterval interval, Sampler& sampler) const {
        MediumSample result;
        if (regions_.empty()) {
            return result;
        }
        for (const auto& part : segments(ray, interval)) {
            const auto&  medium = regions_[part.region];
            const double length = part.maximum - part.minimum;
            if (medium.scattering.x == 0 && medium.scattering.y == 0 && medium.scattering.z == 0) {
                result.weight *= medium_transmittance(medium, length);
                continue;
            }
            const double channel  = sampler.next_1d();
            const double distance = sampler.next_1d();
            const auto   sampled  = sample_medium_distance(medium, length, channel, distance);
            result.weight *= sampled.weight;
            if (sampled.scattered) {
                const double t     = part.minimum + sampled.distance;
                result.interaction = MediumInteraction{ray.origin + t * ray.direction, t,
                                                       medium.anisotropy};
                break;
            }
        }
        return result;
    }

    bool empty() const { return regions_.empty(); }

  private:
    std::vector<MediumRegion> regions_;
};

// ---- path tracer (src/render/path_tracer.cpp) ----------------------------------------------

struct IntegratorSettings {
    std::uint32_t mode           = MR_SAMPLING_MIS;
    std::uint32_t maximum_depth  = 8;
    bool          russian_roulette = true;
    std::uint32_t roulette_depth = 3;
    void          validate() const {  // path_tracer.cpp:55-64
        require(mode <= MR_SAMPLING_MIS, "Sampling mode must be bsdf, light or mis");
        require(maximum_depth <= 128 && roulette_depth <= 128,
                "Path and roulette depths must not exceed 128");
    }
};

struct RenderSettings {
    std::size_t   width = 256, height = 256;
    std::uint32_t samples_per_pixel = 64;
    std::uint64_t seed              = 1;
    void          validate() const {  // path_tracer.cpp:66-71
        if (width == 0 || height == 0 || width > 16384 || height > 16384 ||
            width * height > 64U * 1024U * 1024U || samples_per_pixel == 0) {
            throw std::invalid_argument("Render dimensions or sample count exceed the image budget");
        }
    }
};

struct PathStatistics {
    TraceStatistics geometry;
    std::uint64_t   paths = 0, shadow_rays = 0, scattering_events = 0, roulette_terminations = 0,
                  medium_scattering_events = 0;
    void add(const PathStatistics& o) {
        geometry.bounds_tests += o.geometry.bounds_tests;
        geometry.triangle_tests += o.geometry.triangle_tests;
        paths += o.paths;
        shadow_rays += o.shadow_rays;
        scattering_events += o.scattering_events;
        roulette_terminations += o.roulette_terminations;
        medium_scattering_events += o.medium_scattering_events;
    }
};

void check_radiance(dvec3 value) {  // path_tracer.cpp:22-26
    if (!finite3(value) || value.x < 0 || value.y < 0 || value.z < 0) {
        throw std::runtime_error("Path contribution is nonfinite or negative");
    }
}

double power_heuristic(double sampled_pdf, double other_pdf) {  // path_tracer.cpp:73-85
    if (!std::isfinite(sampled_pdf) || !std::isfinite(other_pdf) || sampled_pdf < 0 ||
        other_pdf < 0) {
        throw std::invalid_argument("MIS probabilities must be finite and nonnegative");
    }
    const double scale = std::max(sampled_pdf, other_pdf);
    if (scale == 0) {
        return 0;
    }
    const double a = sampled_pdf / scale;
    const double b = other_pdf / scale;
    return a * a / (a * a + b * b);
}

dvec3 offset_origin(dvec3 position, fvec3 geometric_normal, dvec3 position_error,
                    dvec3 direction) {  // path_tracer.cpp:87-105
    auto normal = normalize(widen(geometric_normal));
    if (dot(normal, direction) < 0) {
        normal = -normal;
    }
    const double numeric_floor =
        static_cast<double>(std::numeric_limits<float>::min()) * std::numeric_limits<float>::min();
    const double distance = std::max(dot(dabs(normal), position_error), numeric_floor);
    auto         origin   = position + distance * normal;
    for (int axis = 0; axis < 3; ++axis) {
        if (normal[axis] != 0) {
            origin[axis] = std::nextafter(origin[axis], std::copysign(infinity, normal[axis]));
        }
    }
    return origin;
}

Ray spawn_ray(const SurfaceHit& hit, dvec3 direction) {  // path_tracer.cpp:107-109
    return {offset_origin(hit.position, hit.geometric_normal, hit.position_error, direction),
            normalize(direction)};
}

class PathTracer {
  public:
    PathTracer(std::shared_ptr<const Snapshot> scene, IntegratorSettings settings,
               const mr_bvh_desc* imported = nullptr)
        : scene_(std::move(scene)), bvh_(scene_, imported), lights_(*scene_),
          media_(scene_->media), settings_(settings) {
        settings_.validate();
    }

    // path_tracer.cpp:126-151
    dvec3 shadow_transmittance(Ray ray, const LightSample& light, PathStatistics* statistics) const {
        if (statistics) {
            ++statistics->shadow_rays;
        }
        double limit = infinity;
        if (std::isfinite(light.distance)) {
            const auto target = offset_origin(light.position, narrow(light.normal),
                                              light.position_error, -light.direction);
            const auto difference = target - ray.origin;
            limit                 = length(difference);
            if (limit == 0) {
                return {0, 0, 0};
            }
            ray.direction = difference / limit;
            limit         = std::nextafter(limit, 0.0);
        }
        if (bvh_.occluded(ray, {0, limit}, statistics ? &statistics->geometry : nullptr)) {
            return {0, 0, 0};
        }
        return media_.transmittance(ray, {0, limit});
    }

    // path_tracer.cpp:153-366 (subsurface branch omitted: the material is rejected).
    dvec3 trace(Ray ray, Sampler& sampler, RayInterval primary_interval,
                PathStatistics* statistics) const {
        if (statistics) {
            ++statistics->paths;
        }
        dvec3  result;
        dvec3  beta{1, 1, 1};
        dvec3  previous_reference;
        double previous_pdf   = 0;
        double eta_scale      = 1;
        bool   previous_delta = true;
        for (std::uint32_t depth = 0;; ++depth) {
            const auto interval = depth == 0 ? primary_interval : RayInterval{0, infinity};
            const auto hit =
                bvh_.intersect(ray, interval, statistics ? &statistics->geometry : nullptr);
            const auto medium =
                media_.sample(ray, {interval.minimum, hit ? hit->distance : interval.maximum}, sampler);
            beta *= medium.weight;
            check_radiance(beta);
            if (max3(beta) == 0) {
                break;
            }
            if (medium.interaction) {
                if (depth == settings_.maximum_depth) {
                    break;
                }
                const auto&  vertex          = *medium.interaction;
                const auto   wo              = -ray.direction;
                const double light_u         = sampler.next_1d();
                const auto   light_surface_u = sampler.next_2d();
                const auto   phase_u         = sampler.next_2d();
                const auto   light           = lights_.sample(vertex.position, light_u, light_surface_u);
                if (light && (settings_.mode != MR_SAMPLING_BSDF || light->discrete)) {
                    const double phase = henyey_greenstein(wo, light->direction, vertex.anisotropy);
                    const auto   transmission =
                        shadow_transmittance({vertex.position, light->direction}, *light, statistics);
                    double weight = 1;
                    if (settings_.mode == MR_SAMPLING_MIS && !light->discrete) {
                        weight = power_heuristic(light->probability, phase);
                    }
                    result += beta * transmission * light->radiance *
                              (phase * weight / light->probability);
                }
                const auto phase   = sample_henyey_greenstein(wo, vertex.anisotropy, phase_u);
                previous_reference = vertex.position;
                previous_pdf       = phase.probability;
                previous_delta     = false;
                ray                = {vertex.position, phase.direction};
                if (statistics) {
                    ++statistics->scattering_events;
                    ++statistics->medium_scattering_events;
                }
                const double roulette_u = sampler.next_1d();
                if (settings_.russian_roulette && depth + 1 >= settings_.roulette_depth) {
                    const double survival = std::clamp(max3(beta * eta_scale), 0.05, 0.95);
                    if (roulette_u >= survival) {
                        if (statistics) {
                            ++statistics->roulette_terminations;
                        }
                        break;
                    }
                    beta /= survival;
                }
                continue;
            }
            const auto emission_weight = [&](double light_pdf) {
                if (depth == 0 || previous_delta || settings_.mode == MR_SAMPLING_BSDF) {
                    return 1.0;
                }
                return settings_.mode == MR_SAMPLING_MIS ? power_heuristic(previous_pdf, light_pdf)
                                                         : 0.0;
            };
            if (!hit) {
                result += beta * lights_.environment_evaluate(ray.direction) *
                          emission_weight(lights_.environment_pdf(ray.direction));
                break;
            }
            const auto& instance = scene_->instances[hit->instance_index];
            result += beta * widen(instance.material.emission) *
                      emission_weight(lights_.area_pdf(previous_reference, *hit));
            if (depth == settings_.maximum_depth) {
                break;
            }
            auto normal = widen(instance.material.kind == MR_MATERIAL_DIELECTRIC
                                    ? hit->geometric_normal
                                    : hit->shading_normal);
            const auto wo_world = -ray.direction;
            if (dot(normal, wo_world) < 0) {
                normal = -normal;
            }
            const ShadingFrame frame(normal);
            const auto         wo = frame.to_local(wo_world);
            const fvec3 texture_color = instance.material.base_color_texture
                                            ? instance.material.base_color_texture->sample(
                                                  hit->uv, 0, instance.material.texture_filter)
                                            : fvec3{1, 1, 1};  // path_tracer.cpp:279-282
            const Bsdf         bsdf(instance.material, hit->front_face, false, texture_color);
            const double       light_u     = sampler.next_1d();
            const auto         surface_u   = sampler.next_2d();
            const double       component   = sampler.next_1d();
            const auto         direction_u = sampler.next_2d();
            if (!bsdf.is_delta()) {
                const auto light = lights_.sample(hit->position, light_u, surface_u);
                if (light && (settings_.mode != MR_SAMPLING_BSDF || light->discrete)) {
                    const auto wi = frame.to_local(light->direction);
                    const bool reflection_side =
                        dot(wo_world, widen(hit->geometric_normal)) *
                            dot(light->direction, widen(hit->geometric_normal)) >
                        0;
                    if (wi.z > 0 && reflection_side) {
                        const auto transmission =
                            shadow_transmittance(spawn_ray(*hit, light->direction), *light, statistics);
                        if (max3(transmission) > 0) {
                            double weight = 1;
                            if (settings_.mode == MR_SAMPLING_MIS && !light->discrete) {
                                weight = power_heuristic(light->probability, bsdf.pdf(wo, wi));
                            }
                            result += beta * transmission * bsdf.evaluate(wo, wi) * wi.z *
                                      light->radiance * (weight / light->probability);
                        }
                    }
                }
            }
            const auto sample = bsdf.sample(wo, component, direction_u);
            if (!sample || max3(sample->weight) == 0) {
                break;
            }
            const auto   wi_world = normalize(frame.to_world(sample->direction));
            const double sides    = dot(wo_world, widen(hit->geometric_normal)) *
                                 dot(wi_world, widen(hit->geometric_normal));
            const bool transmission = sample->event == Event::specular_transmission;
            if ((transmission && sides >= 0) || (!transmission && sides <= 0)) {
                break;
            }
            beta *= sample->weight;
            check_radiance(beta);
            previous_reference = hit->position;
            previous_pdf       = sample->probability;
            previous_delta     = sample->discrete;
            eta_scale *= sample->eta * sample->eta;
            if (statistics) {
                ++statistics->scattering_events;
            }
            ray                     = spawn_ray(*hit, wi_world);
            const double roulette_u = sampler.next_1d();
            if (settings_.russian_roulette && depth + 1 >= settings_.roulette_depth) {
                const double survival = std::clamp(max3(beta * eta_scale), 0.05, 0.95);
                if (roulette_u >= survival) {
                    if (statistics) {
                        ++statistics->roulette_terminations;
                    }
                    break;
                }
                beta /= survival;
            }
        }
        check_radiance(result);
        return result;
    }

    // path_tracer.cpp:368-386 (also returns the camera ray and its interval).
    dvec3 sample_pixel(std::size_t x, std::size_t y, std::uint64_t sample_index,
                       const RenderSettings& settings, PathStatistics* statistics,
                       Ray* ray_out = nullptr, RayInterval* interval_out = nullptr) const {
        auto       sampler = Sampler::for_sample(settings.seed, y * settings.width + x, sample_index);
        const auto film    = sampler.next_2d();
        const auto lens    = sampler.next_2d();
        const dvec2 uv{(static_cast<double>(x) + film.x) / static_cast<double>(settings.width),
                       (static_cast<double>(y) + film.y) / static_cast<double>(settings.height)};
        const auto ray = generate_lens_ray(
            uv, static_cast<double>(settings.width) / static_cast<double>(settings.height), lens);
        const auto&  camera  = scene_->camera;
        const auto   forward = normalize(from(camera.target) - from(camera.position));
        const double cosine  = dot(ray.direction, forward);
        const RayInterval interval{camera.near_plane / cosine, camera.far_plane / cosine};
        if (ray_out) {
            *ray_out = ray;
        }
        if (interval_out) {
            *interval_out = interval;
        }
        return trace(ray, sampler, interval, statistics);
    }

    // scene.cpp:171-199
    Ray generate_ray(dvec2 pixel_uv, double aspect) const {
        const auto&  c           = scene_->camera;
        const auto   forward     = normalize(from(c.target) - from(c.position));
        const auto   right       = normalize(cross(forward, from(c.up)));
        const auto   camera_up   = cross(right, forward);
        const double half_height = std::tan(static_cast<double>(c.vertical_fov_degrees) *
                                            (pi / 180.0) * 0.5);
        const auto direction = forward + (2 * pixel_uv.x - 1) * aspect * half_height * right +
                               (1 - 2 * pixel_uv.y) * half_height * camera_up;
        return {from(c.position), normalize(direction)};
    }
    Ray generate_lens_ray(dvec2 pixel_uv, double aspect, dvec2 lens_u) const {
        const auto  pinhole = generate_ray(pixel_uv, aspect);
        const auto& c       = scene_->camera;
        if (c.aperture_radius == 0) {
            return pinhole;
        }
        const auto d         = sample_disk(lens_u);
        const dvec2 disk{d.x * static_cast<double>(c.aperture_radius),
                         d.y * static_cast<double>(c.aperture_radius)};
        const auto forward   = normalize(from(c.target) - from(c.position));
        const auto right     = normalize(cross(forward, from(c.up)));
        const auto camera_up = cross(right, forward);
        const auto focus     = pinhole.origin + pinhole.direction * (static_cast<double>(c.focus_distance) /
                                                                 dot(pinhole.direction, forward));
        const auto origin    = from(c.position) + disk.x * right + disk.y * camera_up;
        return {origin, normalize(focus - origin)};
    }

    const SceneBvh&     bvh() const { return bvh_; }
    const LightSampler& lights() const { return lights_; }
    const MediumField&  media() const { return media_; }
    const Snapshot&     scene() const { return *scene_; }

  private:
    std::shared_ptr<const Snapshot> scene_;
    SceneBvh                        bvh_;
    LightSampler                    lights_;
    MediumField                     media_;
    IntegratorSettings              settings_;
};

// Tile-parallel render with the accumulation order of RenderSession (render_session.cpp:386-459):
// each pixel's samples are summed in sample order in double, so the image is bitwise identical
// to the serial PathTracer::render (path_tracer.cpp:388-405) for any thread count.
void render_rows(const PathTracer& tracer, const RenderSettings& settings, std::size_t row_begin,
                 std::size_t row_end, unsigned threads, float* rgb, PathStatistics* statistics) {
    settings.validate();
    const std::size_t tile       = 16;
    const std::size_t columns    = (settings.width + tile - 1) / tile;
    const std::size_t rows       = (row_end - row_begin + tile - 1) / tile;
    const std::size_t tile_count = columns * rows;
    std::atomic<std::size_t> next_tile{0};
    std::atomic<bool>        failed{false};
    std::string              failure;
    int                      failure_kind = 0;
    std::mutex               failure_mutex;
    std::vector<PathStatistics> local(std::max(1U, threads));
    const auto work = [&](unsigned worker) {
        try {
            while (!failed.load()) {
                const auto t = next_tile.fetch_add(1);
                if (t >= tile_count) {
                    break;
                }
                const auto x0 = (t % columns) * tile;
                const auto y0 = row_begin + (t / columns) * tile;
                const auto w  = std::min(tile, settings.width - x0);
                const auto h  = std::min(tile, row_end - y0);
                for (std::size_t y = y0; y < y0 + h; ++y) {
                    for (std::size_t x = x0; x < x0 + w; ++x) {
                        dvec3 sum;
                        for (std::uint32_t s = 0; s < settings.samples_per_pixel; ++s) {
                            sum += tracer.sample_pixel(x, y, s, settings,
                                                       statistics ? &local[worker] : nullptr);
                        }
                        const auto value = sum / static_cast<double>(settings.samples_per_pixel);
                        if (max3(value) > std::numeric_limits<float>::max()) {
                            throw std::overflow_error("Rendered radiance exceeds the float image range");
                        }
                        float* out = rgb + 3 * ((y - row_begin) * settings.width + x);
                        out[0]     = static_cast<float>(value.x);
                        out[1]     = static_cast<float>(value.y);
                        out[2]     = static_cast<float>(value.z);
                    }
                }
            }
        } catch (const std::overflow_error& e) {
            std::lock_guard lock(failure_mutex);
            failed = true;
            failure = e.what();
            failure_kind = MR_OVERFLOW;
        } catch (const std::invalid_argument& e) {
            std::lock_guard lock(failure_mutex);
            failed = true;
            failure = e.what();
            failure_kind = MR_INVALID_ARGUMENT;
        } catch (const std::exception& e) {
            std::lock_guard lock(failure_mutex);
            failed = true;
            failure = e.what();
            failure_kind = MR_RUNTIME_ERROR;
        }
    };
    std::vector<std::thread> pool;
    for (unsigned i = 1; i < threads; ++i) {
        pool.emplace_back(work, i);
    }
    work(0);
    for (auto& t : pool) {
        t.join();
    }
    if (failed) {
        if (failure_kind == MR_OVERFLOW) {
            throw std::overflow_error(failure);
        }
        if (failure_kind == MR_INVALID_ARGUMENT) {
            throw std::invalid_argument(failure);
        }
        throw std::runtime_error(failure);
    }
    if (statistics) {
        for (const auto& s : local) {
            statistics->add(s);
        }
    }
}

}  // namespace oracle

// ==== C ABI for the tests (ctypes) ==========================================================

namespace {

thread_local std::string last_error;

template <typename F> int guarded(F&& f) {
    try {
        f();
        return MR_OK;
    } catch (const std::invalid_argument& e) {
        last_error = e.what();
        return MR_INVALID_ARGUMENT;
    } catch (const std::out_of_range& e) {
        last_error = e.what();
        return MR_OUT_OF_RANGE;
    } catch (const std::overflow_error& e) {
        last_error = e.what();
        return MR_OVERFLOW;
    } catch (const std::length_error& e) {
        last_error = e.what();
        return MR_LENGTH_ERROR;
    } catch (const std::exception& e) {
        last_error = e.what();
        return MR_RUNTIME_ERROR;
    }
}

struct OracleScene {
    std::shared_ptr<oracle::Snapshot>  snapshot;
    std::unique_ptr<oracle::PathTracer> tracer;
};

oracle::IntegratorSettings to_settings(const mr_integrator_settings* s) {
    oracle::IntegratorSettings r;
    if (s) {
        r.mode             = s->mode;
        r.maximum_depth    = s->maximum_depth;
        r.russian_roulette = s->russian_roulette != 0;
        r.roulette_depth   = s->roulette_depth;
    }
    return r;
}

oracle::RenderSettings to_render(const mr_render_settings* s) {
    oracle::RenderSettings r;
    r.width             = s->width;
    r.height            = s->height;
    r.samples_per_pixel = s->samples_per_pixel;
    r.seed              = s->seed;
    return r;
}

void to_path_stats(const oracle::PathStatistics& s, mr_path_statistics* out) {
    if (!out) {
        return;
    }
    std::memset(out, 0, sizeof(*out));
    out->geometry.bounds_tests   = s.geometry.bounds_tests;
    out->geometry.triangle_tests = s.geometry.triangle_tests;
    out->paths                   = s.paths;
    out->shadow_rays             = s.shadow_rays;
    out->scattering_events       = s.scattering_events;
    out->roulette_terminations   = s.roulette_terminations;
    out->medium_scattering_events = s.medium_scattering_events;
}

// Ray in double for the oracle: explicit double rays, or FP32 rays widened.
struct DRay {
    double origin[3];
    double direction[3];
    double minimum;
    double maximum;
};

}  // namespace

namespace {

// Splits [0, count) into contiguous chunks over the host's threads (one chunk below 65,536
// items); every chunk gets its own statistics, summed after the join.
template <typename F>
void parallel_chunks(size_t count, oracle::TraceStatistics& total, F&& body) {
    const size_t threads = count < 65536 ? 1 : std::max(1U, std::thread::hardware_concurrency());
    std::vector<oracle::TraceStatistics> local(threads);
    std::vector<std::exception_ptr>      errors(threads);
    const auto run = [&](size_t t) {
        try {
            body(count * t / threads, count * (t + 1) / threads, local[t]);
        } catch (...) {
            errors[t] = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < threads; ++t) {
        pool.emplace_back(run, t);
    }
    run(0);
    for (auto& t : pool) {
        t.join();
    }
    for (size_t t = 0; t < threads; ++t) {
        if (errors[t]) {
            std::rethrow_exception(errors[t]);
        }
        total.bounds_tests += local[t].bounds_tests;
        total.triangle_tests += local[t].triangle_tests;
    }
}

}  // namespace

extern "C" {

size_t or_last_error(char* buffer, size_t capacity) {
    if (buffer && capacity) {
        const auto n = std::min(capacity - 1, last_error.size());
        std::memcpy(buffer, last_error.data(), n);
        buffer[n] = 0;
    }
    return last_error.size();
}

// --- sampling primitives ---
void or_pcg_sequence(uint64_t seed, uint64_t sequence, size_t count, uint32_t* out) {
    oracle::Sampler s(seed, sequence);
    for (size_t i = 0; i < count; ++i) {
        out[i] = s.next_u32();
    }
}

void or_stream_1d(uint64_t seed, uint64_t pixel, uint64_t sample, size_t count, double* out) {
    auto s = oracle::Sampler::for_sample(seed, pixel, sample);
    for (size_t i = 0; i < count; ++i) {
        out[i] = s.next_1d();
    }
}

void or_sampler_state(uint64_t seed, uint64_t pixel, uint64_t sample, uint64_t* state_increment) {
    const auto s       = oracle::Sampler::for_sample(seed, pixel, sample);
    state_increment[0] = s.state();
    state_increment[1] = s.increment();
}

int or_warp(int kind, const double* u, size_t count, double* out) {
    return guarded([&] {
        for (size_t i = 0; i < count; ++i) {
            const oracle::dvec2 uu{u[2 * i], u[2 * i + 1]};
            double* o = out + 3 * i;
            if (kind == 0) {
                const auto d = oracle::sample_disk(uu);
                o[0] = d.x, o[1] = d.y, o[2] = 0;
            } else {
                oracle::dvec3 v;
                if (kind == 1) v = oracle::sample_sphere(uu);
                else if (kind == 2) v = oracle::sample_hemisphere(uu);
                else if (kind == 3) v = oracle::sample_cosine_hemisphere(uu);
                else v = oracle::sample_triangle(uu);
                o[0] = v.x, o[1] = v.y, o[2] = v.z;
            }
        }
    });
}

int or_distribution(const double* weights, size_t count, const double* u, size_t samples,
                    double* probabilities, uint64_t* indices, double* masses, double* remapped) {
    return guarded([&] {
        const oracle::DiscreteDistribution d(std::vector<double>(weights, weights + count));
        for (size_t i = 0; i < d.size(); ++i) {
            probabilities[i] = d.probability(i);
        }
        for (size_t i = 0; i < samples; ++i) {
            const auto s = d.sample(u[i]);
            indices[i]   = s ? s->index : UINT64_MAX;
            masses[i]    = s ? s->probability : 0;
            remapped[i]  = s ? s->remapped : 0;
        }
    });
}

int or_fresnel_dielectric(double cosine, double eta_i, double eta_t, double* out) {
    return guarded([&] { *out = oracle::fresnel_dielectric(cosine, eta_i, eta_t); });
}

// Bsdf::sample/evaluate/pdf on one material (result: dir[3], weight[3], probability, discrete,
// event, eta, valid).
int or_bsdf_sample(const mr_material* material, int front_face, int importance, const double* wo,
                   double component, const double* u, double* result) {
    return guarded([&] {
        oracle::Material m;
        m.kind       = material->kind;
        m.base_color = {material->base_color[0], material->base_color[1], material->base_color[2]};
        m.roughness  = material->roughness;
        m.ior        = material->ior;
        const oracle::Bsdf b(m, front_face != 0, importance != 0);
        const auto         s = b.sample({wo[0], wo[1], wo[2]}, component, {u[0], u[1]});
        std::memset(result, 0, sizeof(double) * 11);
        if (s) {
            result[0] = s->direction.x, result[1] = s->direction.y, result[2] = s->direction.z;
            result[3] = s->weight.x, result[4] = s->weight.y, result[5] = s->weight.z;
            result[6] = s->probability;
            result[7] = s->discrete;
            result[8] = static_cast<double>(s->event);
            result[9] = s->eta;
            result[10] = 1;
        }
    });
}

int or_bsdf_eval(const mr_material* material, int front_face, const double* wo, const double* wi,
                 double* value, double* pdf, int* delta) {
    return guarded([&] {
        oracle::Material m;
        m.kind       = material->kind;
        m.base_color = {material->base_color[0], material->base_color[1], material->base_color[2]};
        m.roughness  = material->roughness;
        m.ior        = material->ior;
        const oracle::Bsdf b(m, front_face != 0);
        const auto v = b.evaluate({wo[0], wo[1], wo[2]}, {wi[0], wi[1], wi[2]});
        value[0] = v.x, value[1] = v.y, value[2] = v.z;
        *pdf   = b.pdf({wo[0], wo[1], wo[2]}, {wi[0], wi[1], wi[2]});
        *delta = b.is_delta();
    });
}

int or_power_heuristic(double a, double b, double* out) {
    return guarded([&] { *out = oracle::power_heuristic(a, b); });
}

int or_phase(const double* wo, const double* wi, double g, double* out) {
    return guarded([&] { *out = oracle::henyey_greenstein({wo[0], wo[1], wo[2]}, {wi[0], wi[1], wi[2]}, g); });
}

int or_sample_phase(const double* wo, double g, const double* u, double* out) {
    return guarded([&] {
        const auto s = oracle::sample_henyey_greenstein({wo[0], wo[1], wo[2]}, g, {u[0], u[1]});
        out[0] = s.direction.x, out[1] = s.direction.y, out[2] = s.direction.z, out[3] = s.probability;
    });
}

// sample_medium_distance on one region (absorption[3], scattering[3]).
int or_medium_distance(const double* absorption, const double* scattering, double length,
                       double channel_u, double distance_u, double* out) {
    return guarded([&] {
        oracle::MediumRegion r;
        r.absorption = {absorption[0], absorption[1], absorption[2]};
        r.scattering = {scattering[0], scattering[1], scattering[2]};
        const auto s = oracle::sample_medium_distance(r, length, channel_u, distance_u);
        out[0] = s.scattered, out[1] = s.distance, out[2] = s.weight.x, out[3] = s.weight.y,
        out[4] = s.weight.z;
    });
}

// --- scene ---
int or_scene_create(const mr_scene_desc* desc, const mr_bvh_desc* bvh,
                    const mr_integrator_settings* integrator, void** out) {
    return guarded([&] {
        auto s      = std::make_unique<OracleScene>();
        s->snapshot = oracle::make_snapshot(*desc);
        s->tracer = std::make_unique<oracle::PathTracer>(s->snapshot, to_settings(integrator), bvh);
        *out      = s.release();
    });
}

void or_scene_destroy(void* scene) {
    delete static_cast<OracleScene*>(scene);
}

int or_bvh_counts(void* scene, uint64_t* nodes, uint64_t* primitives, uint64_t* leaves,
                  uint64_t* depth) {
    return guarded([&] {
        const auto& bvh = static_cast<OracleScene*>(scene)->tracer->bvh();
        *nodes          = bvh.nodes().size();
        *primitives     = bvh.primitives().size();
        *leaves         = bvh.statistics().leaves;
        *depth          = bvh.statistics().maximum_depth;
    });
}

int or_bvh_export(void* scene, mr_bvh_node* nodes, uint32_t* order) {
    return guarded([&] {
        const auto& bvh = static_cast<OracleScene*>(scene)->tracer->bvh();
        for (size_t i = 0; i < bvh.nodes().size(); ++i) {
            const auto& n = bvh.nodes()[i];
            for (int a = 0; a < 3; ++a) {
                nodes[i].minimum[a] = n.bounds.minimum[a];
                nodes[i].maximum[a] = n.bounds.maximum[a];
            }
            nodes[i].first = n.first;
            nodes[i].right = n.right;
            nodes[i].count = n.count;
        }
        std::memcpy(order, bvh.order().data(), bvh.order().size() * sizeof(uint32_t));
    });
}

int or_sah_cost(void* scene, double* cost) {
    return guarded([&] { *cost = static_cast<OracleScene*>(scene)->tracer->bvh().sah_cost(); });
}

// World-space primitive vertices (9 floats each) in primitive order.
int or_primitives(void* scene, float* vertices) {
    return guarded([&] {
        const auto& prims = static_cast<OracleScene*>(scene)->tracer->bvh().primitives();
        for (size_t i = 0; i < prims.size(); ++i) {
            for (int c = 0; c < 3; ++c) {
                vertices[9 * i + 3 * c + 0] = prims[i].vertices[c].x;
                vertices[9 * i + 3 * c + 1] = prims[i].vertices[c].y;
                vertices[9 * i + 3 * c + 2] = prims[i].vertices[c].z;
            }
        }
    });
}

// Nearest hit / occlusion for double rays. hits: per ray [hit, distance, instance, triangle,
// primitive, b0, b1, b2, front_face, px, py, pz, ngx, ngy, ngz, nsx, nsy, nsz].
int or_intersect(void* scene, const DRay* rays, size_t count, double* hits, uint64_t* counters) {
    return guarded([&] {
        const auto&             bvh = static_cast<OracleScene*>(scene)->tracer->bvh();
        oracle::TraceStatistics stats;
        parallel_chunks(count, stats, [&](size_t begin, size_t end, oracle::TraceStatistics& st) {
            for (size_t i = begin; i < end; ++i) {
                const auto& r = rays[i];
                const oracle::Ray ray{{r.origin[0], r.origin[1], r.origin[2]},
                                      {r.direction[0], r.direction[1], r.direction[2]}};
                const auto hit = bvh.intersect(ray, {r.minimum, r.maximum}, &st);
                double*    o   = hits + 18 * i;
                std::memset(o, 0, sizeof(double) * 18);
                if (hit) {
                    o[0] = 1, o[1] = hit->distance, o[2] = hit->instance_index,
                    o[3] = hit->triangle_index;
                    o[4] = hit->primitive;
                    o[5] = hit->barycentric.x, o[6] = hit->barycentric.y, o[7] = hit->barycentric.z;
                    o[8] = hit->front_face;
                    o[9] = hit->position.x, o[10] = hit->position.y, o[11] = hit->position.z;
                    o[12] = hit->geometric_normal.x, o[13] = hit->geometric_normal.y,
                    o[14] = hit->geometric_normal.z;
                    o[15] = hit->shading_normal.x, o[16] = hit->shading_normal.y,
                    o[17] = hit->shading_normal.z;
                }
            }
        });
        if (counters) {
            counters[0] += stats.bounds_tests;
            counters[1] += stats.triangle_tests;
        }
    });
}

int or_occluded(void* scene, const DRay* rays, size_t count, uint8_t* out, uint64_t* counters) {
    return guarded([&] {
        const auto&             bvh = static_cast<OracleScene*>(scene)->tracer->bvh();
        oracle::TraceStatistics stats;
        parallel_chunks(count, stats, [&](size_t begin, size_t end, oracle::TraceStatistics& st) {
            for (size_t i = begin; i < end; ++i) {
                const auto&       r = rays[i];
                const oracle::Ray ray{{r.origin[0], r.origin[1], r.origin[2]},
                                      {r.direction[0], r.direction[1], r.direction[2]}};
                out[i] = bvh.occluded(ray, {r.minimum, r.maximum}, &st) ? 1 : 0;
            }
        });
        if (counters) {
            counters[0] += stats.bounds_tests;
            counters[1] += stats.triangle_tests;
        }
    });
}

// PathTracer::trace for explicit rays and stream keys.
int or_trace_paths(void* scene, const DRay* rays, const uint64_t* keys, size_t count,
                   double* radiance, mr_path_statistics* statistics) {
    return guarded([&] {
        const auto&            tracer = *static_cast<OracleScene*>(scene)->tracer;
        oracle::PathStatistics stats;
        for (size_t i = 0; i < count; ++i) {
            const auto& r       = rays[i];
            auto        sampler = oracle::Sampler::for_sample(keys[3 * i], keys[3 * i + 1], keys[3 * i + 2]);
            const auto  value   = tracer.trace(
                {{r.origin[0], r.origin[1], r.origin[2]}, {r.direction[0], r.direction[1], r.direction[2]}},
                sampler, {r.minimum, r.maximum}, &stats);
            radiance[3 * i] = value.x, radiance[3 * i + 1] = value.y, radiance[3 * i + 2] = value.z;
        }
        to_path_stats(stats, statistics);
    });
}

// PathTracer::sample_pixel for (x, y, sample) triples; optionally returns camera rays.
int or_sample_pixels(void* scene, const mr_render_settings* render, const uint32_t* pixels,
                     const uint64_t* samples, size_t count, double* radiance, DRay* rays,
                     mr_path_statistics* statistics) {
    return guarded([&] {
        const auto&            tracer   = *static_cast<OracleScene*>(scene)->tracer;
        const auto             settings = to_render(render);
        oracle::PathStatistics stats;
        settings.validate();
        for (size_t i = 0; i < count; ++i) {
            if (pixels[2 * i] >= settings.width || pixels[2 * i + 1] >= settings.height) {
                throw std::out_of_range("Pixel coordinates are outside the render image");
            }
            oracle::Ray         ray;
            oracle::RayInterval interval;
            const auto value = tracer.sample_pixel(pixels[2 * i], pixels[2 * i + 1], samples[i], settings,
                                                   &stats, &ray, &interval);
            radiance[3 * i] = value.x, radiance[3 * i + 1] = value.y, radiance[3 * i + 2] = value.z;
            if (rays) {
                for (int a = 0; a < 3; ++a) {
                    rays[i].origin[a]    = ray.origin[a];
                    rays[i].direction[a] = ray.direction[a];
                }
                rays[i].minimum = interval.minimum;
                rays[i].maximum = interval.maximum;
            }
        }
        to_path_stats(stats, statistics);
    });
}

// Pinhole camera rays at explicit film coordinates with the clip interval of the primary-ray
// diagnostic (src/app/cli.cpp:60-81: Camera::generate_ray at the pixel centre, interval
// near/cos .. far/cos with cos the ray's cosine to the view direction).
int or_camera_rays(void* scene, const double* uv, size_t count, double aspect, DRay* rays) {
    return guarded([&] {
        const auto& tracer  = *static_cast<OracleScene*>(scene)->tracer;
        const auto& camera  = tracer.scene().camera;
        const auto  forward = oracle::normalize(oracle::from(camera.target) - oracle::from(camera.position));
        for (size_t i = 0; i < count; ++i) {
            const auto   ray    = tracer.generate_ray({uv[2 * i], uv[2 * i + 1]}, aspect);
            const double cosine = oracle::dot(ray.direction, forward);
            for (int a = 0; a < 3; ++a) {
                rays[i].origin[a]    = ray.origin[a];
                rays[i].direction[a] = ray.direction[a];
            }
            rays[i].minimum = camera.near_plane / cosine;
            rays[i].maximum = camera.far_plane / cosine;
        }
    });
}

// Tile-parallel render of rows [row_begin, row_end) with `threads` workers.
int or_render_rows(void* scene, const mr_render_settings* render, uint64_t row_begin,
                   uint64_t row_end, uint32_t threads, float* rgb, mr_path_statistics* statistics) {
    return guarded([&] {
        const auto settings = to_render(render);
        if (row_begin > row_end || row_end > settings.height) {
            throw std::out_of_range("Row range is outside the render image");
        }
        oracle::PathStatistics stats;
        oracle::render_rows(*static_cast<OracleScene*>(scene)->tracer, settings, row_begin, row_end,
                            std::max(1U, threads), rgb, statistics ? &stats : nullptr);
        to_path_stats(stats, statistics);
    });
}

// LightSampler::sample at a reference point. out: [valid, dir3, radiance3, distance,
// probability, discrete, kind, emitter, position3, normal3, error3].
int or_light_sample(void* scene, const double* reference, double light_u, const double* surface_u,
                    double* out) {
    return guarded([&] {
        const auto& lights = static_cast<OracleScene*>(scene)->tracer->lights();
        const auto  s      = lights.sample({reference[0], reference[1], reference[2]}, light_u,
                                           {surface_u[0], surface_u[1]});
        std::memset(out, 0, sizeof(double) * 22);
        if (s) {
            out[0] = 1;
            out[1] = s->direction.x, out[2] = s->direction.y, out[3] = s->direction.z;
            out[4] = s->radiance.x, out[5] = s->radiance.y, out[6] = s->radiance.z;
            out[7] = s->distance, out[8] = s->probability, out[9] = s->discrete;
            out[10] = static_cast<double>(s->kind), out[11] = static_cast<double>(s->emitter);
            out[12] = s->position.x, out[13] = s->position.y, out[14] = s->position.z;
            out[15] = s->normal.x, out[16] = s->normal.y, out[17] = s->normal.z;
            out[18] = s->position_error.x, out[19] = s->position_error.y, out[20] = s->position_error.z;
        }
    });
}

int or_light_table(void* scene, uint64_t* count, double* probabilities) {
    return guarded([&] {
        const auto& lights = static_cast<OracleScene*>(scene)->tracer->lights();
        *count             = lights.size();
        if (probabilities) {
            for (size_t i = 0; i < lights.size(); ++i) {
                probabilities[i] = lights.selection_probability(i);
            }
        }
    });
}

// Shadow test between a point and a light sample as PathTracer::shadow_transmittance builds it:
// origin/direction given in `ray` (spawned by the caller), returns transmittance.
int or_area_pdf_at_hit(void* scene, const double* reference, const DRay* ray, double* out) {
    return guarded([&] {
        const auto& tracer = *static_cast<OracleScene*>(scene)->tracer;
        const oracle::Ray r{{ray->origin[0], ray->origin[1], ray->origin[2]},
                            {ray->direction[0], ray->direction[1], ray->direction[2]}};
        const auto hit = tracer.bvh().intersect(r, {ray->minimum, ray->maximum}, nullptr);
        *out = hit ? tracer.lights().area_pdf({reference[0], reference[1], reference[2]}, *hit) : -1;
    });
}

int or_display_image(const float* linear, uint64_t width, uint64_t height, double exposure,
                     float* display) {  // path_tracer.cpp:407-424
    return guarded([&] {
        if (!std::isfinite(exposure) || std::abs(exposure) > 64) {
            throw std::invalid_argument("Display exposure must be finite and in [-64,64]");
        }
        const double scale = std::exp2(exposure);
        for (uint64_t i = 0; i < width * height * 3; ++i) {
            const double v = linear[i];
            if (!std::isfinite(v)) {
                throw std::invalid_argument("Display input contains nonfinite radiance");
            }
            const double p = std::max(v, 0.0) * scale;
            display[i]     = static_cast<float>(p / (1.0 + p));
        }
    });
}

}  // extern "C"
