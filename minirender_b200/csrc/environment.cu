// environment.cu — scene textures on the device and the environment map's importance
// distribution (host side of textures.cuh).
//
// Textures are validated as Texture's constructor validates them (src/core/texture.cpp:54-74)
// and uploaded as level 0 only (the path tracer samples at lod 0). The environment map's
// distribution follows EnvironmentLight's constructor (src/render/light.cpp:61-110) in double on
// the host: the grid is the first mip level of at most 1024x512 texels (area-weighted
// downsampling, texture.cpp:25-50), each texel weighted by its luminance (negative channels
// clamped to 0) times its solid angle; its luminance integral, taken on level 0, adds to the
// constant environment's for light selection. The distribution is uploaded as a row marginal
// CDF and per-row conditional CDFs in FP32.
#include <algorithm>
#include <cmath>
#include <vector>

#include "errors.hpp"
#include "scene.cuh"

namespace mr {

namespace {

struct HostImage {
    size_t             width = 0, height = 0;
    std::vector<float> rgb;  // 3 per texel
    const float* at(size_t x, size_t y) const { return rgb.data() + 3 * (y * width + x); }
};

HostImage downsample(const HostImage& source) {  // texture.cpp:25-50
    HostImage target;
    target.width  = std::max<size_t>(1, source.width / 2);
    target.height = std::max<size_t>(1, source.height / 2);
    target.rgb.resize(3 * target.width * target.height);
    for (size_t y = 0; y < target.height; ++y) {
        for (size_t x = 0; x < target.width; ++x) {
            const double left   = double(x) * double(source.width) / double(target.width);
            const double right  = double(x + 1) * double(source.width) / double(target.width);
            const double top    = double(y) * double(source.height) / double(target.height);
            const double bottom = double(y + 1) * double(source.height) / double(target.height);
            double       sum[3] = {0, 0, 0}, weight_sum = 0;
            for (size_t sy = static_cast<size_t>(top); sy < static_cast<size_t>(std::ceil(bottom)); ++sy) {
                for (size_t sx = static_cast<size_t>(left); sx < static_cast<size_t>(std::ceil(right)); ++sx) {
                    const double weight = (std::min(right, double(sx + 1)) - std::max(left, double(sx))) *
                                          (std::min(bottom, double(sy + 1)) - std::max(top, double(sy)));
                    const float* p = source.at(sx, sy);
                    for (int c = 0; c < 3; ++c) {
                        sum[c] += double(p[c]) * weight;
                    }
                    weight_sum += weight;
                }
            }
            float* out = target.rgb.data() + 3 * (y * target.width + x);
            for (int c = 0; c < 3; ++c) {
                out[c] = static_cast<float>(sum[c] / weight_sum);
            }
        }
    }
    return target;
}

double positive_luminance(const float* p) {  // luminance(positive(c)), light.cpp:21-27
    return (std::max(double(p[0]), 0.0) * 0.2126 + std::max(double(p[1]), 0.0) * 0.7152) +
           std::max(double(p[2]), 0.0) * 0.0722;
}

double row_solid_angle(size_t y, size_t width, size_t height) {  // light.cpp:81-84
    const double pi     = 3.14159265358979323846;
    const double theta0 = pi * double(y) / double(height);
    const double theta1 = pi * double(y + 1) / double(height);
    return (2 * pi / double(width)) * 2 * std::sin((theta0 + theta1) * 0.5) * std::sin((theta1 - theta0) * 0.5);
}

}  // namespace

void upload_textures(Scene& scene, const mr_scene_desc& desc, cudaStream_t stream) {
    scene.d.textures    = nullptr;
    scene.d.texels      = nullptr;
    scene.d.env_texture = -1;
    scene.d.env_uniform = 1;
    if (desc.texture_count == 0) {
        return;
    }
    require(desc.textures != nullptr, "Texture table is missing");
    std::vector<DeviceTexture> records(desc.texture_count);
    uint64_t                   total = 0;
    for (uint32_t i = 0; i < desc.texture_count; ++i) {
        const mr_texture& t = desc.textures[i];
        require(t.rgb != nullptr && t.width > 0 && t.height > 0, "Texture data is missing");
        require(t.width <= 16384 && t.height <= 16384 && uint64_t(t.width) * t.height <= 64ull * 1024 * 1024,
                "Texture exceeds the 64-megapixel budget");
        for (uint64_t k = 0; k < 3ull * t.width * t.height; ++k) {
            require(std::isfinite(t.rgb[k]), "Texture contains nonfinite samples");
        }
        records[i] = {t.width, t.height, total};
        total += uint64_t(t.width) * t.height;
    }
    std::vector<float4> texels(total);
    for (uint32_t i = 0; i < desc.texture_count; ++i) {
        const mr_texture& t = desc.textures[i];
        for (uint64_t k = 0; k < uint64_t(t.width) * t.height; ++k) {
            texels[records[i].offset + k] = make_float4(t.rgb[3 * k], t.rgb[3 * k + 1], t.rgb[3 * k + 2], 0.0f);
        }
    }
    scene.texels.allocate(texels.size());
    scene.texture_table.allocate(records.size());
    MR_CUDA(cudaMemcpyAsync(scene.texels.ptr, texels.data(), texels.size() * sizeof(float4), cudaMemcpyHostToDevice,
                            stream));
    MR_CUDA(cudaMemcpyAsync(scene.texture_table.ptr, records.data(), records.size() * sizeof(DeviceTexture),
                            cudaMemcpyHostToDevice, stream));
    MR_CUDA(cudaStreamSynchronize(stream));  // the host vectors go away with this function
    scene.d.texels   = scene.texels.ptr;
    scene.d.textures = scene.texture_table.ptr;
}

double prepare_environment(Scene& scene, const mr_scene_desc& desc, cudaStream_t stream) {
    const double pi = 3.14159265358979323846;
    scene.d.env_texture  = -1;
    scene.d.env_uniform  = 1;
    scene.d.env_strength = desc.environment_strength;
    scene.d.env_rotation = static_cast<float>(std::remainder(double(desc.environment_rotation_degrees), 360.0) * pi / 180);
    if (desc.environment_texture == 0) {
        return 0;
    }
    require(desc.environment_texture <= desc.texture_count, "Environment references missing texture");
    require(std::isfinite(desc.environment_strength) && std::isfinite(desc.environment_rotation_degrees),
            "Environment strength and rotation must be finite");
    if (desc.environment_strength == 0) {
        return 0;  // the map contributes nothing; the constant stays
    }
    scene.d.env_texture = static_cast<int>(desc.environment_texture - 1);
    const mr_texture& src = desc.textures[desc.environment_texture - 1];
    HostImage         full;
    full.width  = src.width;
    full.height = src.height;
    full.rgb.assign(src.rgb, src.rgb + 3ull * src.width * src.height);
    // The luminance integral over level 0 (light.cpp:96-108).
    double full_integral = 0;
    for (size_t y = 0; y < full.height; ++y) {
        const double angle = row_solid_angle(y, full.width, full.height);
        for (size_t x = 0; x < full.width; ++x) {
            full_integral += positive_luminance(full.at(x, y)) * angle;
        }
    }
    // The grid level and its distribution (light.cpp:71-92).
    HostImage grid = full;
    while (grid.width > 1024 || grid.height > 512) {
        grid = downsample(grid);
    }
    const size_t        w = grid.width, h = grid.height;
    std::vector<double> weights(w * h);
    std::vector<float>  solid(h);
    double              map_integral = 0;
    for (size_t y = 0; y < h; ++y) {
        const double angle = row_solid_angle(y, w, h);
        solid[y]           = static_cast<float>(angle);
        for (size_t x = 0; x < w; ++x) {
            weights[y * w + x] = positive_luminance(grid.at(x, y)) * angle;
            map_integral += weights[y * w + x];
        }
    }
    if (map_integral > 0) {
        // DiscreteDistribution over all grid texels (sampling.cpp:109-127) in double, kept as its
        // row marginal and per-row conditional CDFs.
        double maximum = 0;
        for (double v : weights) {
            maximum = std::max(maximum, v);
        }
        std::vector<double> cdf(w * h + 1, 0.0);
        for (size_t k = 0; k < w * h; ++k) {
            cdf[k + 1] = cdf[k] + weights[k] / maximum;
        }
        const double total = cdf.back();
        for (auto& v : cdf) {
            v /= total;
        }
        std::vector<float> row_cdf(h + 1), col_cdf((w + 1) * h);
        for (size_t y = 0; y <= h; ++y) {
            row_cdf[y] = static_cast<float>(cdf[y * w]);
        }
        row_cdf[h] = 1.0f;
        for (size_t y = 0; y < h; ++y) {
            const double start = cdf[y * w], mass = cdf[(y + 1) * w] - cdf[y * w];
            for (size_t x = 0; x <= w; ++x) {
                col_cdf[y * (w + 1) + x] = mass > 0 ? static_cast<float>((cdf[y * w + x] - start) / mass)
                                                    : static_cast<float>(double(x) / double(w));
            }
            col_cdf[y * (w + 1) + w] = 1.0f;
        }
        scene.env_row_cdf.allocate(row_cdf.size());
        scene.env_col_cdf.allocate(col_cdf.size());
        scene.env_solid_angle.allocate(solid.size());
        MR_CUDA(cudaMemcpyAsync(scene.env_row_cdf.ptr, row_cdf.data(), row_cdf.size() * sizeof(float),
                                cudaMemcpyHostToDevice, stream));
        MR_CUDA(cudaMemcpyAsync(scene.env_col_cdf.ptr, col_cdf.data(), col_cdf.size() * sizeof(float),
                                cudaMemcpyHostToDevice, stream));
        MR_CUDA(cudaMemcpyAsync(scene.env_solid_angle.ptr, solid.data(), solid.size() * sizeof(float),
                                cudaMemcpyHostToDevice, stream));
        MR_CUDA(cudaStreamSynchronize(stream));
        scene.d.env_uniform     = 0;
        scene.d.env_w           = static_cast<uint32_t>(w);
        scene.d.env_h           = static_cast<uint32_t>(h);
        scene.d.env_row_cdf     = scene.env_row_cdf.ptr;
        scene.d.env_col_cdf     = scene.env_col_cdf.ptr;
        scene.d.env_solid_angle = scene.env_solid_angle.ptr;
    }
    return double(desc.environment_strength) * full_integral;
}

}  // namespace mr
