// minirender_b200.hpp — header-only C++ adapter over the C ABI (minirender_b200.h).
//
// Re-exposes the two classes a MiniRender caller links against, with the reference's names,
// argument meaning and exception types:
//   minirender_b200::PathTracer    ~ minirender::PathTracer    (include/minirender/render/path_tracer.hpp:79-128)
//   minirender_b200::RenderSession ~ minirender::RenderSession (include/minirender/render/render_session.hpp:82-115)
// A status from the library is rethrown as the exception the reference would throw
// (std::invalid_argument, std::out_of_range, std::overflow_error, std::logic_error,
// std::length_error, std::runtime_error). Images are row-major linear RGB floats, origin top-left.
// render_batch and RenderServer (many renders at once) have no reference counterpart.
#pragma once

#include <chrono>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "minirender_b200.h"

namespace minirender_b200 {

inline std::string last_error() {
    char buffer[1024];
    mr_last_error(buffer, sizeof(buffer));
    return buffer;
}

inline void check(mr_status status) {
    switch (status) {
    case MR_OK:
        return;
    case MR_INVALID_ARGUMENT:
        throw std::invalid_argument(last_error());
    case MR_OUT_OF_RANGE:
        throw std::out_of_range(last_error());
    case MR_OVERFLOW:
        throw std::overflow_error(last_error());
    case MR_LOGIC_ERROR:
        throw std::logic_error(last_error());
    case MR_LENGTH_ERROR:
        throw std::length_error(last_error());
    default:
        throw std::runtime_error(last_error());
    }
}

// RGB float image (include/minirender/core/image.hpp), width*height*3 floats.
struct Image {
    std::size_t        width  = 0;
    std::size_t        height = 0;
    std::vector<float> rgb;
};

// An uploaded snapshot: device geometry, BVH, lights and media.
class Scene {
  public:
    explicit Scene(const mr_scene_desc& desc, const mr_bvh_desc* bvh = nullptr) {
        mr_scene* s = nullptr;
        check(mr_scene_create(&desc, bvh, &s));
        handle_.reset(s);
    }
    mr_scene* get() const noexcept { return handle_.get(); }
    mr_bvh_statistics statistics() const {
        mr_bvh_statistics s{};
        check(mr_scene_bvh_statistics(handle_.get(), &s));
        return s;
    }

  private:
    struct Deleter {
        void operator()(mr_scene* s) const noexcept { mr_scene_destroy(s); }
    };
    std::unique_ptr<mr_scene, Deleter> handle_;
};

class PathTracer {
  public:
    PathTracer(std::shared_ptr<const Scene> scene, mr_integrator_settings settings = {MR_SAMPLING_MIS, 8, 1, 3})
        : scene_(std::move(scene)), settings_(settings) {
        if (!scene_) {
            throw std::invalid_argument("PathTracer requires a scene");
        }
    }
    // PathTracer::render (src/render/path_tracer.cpp:388-405).
    Image render(const mr_render_settings& settings, mr_path_statistics* statistics = nullptr) const {
        Image image{static_cast<std::size_t>(settings.width), static_cast<std::size_t>(settings.height), {}};
        image.rgb.resize(3 * image.width * image.height);
        check(mr_render(scene_->get(), &settings_, &settings, image.rgb.data(), statistics));
        return image;
    }
    // PathTracer::trace for a batch of rays and (seed, pixel, sample) sampler keys.
    std::vector<float> trace(const std::vector<mr_ray>& rays, const std::vector<uint64_t>& keys,
                             mr_path_statistics* statistics = nullptr) const {
        if (keys.size() != 3 * rays.size()) {
            throw std::invalid_argument("trace needs three sampler keys per ray");
        }
        std::vector<float> radiance(3 * rays.size());
        check(mr_trace_paths(scene_->get(), &settings_, rays.data(), keys.data(), rays.size(),
                             radiance.data(), statistics));
        return radiance;
    }
    // Rows [row_begin, row_end) of render(): bit for bit the full image's rows (row bands of
    // one frame rendered by several ranks).
    Image render_rows(const mr_render_settings& settings, uint64_t row_begin, uint64_t row_end,
                      mr_path_statistics* statistics = nullptr) const {
        Image image{static_cast<std::size_t>(settings.width),
                    static_cast<std::size_t>(row_end > row_begin ? row_end - row_begin : 0), {}};
        image.rgb.resize(3 * image.width * image.height);
        check(mr_render_rows(scene_->get(), &settings_, &settings, row_begin, row_end,
                             image.rgb.empty() ? nullptr : image.rgb.data(), statistics));
        return image;
    }
    const Scene& scene() const noexcept { return *scene_; }
    const mr_integrator_settings& settings() const noexcept { return settings_; }

  private:
    std::shared_ptr<const Scene> scene_;
    mr_integrator_settings       settings_;
};

// Many renders at once (mr_render_batch; no reference counterpart): each image is bitwise the
// one PathTracer::render gives alone. Throws the first failing job's exception.
struct BatchJob {
    std::shared_ptr<const Scene> scene;
    mr_render_settings           render;
    mr_integrator_settings       integrator{MR_SAMPLING_MIS, 8, 1, 3};
};

inline std::vector<Image> render_batch(const std::vector<BatchJob>& jobs,
                                       const mr_batch_settings* settings = nullptr,
                                       mr_batch_statistics* statistics = nullptr) {
    std::vector<Image>        images(jobs.size());
    std::vector<mr_batch_job> records(jobs.size());
    for (std::size_t i = 0; i < jobs.size(); ++i) {
        if (!jobs[i].scene) {
            throw std::invalid_argument("Batch job requires a scene");
        }
        images[i].width  = static_cast<std::size_t>(jobs[i].render.width);
        images[i].height = static_cast<std::size_t>(jobs[i].render.height);
        images[i].rgb.resize(3 * images[i].width * images[i].height);
        records[i] = {jobs[i].scene->get(), jobs[i].integrator, jobs[i].render, images[i].rgb.data(), MR_OK};
    }
    mr_batch_settings defaults{0, 0, 0, 0, 1, 0};
    check(mr_render_batch(records.data(), records.size(), settings ? settings : &defaults, statistics));
    return images;
}

// Request loop over the GPU (mr_server_*; no reference counterpart): jobs are admitted by HBM
// budget, rendered together, and paused, resumed or cancelled per job. The scenes of submitted
// jobs are kept alive here until the server is destroyed.
class RenderServer {
  public:
    explicit RenderServer(const mr_server_settings* settings = nullptr) {
        mr_server_settings defaults{};
        defaults.batch.use_graphs = 1;
        mr_server* s = nullptr;
        check(mr_server_create(settings ? settings : &defaults, &s));
        handle_.reset(s);
    }
    uint64_t submit(std::shared_ptr<const Scene> scene, const mr_render_settings& render,
                    const mr_integrator_settings& integrator = {MR_SAMPLING_MIS, 8, 1, 3}) {
        if (!scene) {
            throw std::invalid_argument("Render job requires a scene");
        }
        uint64_t job = 0;
        check(mr_server_submit(handle_.get(), scene->get(), &render, &integrator, &job));
        sizes_.emplace_back(job, std::make_pair(render.width, render.height));
        scenes_.push_back(std::move(scene));
        return job;
    }
    bool pause(uint64_t job) {
        int accepted = 0;
        check(mr_server_pause(handle_.get(), job, &accepted));
        return accepted != 0;
    }
    bool resume(uint64_t job) {
        int accepted = 0;
        check(mr_server_resume(handle_.get(), job, &accepted));
        return accepted != 0;
    }
    void cancel(uint64_t job) { check(mr_server_cancel(handle_.get(), job)); }
    bool wait_for(uint64_t job, std::chrono::milliseconds timeout) {
        int done = 0;
        check(mr_server_wait(handle_.get(), job, static_cast<uint32_t>(timeout.count()), &done));
        return done != 0;
    }
    mr_job_info info(uint64_t job) {
        mr_job_info i{};
        check(mr_server_job_info(handle_.get(), job, &i));
        return i;
    }
    Image result(uint64_t job) {
        for (const auto& [id, size] : sizes_) {
            if (id == job) {
                Image image{static_cast<std::size_t>(size.first), static_cast<std::size_t>(size.second), {}};
                image.rgb.resize(3 * image.width * image.height);
                check(mr_server_result(handle_.get(), job, image.rgb.data(), image.rgb.size()));
                return image;
            }
        }
        throw std::out_of_range("Unknown job");
    }
    void release(uint64_t job) { check(mr_server_release(handle_.get(), job)); }

  private:
    struct Deleter {
        void operator()(mr_server* s) const noexcept { mr_server_destroy(s); }
    };
    std::unique_ptr<mr_server, Deleter>                             handle_;
    std::vector<std::pair<uint64_t, std::pair<uint64_t, uint64_t>>> sizes_;
    std::vector<std::shared_ptr<const Scene>>                       scenes_;
};

class RenderSession {
  public:
    RenderSession() {
        mr_session* s = nullptr;
        check(mr_session_create(&s));
        handle_.reset(s);
    }
    RenderSession(const RenderSession&)            = delete;
    RenderSession& operator=(const RenderSession&) = delete;

    void start(std::shared_ptr<const Scene> scene, mr_render_settings render,
               mr_integrator_settings integrator = {MR_SAMPLING_MIS, 8, 1, 3},
               mr_session_settings session = {0, 16, 4}) {
        if (!scene) {
            throw std::invalid_argument("Render session requires a scene snapshot");
        }
        check(mr_session_start(handle_.get(), scene->get(), &render, &integrator, &session));
        scene_  = std::move(scene);  // kept alive for the job, as the reference keeps its snapshot
        render_ = render;
    }
    bool pause() {
        int accepted = 0;
        check(mr_session_pause(handle_.get(), &accepted));
        return accepted != 0;
    }
    bool resume() {
        int accepted = 0;
        check(mr_session_resume(handle_.get(), &accepted));
        return accepted != 0;
    }
    void cancel() { check(mr_session_cancel(handle_.get())); }
    void wait() { check(mr_session_wait(handle_.get())); }
    bool wait_for(std::chrono::milliseconds timeout) const {
        int done = 0;
        check(mr_session_wait_for(handle_.get(), static_cast<uint32_t>(timeout.count()), &done));
        return done != 0;
    }
    mr_render_progress progress() const {
        mr_render_progress p{};
        check(mr_session_progress(handle_.get(), &p));
        return p;
    }
    // Shared immutable result; empty unless the job completed.
    std::shared_ptr<const Image> result() const {
        uint64_t w = 0, h = 0;
        if (mr_session_result(handle_.get(), nullptr, 0, &w, &h) != MR_OK) {
            return nullptr;
        }
        auto image = std::make_shared<Image>();
        image->width  = static_cast<std::size_t>(w);
        image->height = static_cast<std::size_t>(h);
        image->rgb.resize(3 * w * h);
        check(mr_session_result(handle_.get(), image->rgb.data(), image->rgb.size(), nullptr, nullptr));
        return image;
    }

  private:
    struct Deleter {
        void operator()(mr_session* s) const noexcept { mr_session_destroy(s); }
    };
    std::unique_ptr<mr_session, Deleter> handle_;
    std::shared_ptr<const Scene>         scene_;
    mr_render_settings                   render_{};
};

}  // namespace minirender_b200
