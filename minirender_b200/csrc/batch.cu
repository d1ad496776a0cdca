// batch.cu — many renders on one GPU: the render server (continuous batching) and the batch
// call built on it.
//
// Every admitted job keeps a device accumulator (sum and compensation per pixel) and a device
// image. The controller thread packs pieces of the admitted jobs into waves: a piece is a pixel
// rectangle x sample range of one job (whole frames of several samples while they fit, else row
// bands of one sample), and a wave holds up to `wave_paths` paths from up to kMaxSegments pieces.
// A wave's descriptor (scene, settings and buffers per piece) is copied to the device and the
// wave runs as one launch of a CUDA graph captured per path depth: init, trace + shade per
// bounce, resolve. Each job's samples are issued in increasing order and a job never has two
// pieces in one wave, so every pixel accumulates its samples in sample order exactly as a
// single-job render does: a job's image does not depend on what it was batched with.
//
// Waves run on `concurrent_waves` lanes, each a stream with its own path state, so while one
// wave's bounce kernel waits on its slowest rays the next wave's kernels use the idle SMs. The
// resolves of all lanes form one chain (each waits for the previous wave's resolve), so a
// job's pixels still receive their samples in order. Two waves per lane are enqueued ahead of
// the device, so the host packs and uploads the next waves while the current ones run. Job
// buffers are allocated and freed on an admin stream that the lanes synchronise with by events.
// A finished job's image is copied to host memory by a second thread on its own stream, after
// which its device buffers return to the server's memory pool and the budget they held admits
// the next queued jobs.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "errors.hpp"
#include "validation.hpp"
#include "wavefront.cuh"

struct mr_scene {
    std::unique_ptr<mr::Scene> impl;
};

namespace mr {

void set_last_error(const std::string& message);

namespace {

using Clock = std::chrono::steady_clock;

constexpr uint32_t kAheadPerLane = 2;  // waves enqueued ahead of the device per lane
constexpr uint32_t kMaxLanes     = 4;
constexpr uint32_t kMaxDepth     = 128;
constexpr size_t   kBytesPerPixel = 2 * sizeof(float4) + 3 * sizeof(float);

struct Cursor {
    uint32_t sample = 0;  // first sample not yet issued
    uint32_t row    = 0;  // row band progress inside that sample (band mode)
};

struct Job {
    uint64_t           id = 0;
    const Scene*       scene = nullptr;
    IntegratorParams   p{};
    mr_render_settings render{};
    uint32_t           width = 0, height = 0, spp = 0;
    size_t             pixels = 0;
    uint64_t           total_samples = 0;
    uint32_t           state = MR_JOB_QUEUED;
    bool               paused = false;
    bool               finishing = false;  // last wave retired, image being copied out
    bool               released  = false;  // forgotten by the caller; erased once no wave holds it
    uint32_t           inflight  = 0;      // enqueued waves carrying a piece of this job
    Cursor             issued, done;
    uint64_t           issued_samples = 0, done_samples = 0;
    int                slot = -1;
    float4*            accumulator = nullptr;
    float*             rgb = nullptr;
    size_t             device_bytes = 0;
    float*             output = nullptr;  // caller's image (batch call); else `result`
    bool               copy_back = true;  // false: the image is not needed on the host
    std::vector<float> result;
    double             submitted = 0, admitted = 0, finished = 0;
    mr_status          status = MR_OK;
    std::string        error;
};

bool terminal(uint32_t state) {
    return state == MR_JOB_COMPLETED || state == MR_JOB_CANCELLED || state == MR_JOB_FAILED;
}

// Makes the server's device current for a caller's thread and restores the caller's afterwards.
struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&previous) != cudaSuccess || previous != device) {
            MR_CUDA(cudaSetDevice(device));
        } else {
            previous = -1;
        }
    }
    ~DeviceGuard() {
        if (previous >= 0) {
            cudaSetDevice(previous);
        }
    }
};

struct Piece {
    Job*     job;
    Cursor   after;
    uint64_t paths;
    bool     last;
};

struct WaveRecord {
    uint32_t           stage = 0;
    cudaEvent_t        start = nullptr, done = nullptr;
    std::vector<Piece> pieces;
};

// A stream that runs waves, with its own path state, descriptor buffer and captured graphs.
struct Lane {
    cudaStream_t                                         stream = nullptr;
    std::shared_ptr<Workspace>                           ws;
    WaveDesc*                                            d_wave = nullptr;
    cudaEvent_t                                          mark   = nullptr;
    std::map<std::pair<uint32_t, int>, cudaGraphExec_t> graphs;  // by depth, media | two levels << 1 | ray sort << 2
};

// Mean of the samples accumulated so far (preview of a running job): pixels in rows < row have
// sample + 1 samples, the others `sample`.
__global__ void preview_kernel(const float4* accumulator, uint32_t width, size_t pixels,
                               uint32_t sample, uint32_t row, float* out) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= pixels) {
        return;
    }
    const uint32_t n = sample + (i / width < row ? 1u : 0u);
    float r = 0, g = 0, b = 0;
    if (n > 0) {
        const float4 s = accumulator[2 * i];
        const float4 c = accumulator[2 * i + 1];
        r = (s.x + c.x) / static_cast<float>(n);
        g = (s.y + c.y) / static_cast<float>(n);
        b = (s.z + c.z) / static_cast<float>(n);
    }
    out[3 * i]     = r;
    out[3 * i + 1] = g;
    out[3 * i + 2] = b;
}

}  // namespace

class Server {
  public:
    explicit Server(const mr_server_settings& settings) : settings_(settings) {
        MR_CUDA(cudaGetDevice(&device_));
        MR_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
        if (settings_.max_jobs == 0) {
            settings_.max_jobs = 1024;
        }
        require(settings_.max_jobs <= 65536, "A server admits at most 65536 jobs at once");
        require(settings_.policy <= MR_SCHEDULE_ARRIVAL, "Unknown scheduling policy");
        mr_batch_settings& b = settings_.batch;
        if (b.wave_paths == 0) {
            b.wave_paths = size_t(1) << 22;
        }
        require(b.wave_paths >= 1024 && b.wave_paths <= (size_t(1) << 26),
                "Paths per wave must lie in [1024, 2^26]");
        int trace_max = 0, shade_max = 0;
        Engine::batch_occupancy(trace_max, shade_max);
        shape_.trace_blocks = sms_ * static_cast<int>(b.trace_blocks_per_sm == 0
                                                          ? trace_max
                                                          : std::min<uint32_t>(b.trace_blocks_per_sm, trace_max));
        shape_.shade_blocks = sms_ * static_cast<int>(b.shade_blocks_per_sm == 0
                                                          ? shade_max
                                                          : std::min<uint32_t>(b.shade_blocks_per_sm, shade_max));
        if (b.concurrent_waves == 0) {
            b.concurrent_waves = 2;
        }
        require(b.concurrent_waves <= kMaxLanes, "At most 4 concurrent waves");
        if (settings_.hbm_budget_bytes == 0) {
            size_t free_bytes = 0, total_bytes = 0;
            MR_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
            settings_.hbm_budget_bytes = free_bytes / 2;
        }
        MR_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        MR_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
        MR_CUDA(cudaEventCreateWithFlags(&admin_ready_, cudaEventDisableTiming));
        MR_CUDA(cudaEventCreateWithFlags(&resolve_chain_, cudaEventDisableTiming));
        cudaMemPoolProps props{};
        props.allocType     = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id   = device_;
        MR_CUDA(cudaMemPoolCreate(&pool_, &props));
        uint64_t keep = UINT64_MAX;
        MR_CUDA(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
        lanes_.resize(b.concurrent_waves);
        for (Lane& lane : lanes_) {
            MR_CUDA(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking));
            MR_CUDA(cudaEventCreateWithFlags(&lane.mark, cudaEventDisableTiming));
            lane.ws = acquire_workspace(b.wave_paths, kMaxDepth + 1, 0);
            MR_CUDA(cudaMalloc(&lane.d_wave, sizeof(WaveDesc)));
            MR_CUDA(cudaMemsetAsync(lane.ws->queues.stats, 0, kStatCount * sizeof(unsigned long long),
                                    lane.stream));
            MR_CUDA(cudaStreamSynchronize(lane.stream));
        }
        stages_ = kAheadPerLane * b.concurrent_waves + 1;
        MR_CUDA(cudaMalloc(&d_errors_, settings_.max_jobs * sizeof(unsigned)));
        MR_CUDA(cudaMemset(d_errors_, 0, settings_.max_jobs * sizeof(unsigned)));
        stage_.assign(stages_, nullptr);
        h_errors_.assign(stages_, nullptr);
        for (uint32_t k = 0; k < stages_; ++k) {
            MR_CUDA(cudaMallocHost(&stage_[k], sizeof(WaveDesc)));
            MR_CUDA(cudaMallocHost(&h_errors_[k], settings_.max_jobs * sizeof(unsigned)));
        }
        for (uint32_t s = settings_.max_jobs; s > 0; --s) {
            free_slots_.push_back(static_cast<int>(s - 1));
        }
        epoch_      = Clock::now();
        controller_ = std::thread([this] { run_controller(); });
        finisher_   = std::thread([this] { run_finisher(); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            for (auto& [id, job] : jobs_) {
                if (!terminal(job->state) && !job->finishing) {
                    cancel_locked(*job);
                }
            }
            stop_ = true;
        }
        work_.notify_all();
        finish_cv_.notify_all();
        controller_.join();
        finisher_.join();
        DeviceGuard guard(device_);
        for (Lane& lane : lanes_) {
            cudaStreamSynchronize(lane.stream);
        }
        cudaStreamSynchronize(stream_);
        cudaStreamSynchronize(copy_stream_);
        for (auto& [id, job] : jobs_) {
            free_buffers(*job, stream_);
        }
        cudaStreamSynchronize(stream_);
        for (Lane& lane : lanes_) {
            for (auto& [key, exec] : lane.graphs) {
                cudaGraphExecDestroy(exec);
            }
            cudaFree(lane.d_wave);
            cudaEventDestroy(lane.mark);
            cudaStreamDestroy(lane.stream);
            release_workspace(std::move(lane.ws));
        }
        for (auto& rec : records_) {
            cudaEventDestroy(rec.start);
            cudaEventDestroy(rec.done);
        }
        for (uint32_t k = 0; k < stages_; ++k) {
            cudaFreeHost(stage_[k]);
            cudaFreeHost(h_errors_[k]);
        }
        cudaFree(d_errors_);
        cudaMemPoolDestroy(pool_);
        cudaEventDestroy(admin_ready_);
        cudaEventDestroy(resolve_chain_);
        cudaStreamDestroy(stream_);
        cudaStreamDestroy(copy_stream_);
    }

    uint64_t submit(const Scene* scene, const mr_render_settings* render,
                    const mr_integrator_settings* integrator, float* output, bool copy_back = true) {
        require(scene != nullptr, "Scene handle is null");
        const IntegratorParams p = integrator_params(integrator);
        validate_render(render);
        auto job           = std::make_unique<Job>();
        job->scene         = scene;
        job->p             = p;
        job->render        = *render;
        job->width         = static_cast<uint32_t>(render->width);
        job->height        = static_cast<uint32_t>(render->height);
        job->spp           = render->samples_per_pixel;
        job->pixels        = static_cast<size_t>(job->width) * job->height;
        job->total_samples = job->pixels * job->spp;
        job->device_bytes  = job->pixels * kBytesPerPixel;
        job->output        = output;
        job->copy_back     = copy_back;
        if (job->width > settings_.batch.wave_paths) {
            fail(MR_INVALID_ARGUMENT, "An image row does not fit in one wave");
        }
        if (job->device_bytes > settings_.hbm_budget_bytes) {
            fail(MR_OUT_OF_MEMORY, "The job's buffers exceed the server's HBM budget");
        }
        std::lock_guard<std::mutex> lock(mutex_);
        require(!stop_, "The server is shutting down");
        job->id        = ++last_id_;
        job->submitted = now();
        Job* raw       = job.get();
        jobs_.emplace(raw->id, std::move(job));
        queued_.push_back(raw);
        ++stats_.submitted;
        work_.notify_all();
        return raw->id;
    }

    bool pause(uint64_t id) {
        std::lock_guard<std::mutex> lock(mutex_);
        Job& j = find(id);
        if (terminal(j.state) || j.finishing || j.paused) {
            return false;
        }
        j.paused = true;
        if (j.state == MR_JOB_RUNNING) {
            j.state = MR_JOB_PAUSED;
        }
        changed_.notify_all();
        return true;
    }

    bool resume(uint64_t id) {
        std::lock_guard<std::mutex> lock(mutex_);
        Job& j = find(id);
        if (!j.paused || terminal(j.state)) {
            return false;
        }
        j.paused = false;
        if (j.state == MR_JOB_PAUSED) {
            j.state = MR_JOB_RUNNING;
        }
        changed_.notify_all();
        work_.notify_all();
        return true;
    }

    void cancel(uint64_t id) {
        std::lock_guard<std::mutex> lock(mutex_);
        Job& j = find(id);
        if (!terminal(j.state) && !j.finishing) {
            cancel_locked(j);
        }
    }

    bool wait(uint64_t id, uint32_t milliseconds) {
        std::unique_lock<std::mutex> lock(mutex_);
        Job& j = find(id);
        return changed_.wait_for(lock, std::chrono::milliseconds(milliseconds),
                                 [&] { return terminal(j.state); });
    }

    void wait_all() {
        std::unique_lock<std::mutex> lock(mutex_);
        changed_.wait(lock, [&] {
            for (auto& [id, job] : jobs_) {
                if (!terminal(job->state)) {
                    return false;
                }
            }
            return true;
        });
    }

    mr_job_info info(uint64_t id) {
        std::lock_guard<std::mutex> lock(mutex_);
        const Job&  j = find(id);
        mr_job_info out{};
        out.state             = j.state;
        out.status            = j.status;
        out.total_samples     = j.total_samples;
        out.completed_samples = j.done_samples;
        out.submitted_seconds = j.submitted;
        out.admitted_seconds  = j.admitted;
        out.finished_seconds  = j.finished;
        std::snprintf(out.error, sizeof(out.error), "%s", j.error.c_str());
        return out;
    }

    void result(uint64_t id, float* rgb, size_t capacity) {
        std::lock_guard<std::mutex> lock(mutex_);
        const Job& j = find(id);
        if (j.state != MR_JOB_COMPLETED) {
            fail(MR_OUT_OF_RANGE, "The job has not completed");
        }
        require(rgb != nullptr, "Output image is null");
        require(capacity >= 3 * j.pixels, "Output image is too small");
        if (!j.output && j.result.empty()) {
            fail(MR_OUT_OF_RANGE, "The job's image was not kept");
        }
        const float* src = j.output ? j.output : j.result.data();
        std::memcpy(rgb, src, 3 * j.pixels * sizeof(float));
    }

    uint64_t preview(uint64_t id, float* rgb, size_t capacity) {
        std::unique_lock<std::mutex> lock(mutex_);
        Job& j = find(id);
        require(rgb != nullptr, "Output image is null");
        require(capacity >= 3 * j.pixels, "Output image is too small");
        if (j.state == MR_JOB_COMPLETED && (j.output || !j.result.empty())) {
            std::memcpy(rgb, j.output ? j.output : j.result.data(), 3 * j.pixels * sizeof(float));
            return j.spp;
        }
        if (!j.accumulator || j.finishing || terminal(j.state)) {
            std::memset(rgb, 0, 3 * j.pixels * sizeof(float));
            return 0;
        }
        // Enqueued behind every issued wave, so the accumulator holds exactly the issued samples.
        DeviceGuard guard(device_);
        admin_after_lanes();
        float* d = nullptr;
        MR_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d), 3 * j.pixels * sizeof(float), pool_,
                                        stream_));
        preview_kernel<<<static_cast<unsigned>((j.pixels + 255) / 256), 256, 0, stream_>>>(
            j.accumulator, j.width, j.pixels, j.issued.sample, j.issued.row, d);
        MR_CUDA(cudaGetLastError());
        cudaEvent_t ready = nullptr;
        MR_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        MR_CUDA(cudaEventRecord(ready, stream_));
        const uint64_t samples = j.issued.sample;
        const size_t   bytes   = 3 * j.pixels * sizeof(float);
        lock.unlock();
        cudaStream_t s = nullptr;
        MR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        MR_CUDA(cudaStreamWaitEvent(s, ready, 0));
        MR_CUDA(cudaMemcpyAsync(rgb, d, bytes, cudaMemcpyDeviceToHost, s));
        MR_CUDA(cudaFreeAsync(d, s));
        MR_CUDA(cudaStreamSynchronize(s));
        cudaStreamDestroy(s);
        cudaEventDestroy(ready);
        return samples;
    }

    // A released job disappears from queries at once; its record is erased when no enqueued
    // wave refers to it any more (a cancelled or failed job can still have waves in flight).
    void release(uint64_t id) {
        std::lock_guard<std::mutex> lock(mutex_);
        Job& j = find(id);
        if (!terminal(j.state)) {
            fail(MR_LOGIC_ERROR, "The job is still active");
        }
        j.released = true;
        active_.erase(std::remove(active_.begin(), active_.end(), &j), active_.end());
        queued_.erase(std::remove(queued_.begin(), queued_.end(), &j), queued_.end());
        if (j.inflight == 0) {
            jobs_.erase(id);
        }
    }

    mr_server_statistics statistics() {
        std::lock_guard<std::mutex> lock(mutex_);
        mr_server_statistics s = stats_;
        s.resident_bytes       = resident_bytes_;
        s.elapsed_seconds      = now();
        return s;
    }

    // Records `e` on the admin stream behind everything enqueued on the lanes so far (device
    // timestamps around a batch).
    void record_after_lanes(cudaEvent_t e) {
        std::lock_guard<std::mutex> lock(mutex_);
        DeviceGuard                 guard(device_);
        admin_after_lanes();
        MR_CUDA(cudaEventRecord(e, stream_));
    }

    // Path statistics summed over every wave so far (waits for the waves in flight).
    mr_path_statistics path_statistics() {
        cudaEvent_t e = nullptr;
        {
            std::lock_guard<std::mutex> lock(mutex_);
            DeviceGuard                 guard(device_);
            admin_after_lanes();
            MR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            MR_CUDA(cudaEventRecord(e, stream_));
        }
        MR_CUDA(cudaEventSynchronize(e));
        cudaEventDestroy(e);
        unsigned long long v[kStatCount] = {};
        for (Lane& lane : lanes_) {
            unsigned long long w[kStatCount];
            MR_CUDA(cudaMemcpy(w, lane.ws->queues.stats, sizeof(w), cudaMemcpyDeviceToHost));
            for (int k = 0; k < kStatCount; ++k) {
                v[k] += w[k];
            }
        }
        mr_path_statistics out{};
        out.paths                    = v[kStatPaths];
        out.shadow_rays              = v[kStatShadowRays];
        out.scattering_events        = v[kStatScattering];
        out.roulette_terminations    = v[kStatRoulette];
        out.medium_scattering_events = v[kStatMedium];
        out.geometry.bounds_tests    = v[kStatExtendBounds] + v[kStatShadowBounds];
        out.geometry.triangle_tests  = v[kStatExtendTriangles] + v[kStatShadowTriangles];
        return out;
    }

  private:
    double now() const { return std::chrono::duration<double>(Clock::now() - epoch_).count(); }

    Job& find(uint64_t id) {
        auto it = jobs_.find(id);
        if (it == jobs_.end() || it->second->released) {
            fail(MR_OUT_OF_RANGE, "Unknown job");
        }
        return *it->second;
    }

    // Makes the admin stream wait for everything enqueued on the lanes so far.
    void admin_after_lanes() {
        for (Lane& lane : lanes_) {
            MR_CUDA(cudaEventRecord(lane.mark, lane.stream));
            MR_CUDA(cudaStreamWaitEvent(stream_, lane.mark, 0));
        }
    }

    void free_buffers(Job& j, cudaStream_t stream) {
        if (j.accumulator) {
            cudaFreeAsync(j.accumulator, stream);
            cudaFreeAsync(j.rgb, stream);
            j.accumulator = nullptr;
            j.rgb         = nullptr;
            resident_bytes_ -= j.device_bytes;
        }
        if (j.slot >= 0) {
            free_slots_.push_back(j.slot);
            j.slot = -1;
        }
    }

    // Stream-ordered frees run after every wave already enqueued that carries the job.
    void cancel_locked(Job& j) {
        queued_.erase(std::remove(queued_.begin(), queued_.end(), &j), queued_.end());
        DeviceGuard guard(device_);
        if (j.accumulator) {
            admin_after_lanes();
        }
        free_buffers(j, stream_);
        j.state    = MR_JOB_CANCELLED;
        j.status   = MR_CANCELLED;
        j.error    = "Render cancelled";
        j.finished = now();
        ++stats_.cancelled;
        changed_.notify_all();
        work_.notify_all();
    }

    void fail_locked(Job& j, mr_status status, const std::string& message) {
        queued_.erase(std::remove(queued_.begin(), queued_.end(), &j), queued_.end());
        if (j.accumulator) {
            admin_after_lanes();
        }
        free_buffers(j, stream_);
        j.state    = MR_JOB_FAILED;
        j.status   = status;
        j.error    = message;
        j.finished = now();
        ++stats_.failed;
        changed_.notify_all();
        work_.notify_all();
    }

    // Admission in submission order while the budget and the job slots allow.
    void admit_locked() {
        while (!queued_.empty() && !free_slots_.empty()) {
            Job& j = *queued_.front();
            if (resident_bytes_ + j.device_bytes > settings_.hbm_budget_bytes) {
                break;
            }
            queued_.pop_front();
            void* acc = nullptr;
            void* rgb = nullptr;
            if (cudaMallocFromPoolAsync(&acc, j.pixels * 2 * sizeof(float4), pool_, stream_) != cudaSuccess ||
                cudaMallocFromPoolAsync(&rgb, j.pixels * 3 * sizeof(float), pool_, stream_) != cudaSuccess) {
                cudaGetLastError();
                if (acc) {
                    cudaFreeAsync(acc, stream_);
                }
                fail_locked(j, MR_OUT_OF_MEMORY, "Device allocation of the job's buffers failed");
                continue;
            }
            j.accumulator = static_cast<float4*>(acc);
            j.rgb         = static_cast<float*>(rgb);
            j.slot        = free_slots_.back();
            free_slots_.pop_back();
            MR_CUDA(cudaMemsetAsync(d_errors_ + j.slot, 0, sizeof(unsigned), stream_));
            resident_bytes_ += j.device_bytes;
            j.admitted = now();
            j.state    = j.paused ? MR_JOB_PAUSED : MR_JOB_RUNNING;
            active_.push_back(&j);
            ++stats_.admitted;
            changed_.notify_all();
        }
    }

    static bool runnable(const Job& j) {
        return j.state == MR_JOB_RUNNING && !j.paused && j.issued.sample < j.spp;
    }

    // The next piece of a job that fits in `space` paths: whole frames of several samples when
    // a frame fits and no row band of the current sample is pending, else one sample of a row
    // band.
    static bool next_piece(const Job& j, uint64_t space, WaveSegment& g, Cursor& after, uint64_t& paths) {
        const Cursor c = j.issued;
        if (c.row == 0 && j.pixels <= space) {
            const uint32_t ns = static_cast<uint32_t>(std::min<uint64_t>(j.spp - c.sample, space / j.pixels));
            g.x0 = 0; g.y0 = 0; g.w = j.width; g.h = j.height; g.s0 = c.sample; g.ns = ns;
            after = {c.sample + ns, 0};
            paths = j.pixels * ns;
            return true;
        }
        const uint32_t rows = static_cast<uint32_t>(std::min<uint64_t>(j.height - c.row, space / j.width));
        if (rows == 0) {
            return false;
        }
        g.x0 = 0; g.y0 = c.row; g.w = j.width; g.h = rows; g.s0 = c.sample; g.ns = 1;
        after = c.row + rows == j.height ? Cursor{c.sample + 1, 0} : Cursor{c.sample, c.row + rows};
        paths = static_cast<uint64_t>(j.width) * rows;
        return true;
    }

    cudaGraphExec_t graph_for(Lane& lane, uint32_t depth, bool media, bool two, bool ray_sort) {
        const auto key = std::make_pair(depth, (media ? 1 : 0) | (two ? 2 : 0) | (ray_sort ? 4 : 0));
        auto it = lane.graphs.find(key);
        if (it != lane.graphs.end()) {
            return it->second;
        }
        cudaGraph_t graph = nullptr;
        MR_CUDA(cudaStreamBeginCapture(lane.stream, cudaStreamCaptureModeThreadLocal));
        try {
            Engine::enqueue_batch_paths(lane.d_wave, depth, media, two, ray_sort, shape_, *lane.ws,
                                        lane.stream);
        } catch (...) {
            cudaStreamEndCapture(lane.stream, &graph);
            if (graph) {
                cudaGraphDestroy(graph);
            }
            throw;
        }
        MR_CUDA(cudaStreamEndCapture(lane.stream, &graph));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e  = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        MR_CUDA(e);
        lane.graphs.emplace(key, exec);
        return exec;
    }

    // Packs the runnable jobs into one wave and enqueues it. Returns false when nothing ran.
    bool launch_wave_locked() {
        std::vector<Job*> order;
        for (Job* j : active_) {
            if (runnable(*j)) {
                order.push_back(j);
            }
        }
        if (order.empty()) {
            return false;
        }
        if (settings_.policy == MR_SCHEDULE_SHORTEST_FIRST) {
            std::stable_sort(order.begin(), order.end(), [](const Job* a, const Job* b) {
                return a->total_samples - a->issued_samples < b->total_samples - b->issued_samples;
            });
        }
        const uint32_t stage = static_cast<uint32_t>(wave_counter_ % stages_);
        Lane&          lane  = lanes_[wave_counter_ % lanes_.size()];
        WaveDesc&      h     = *stage_[stage];
        WaveRecord     rec;
        rec.stage            = stage;
        uint64_t space       = settings_.batch.wave_paths;
        uint32_t count = 0, pixels = 0, depth = 0, slots = 0;
        bool     media = false, two = false;
        for (Job* j : order) {
            if (rec.pieces.size() == kMaxSegments || space < 32) {
                break;
            }
            WaveSegment& g = h.seg[rec.pieces.size()];
            Cursor       after;
            uint64_t     paths = 0;
            if (!next_piece(*j, space, g, after, paths)) {
                continue;
            }
            g.scene       = j->scene->d;
            g.p           = j->p;
            g.width       = j->width;
            g.height      = j->height;
            g.spp         = j->spp;
            g.seed        = j->render.seed;
            g.first_path  = count;
            g.accumulator = j->accumulator;
            g.rgb         = j->rgb;
            g.error       = d_errors_ + j->slot;
            h.first_path[rec.pieces.size()]  = count;
            h.first_pixel[rec.pieces.size()] = pixels;
            count += static_cast<uint32_t>(paths);
            pixels += g.w * g.h;
            space -= paths;
            depth = std::max(depth, j->p.maximum_depth);
            media = media || j->scene->d.medium_count > 0;
            two   = two || j->scene->d.two_level != 0;
            slots = std::max(slots, j->scene->d.slot_count);
            j->issued = after;
            j->issued_samples += paths;
            rec.pieces.push_back({j, after, paths, after.sample >= j->spp});
            ++j->inflight;
        }
        if (rec.pieces.empty()) {
            return false;
        }
        const uint32_t n = static_cast<uint32_t>(rec.pieces.size());
        h.count          = count;
        h.segments       = n;
        h.pixels         = pixels;
        h.sort_threshold = settings_.batch.sort_threshold;
        h.first_path[n]  = count;
        h.first_pixel[n] = pixels;
        const size_t bytes = offsetof(WaveDesc, seg) + n * sizeof(WaveSegment);
        if (records_.size() < stages_) {
            WaveRecord fresh;
            MR_CUDA(cudaEventCreate(&fresh.start));
            MR_CUDA(cudaEventCreate(&fresh.done));
            records_.push_back(fresh);
        }
        WaveRecord& slot = records_[stage];
        rec.start        = slot.start;
        rec.done         = slot.done;
        // Buffers of newly admitted jobs (admin stream) before the wave; the descriptor buffer of
        // this lane is free once the lane's previous wave ran (stream order).
        MR_CUDA(cudaEventRecord(admin_ready_, stream_));
        MR_CUDA(cudaStreamWaitEvent(lane.stream, admin_ready_, 0));
        MR_CUDA(cudaMemcpyAsync(lane.d_wave, &h, bytes, cudaMemcpyHostToDevice, lane.stream));
        MR_CUDA(cudaEventRecord(rec.start, lane.stream));
        // Large waves of scenes whose traversal is not trivial sort each bounce's extension rays
        // by where they start and their direction.
        const bool ray_sort = count >= kRaySortMinPaths && slots >= kRaySortMinSlots;
        if (settings_.batch.use_graphs) {
            MR_CUDA(cudaGraphLaunch(graph_for(lane, depth, media, two, ray_sort), lane.stream));
            ++stats_.graph_launches;
        } else {
            Engine::enqueue_batch_paths(lane.d_wave, depth, media, two, ray_sort, shape_, *lane.ws,
                                        lane.stream);
        }
        // Resolves run in wave order across lanes: per pixel, samples accumulate in order.
        MR_CUDA(cudaStreamWaitEvent(lane.stream, resolve_chain_, 0));
        Engine::enqueue_batch_resolve(lane.d_wave, *lane.ws, lane.stream);
        MR_CUDA(cudaEventRecord(resolve_chain_, lane.stream));
        MR_CUDA(cudaMemcpyAsync(h_errors_[stage], d_errors_, settings_.max_jobs * sizeof(unsigned),
                                cudaMemcpyDeviceToHost, lane.stream));
        MR_CUDA(cudaEventRecord(rec.done, lane.stream));
        const uint64_t launches = Engine::batch_wave_launches(depth, ray_sort);
        note_launches(launches);
        stats_.kernel_launches += launches;
        stats_.segments += n;
        ++stats_.waves;
        ++wave_counter_;
        inflight_.push_back(std::move(rec));
        return true;
    }

    // Books a finished wave: per-job progress, errors, and jobs whose last samples it carried.
    void retire_locked(WaveRecord& rec) {
        float ms = 0;
        cudaEventElapsedTime(&ms, rec.start, rec.done);
        stats_.busy_seconds += ms * 1e-3;
        const unsigned* errors = h_errors_[rec.stage];
        for (const Piece& piece : rec.pieces) {
            Job& j = *piece.job;
            stats_.samples += piece.paths;
            if (--j.inflight == 0 && j.released) {
                jobs_.erase(j.id);
                continue;
            }
            if (terminal(j.state)) {
                continue;
            }
            j.done = piece.after;
            j.done_samples += piece.paths;
            const unsigned e = errors[j.slot];
            if (e) {
                std::string     message;
                const mr_status status = error_status(e, message);
                fail_locked(j, status == MR_OK ? MR_RUNTIME_ERROR : status, message);
                continue;
            }
            if (piece.last) {
                active_.erase(std::remove(active_.begin(), active_.end(), &j), active_.end());
                j.finishing = true;
                finish_queue_.push_back(&j);
                finish_cv_.notify_one();
            }
        }
        changed_.notify_all();
    }

    void run_controller() {
        cudaSetDevice(device_);
        std::unique_lock<std::mutex> lock(mutex_);
        while (true) {
            try {
                while (!inflight_.empty() && cudaEventQuery(inflight_.front().done) == cudaSuccess) {
                    retire_locked(inflight_.front());
                    inflight_.pop_front();
                }
                cudaGetLastError();
                if (stop_ && inflight_.empty()) {
                    break;
                }
                if (!stop_) {
                    admit_locked();
                    active_.erase(std::remove_if(active_.begin(), active_.end(),
                                                 [](const Job* j) { return terminal(j->state); }),
                                  active_.end());
                    if (inflight_.size() < kAheadPerLane * lanes_.size() && launch_wave_locked()) {
                        continue;
                    }
                }
                if (!inflight_.empty()) {
                    cudaEvent_t e = inflight_.front().done;
                    lock.unlock();
                    cudaEventSynchronize(e);
                    lock.lock();
                    continue;
                }
                work_.wait(lock);
            } catch (const Error& e) {
                // A device failure ends every job that has not finished.
                for (auto& [id, job] : jobs_) {
                    if (!terminal(job->state) && !job->finishing) {
                        fail_locked(*job, e.status, e.what());
                    }
                }
                for (WaveRecord& rec : inflight_) {
                    for (const Piece& piece : rec.pieces) {
                        if (--piece.job->inflight == 0 && piece.job->released) {
                            jobs_.erase(piece.job->id);
                        }
                    }
                }
                inflight_.clear();
                if (stop_) {
                    break;
                }
            }
        }
    }

    // Copies finished images to host memory and returns their device buffers.
    void run_finisher() {
        cudaSetDevice(device_);
        std::unique_lock<std::mutex> lock(mutex_);
        while (true) {
            finish_cv_.wait(lock, [&] { return stop_ || !finish_queue_.empty(); });
            if (finish_queue_.empty()) {
                if (stop_ && inflight_.empty()) {
                    break;
                }
                if (stop_) {
                    lock.unlock();
                    std::this_thread::sleep_for(std::chrono::milliseconds(1));
                    lock.lock();
                }
                continue;
            }
            Job& j = *finish_queue_.front();
            finish_queue_.pop_front();
            float*       dst   = j.output;
            const size_t bytes = 3 * j.pixels * sizeof(float);
            if (!dst && j.copy_back) {
                j.result.resize(3 * j.pixels);
                dst = j.result.data();
            }
            const float* src = j.rgb;
            lock.unlock();
            cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
            if (dst) {
                e1 = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, copy_stream_);
                e2 = cudaStreamSynchronize(copy_stream_);
            }
            lock.lock();
            free_buffers(j, copy_stream_);
            j.finishing = false;
            if (e1 != cudaSuccess || e2 != cudaSuccess) {
                j.state  = MR_JOB_FAILED;
                j.status = MR_CUDA_ERROR;
                j.error  = std::string("Image copy failed: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2);
                ++stats_.failed;
            } else {
                j.state = MR_JOB_COMPLETED;
                ++stats_.completed;
            }
            j.finished = now();
            changed_.notify_all();
            work_.notify_all();
        }
    }

    mr_server_settings                         settings_;
    int                                        device_ = 0, sms_ = 0;
    BatchShape                                 shape_;
    cudaStream_t                               stream_ = nullptr, copy_stream_ = nullptr;  // admin, copy-out
    cudaEvent_t                                admin_ready_ = nullptr, resolve_chain_ = nullptr;
    cudaMemPool_t                              pool_   = nullptr;
    std::vector<Lane>                          lanes_;
    uint32_t                                   stages_ = 0;  // pinned descriptor buffers (> waves ahead)
    unsigned*                                  d_errors_ = nullptr;
    std::vector<WaveDesc*>                     stage_;
    std::vector<unsigned*>                     h_errors_;
    std::vector<WaveRecord>                    records_;
    std::mutex                                 mutex_;
    std::condition_variable                    work_, changed_, finish_cv_;
    std::map<uint64_t, std::unique_ptr<Job>>   jobs_;
    std::deque<Job*>                           queued_;
    std::vector<Job*>                          active_;
    std::deque<Job*>                           finish_queue_;
    std::deque<WaveRecord>                     inflight_;
    std::vector<int>                           free_slots_;
    size_t                                     resident_bytes_ = 0;
    uint64_t                                   last_id_ = 0, wave_counter_ = 0;
    bool                                       stop_ = false;
    mr_server_statistics                       stats_{};
    Clock::time_point                          epoch_;
    std::thread                                controller_, finisher_;
};

namespace {

template <typename F> mr_status guarded(F&& f) {
    try {
        f();
        return MR_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("Host allocation failed");
        return MR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return MR_RUNTIME_ERROR;
    }
}

const Scene* scene_ptr(const mr_scene* s) {
    require(s != nullptr && s->impl != nullptr, "Scene handle is null");
    return s->impl.get();
}

// One server per device is kept between batch calls, so repeated calls with the same wave shape
// reuse its lanes' path state and captured graphs instead of rebuilding them. A call takes it
// only when no other call holds it (a concurrent call gets a private server) and a call with a
// different shape replaces it. The cache lives until the process exits.
struct CachedServer {
    int                     device = -1;
    mr_batch_settings       key{};
    std::unique_ptr<Server> server;
    bool                    busy = false;
};

std::mutex&                 server_cache_mutex() {
    static std::mutex* m = new std::mutex;
    return *m;
}
std::vector<CachedServer>&  server_cache() {
    static auto* cache = new std::vector<CachedServer>;  // never destroyed: see above
    return *cache;
}

bool same_shape(const mr_batch_settings& a, const mr_batch_settings& b) {
    return a.wave_paths == b.wave_paths && a.trace_blocks_per_sm == b.trace_blocks_per_sm &&
           a.shade_blocks_per_sm == b.shade_blocks_per_sm && a.sort_threshold == b.sort_threshold &&
           a.use_graphs == b.use_graphs && a.concurrent_waves == b.concurrent_waves;
}

// The cached server of the current device for `shape`, marked busy, or null when another call
// holds it.
Server* take_cached_server(const mr_server_settings& ss, size_t& slot) {
    int device = 0;
    MR_CUDA(cudaGetDevice(&device));
    std::lock_guard<std::mutex> lock(server_cache_mutex());
    auto& cache = server_cache();
    for (size_t i = 0; i < cache.size(); ++i) {
        CachedServer& c = cache[i];
        if (c.device != device) {
            continue;
        }
        if (c.busy) {
            return nullptr;
        }
        if (!same_shape(c.key, ss.batch)) {
            c.server.reset();
            c.server = std::make_unique<Server>(ss);
            c.key    = ss.batch;
        }
        c.busy = true;
        slot   = i;
        return c.server.get();
    }
    CachedServer c;
    c.device = device;
    c.key    = ss.batch;
    c.server = std::make_unique<Server>(ss);
    c.busy   = true;
    cache.push_back(std::move(c));
    slot = cache.size() - 1;
    return cache.back().server.get();
}

void return_cached_server(size_t slot) {
    std::lock_guard<std::mutex> lock(server_cache_mutex());
    server_cache()[slot].busy = false;
}

// Renders a job list on the device's cached server (or a private one); fills per-job statuses.
mr_status run_batch(mr_batch_job* jobs, size_t count, const mr_batch_settings* settings,
                    mr_batch_statistics* statistics, bool copy_images) {
    require(jobs != nullptr || count == 0, "Job list is null");
    mr_server_settings ss{};
    ss.policy = MR_SCHEDULE_ARRIVAL;
    if (settings) {
        ss.batch = *settings;
    } else {
        ss.batch.use_graphs = 1;
    }
    size_t free_bytes = 0, total_bytes = 0;
    MR_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
    ss.hbm_budget_bytes = free_bytes / 10 * 8;
    ss.max_jobs         = 4096;
    for (size_t i = 0; i < count; ++i) {
        jobs[i].status = MR_OK;
    }
    const auto              t0 = Clock::now();
    size_t                  slot = 0;
    std::unique_ptr<Server> private_server;
    Server*                 cached = take_cached_server(ss, slot);
    if (!cached) {
        private_server = std::make_unique<Server>(ss);
    }
    struct Return {
        Server* cached;
        size_t  slot;
        ~Return() {
            if (cached) {
                return_cached_server(slot);
            }
        }
    } give_back{cached, slot};
    Server& server = cached ? *cached : *private_server;
    const mr_server_statistics stats_before = server.statistics();
    const mr_path_statistics   paths_before = server.path_statistics();
    cudaEvent_t marks[2] = {nullptr, nullptr};
    MR_CUDA(cudaEventCreate(&marks[0]));
    MR_CUDA(cudaEventCreate(&marks[1]));
    server.record_after_lanes(marks[0]);
    std::vector<uint64_t> ids(count, 0);
    mr_status first = MR_OK;
    for (size_t i = 0; i < count; ++i) {
        try {
            ids[i] = server.submit(scene_ptr(jobs[i].scene), &jobs[i].render, &jobs[i].integrator,
                                   copy_images ? jobs[i].rgb : nullptr, copy_images && jobs[i].rgb);
        } catch (const Error& e) {
            jobs[i].status = e.status;
            if (first == MR_OK) {
                first = e.status;
                set_last_error(e.what());
            }
        }
    }
    server.wait_all();
    const double seconds = std::chrono::duration<double>(Clock::now() - t0).count();
    server.record_after_lanes(marks[1]);
    float device_ms = 0;
    MR_CUDA(cudaEventSynchronize(marks[1]));
    MR_CUDA(cudaEventElapsedTime(&device_ms, marks[0], marks[1]));
    cudaEventDestroy(marks[0]);
    cudaEventDestroy(marks[1]);
    for (size_t i = 0; i < count; ++i) {
        if (ids[i] == 0) {
            continue;
        }
        const mr_job_info info = server.info(ids[i]);
        if (info.state != MR_JOB_COMPLETED) {
            jobs[i].status = static_cast<mr_status>(info.status);
            if (first == MR_OK) {
                first = jobs[i].status;
                set_last_error(info.error);
            }
        }
        server.release(ids[i]);
    }
    if (statistics) {
        const mr_server_statistics s = server.statistics();
        const mr_path_statistics   p = server.path_statistics();
        std::memset(statistics, 0, sizeof(*statistics));
        statistics->waves           = s.waves - stats_before.waves;
        statistics->segments        = s.segments - stats_before.segments;
        statistics->samples         = s.samples - stats_before.samples;
        statistics->kernel_launches = s.kernel_launches - stats_before.kernel_launches;
        statistics->graph_launches  = s.graph_launches - stats_before.graph_launches;
        statistics->seconds         = seconds;
        statistics->busy_seconds    = s.busy_seconds - stats_before.busy_seconds;
        statistics->device_seconds  = device_ms * 1e-3;
        statistics->paths.paths                    = p.paths - paths_before.paths;
        statistics->paths.shadow_rays              = p.shadow_rays - paths_before.shadow_rays;
        statistics->paths.scattering_events        = p.scattering_events - paths_before.scattering_events;
        statistics->paths.roulette_terminations    = p.roulette_terminations - paths_before.roulette_terminations;
        statistics->paths.medium_scattering_events =
            p.medium_scattering_events - paths_before.medium_scattering_events;
        statistics->paths.geometry.bounds_tests =
            p.geometry.bounds_tests - paths_before.geometry.bounds_tests;
        statistics->paths.geometry.triangle_tests =
            p.geometry.triangle_tests - paths_before.geometry.triangle_tests;
    }
    return first;
}

}  // namespace
}  // namespace mr

struct mr_server {
    std::unique_ptr<mr::Server> impl;
};

using namespace mr;

namespace {

Server& server_of(mr_server* s) {
    require(s != nullptr && s->impl != nullptr, "Server handle is null");
    return *s->impl;
}

}  // namespace

extern "C" {

mr_status mr_render_batch(mr_batch_job* jobs, size_t count, const mr_batch_settings* settings,
                          mr_batch_statistics* statistics) {
    mr_status status = MR_OK;
    const mr_status call = guarded([&] { status = run_batch(jobs, count, settings, statistics, true); });
    return call != MR_OK ? call : status;
}

mr_status mr_batch_autotune(const mr_batch_job* jobs, size_t count, mr_batch_settings* best,
                            double* samples_per_second) {
    return guarded([&] {
        require(jobs != nullptr && count > 0, "Calibration jobs are missing");
        require(best != nullptr, "Output is null");
        std::vector<mr_batch_job> local(jobs, jobs + count);
        int trace_max = 0, shade_max = 0;
        Engine::batch_occupancy(trace_max, shade_max);
        const uint64_t waves[]      = {size_t(1) << 21, size_t(1) << 22, size_t(1) << 23};
        const uint32_t lanes[]      = {1u, 2u, 3u, 4u};
        const uint32_t thresholds[] = {0u, 1u << 15};
        // Samples per device second of one calibration render (the engine's own events, so the
        // host-side setup of a new wave shape is not counted).
        const auto rate_of = [&](const mr_batch_settings& c) {
            mr_batch_statistics st{};
            const mr_status     s = run_batch(local.data(), local.size(), &c, &st, false);
            if (s != MR_OK) {
                fail(s, "Calibration render failed");
            }
            const double t = st.device_seconds > 0 ? st.device_seconds : st.seconds;
            return t > 0 ? static_cast<double>(st.samples) / t : 0.0;
        };
        struct Candidate {
            mr_batch_settings settings;
            double            rate;
        };
        std::vector<Candidate> all;
        for (uint64_t w : waves) {
            for (uint32_t l : lanes) {
                for (uint32_t t : thresholds) {
                    mr_batch_settings c{};
                    c.wave_paths       = w;
                    c.concurrent_waves = l;
                    c.sort_threshold   = t;
                    c.use_graphs       = 1;
                    all.push_back({c, rate_of(c)});
                }
            }
        }
        // One short render per shape is noisy (a few percent): the best three shapes, each also
        // with fewer resident traversal blocks (more cache per warp), are rendered twice more and
        // ranked by their best run.
        std::stable_sort(all.begin(), all.end(),
                         [](const Candidate& a, const Candidate& b) { return a.rate > b.rate; });
        std::vector<Candidate> finals;
        for (size_t i = 0; i < all.size() && i < 3; ++i) {
            finals.push_back(all[i]);
            Candidate fewer = all[i];
            fewer.settings.trace_blocks_per_sm = static_cast<uint32_t>(std::max(1, trace_max * 3 / 4));
            fewer.rate = 0;
            finals.push_back(fewer);
        }
        for (int round = 0; round < 2; ++round) {
            for (Candidate& f : finals) {
                f.rate = std::max(f.rate, rate_of(f.settings));
            }
        }
        double            top = -1;
        mr_batch_settings pick{};
        for (const Candidate& f : finals) {
            if (f.rate > top) {
                top  = f.rate;
                pick = f.settings;
            }
        }
        *best = pick;
        if (samples_per_second) {
            *samples_per_second = top;
        }
    });
}

mr_status mr_server_create(const mr_server_settings* settings, mr_server** server) {
    return guarded([&] {
        require(server != nullptr, "Output is null");
        mr_server_settings s{};
        if (settings) {
            s = *settings;
        } else {
            s.batch.use_graphs = 1;
        }
        auto out  = std::make_unique<mr_server>();
        out->impl = std::make_unique<Server>(s);
        *server   = out.release();
    });
}

mr_status mr_server_destroy(mr_server* server) {
    return guarded([&] { delete server; });
}

mr_status mr_server_submit(mr_server* server, const mr_scene* scene, const mr_render_settings* render,
                           const mr_integrator_settings* integrator, uint64_t* job) {
    return guarded([&] {
        require(job != nullptr, "Output is null");
        *job = server_of(server).submit(scene_ptr(scene), render, integrator, nullptr);
    });
}

mr_status mr_server_pause(mr_server* server, uint64_t job, int* accepted) {
    return guarded([&] {
        const bool a = server_of(server).pause(job);
        if (accepted) {
            *accepted = a ? 1 : 0;
        }
    });
}

mr_status mr_server_resume(mr_server* server, uint64_t job, int* accepted) {
    return guarded([&] {
        const bool a = server_of(server).resume(job);
        if (accepted) {
            *accepted = a ? 1 : 0;
        }
    });
}

mr_status mr_server_cancel(mr_server* server, uint64_t job) {
    return guarded([&] { server_of(server).cancel(job); });
}

mr_status mr_server_wait(mr_server* server, uint64_t job, uint32_t milliseconds, int* finished) {
    return guarded([&] {
        const bool done = server_of(server).wait(job, milliseconds);
        if (finished) {
            *finished = done ? 1 : 0;
        }
    });
}

mr_status mr_server_job_info(mr_server* server, uint64_t job, mr_job_info* info) {
    return guarded([&] {
        require(info != nullptr, "Output is null");
        *info = server_of(server).info(job);
    });
}

mr_status mr_server_result(mr_server* server, uint64_t job, float* rgb, size_t capacity) {
    return guarded([&] { server_of(server).result(job, rgb, capacity); });
}

mr_status mr_server_preview(mr_server* server, uint64_t job, float* rgb, size_t capacity,
                            uint64_t* samples) {
    return guarded([&] {
        const uint64_t n = server_of(server).preview(job, rgb, capacity);
        if (samples) {
            *samples = n;
        }
    });
}

mr_status mr_server_release(mr_server* server, uint64_t job) {
    return guarded([&] { server_of(server).release(job); });
}

mr_status mr_server_get_statistics(mr_server* server, mr_server_statistics* statistics) {
    return guarded([&] {
        require(statistics != nullptr, "Output is null");
        *statistics = server_of(server).statistics();
    });
}

}  // extern "C"
