// wavefront.cuh — path state, queues and the wavefront driver interface.
#pragma once

#include <atomic>
#include <mutex>
#include <vector>

#include "scene.cuh"

namespace mr {

// Material bins of the extension result: paths are shaded bin by bin (sorted by material).
enum Bin : int {
    kBinMiss       = 0,
    kBinDiffuse    = 1,
    kBinConductor  = 2,
    kBinMirror     = 3,
    kBinDielectric = 4,
    kBinMedium     = 5,
    kBinCount      = 6,
};

struct BounceCounters {
    uint32_t ext;                 // paths entering this bounce
    uint32_t bins[kBinCount];
    uint32_t shadow;
    uint32_t work_extend;  // work fetch of the bounce's trace launch
    uint32_t pad[7];
};

enum Stat : int {
    kStatPaths = 0,
    kStatShadowRays,
    kStatScattering,
    kStatRoulette,
    kStatMedium,
    kStatExtendBounds,
    kStatExtendTriangles,
    kStatShadowBounds,
    kStatShadowTriangles,
    kStatCount
};

struct IntegratorParams {
    uint32_t mode;
    uint32_t maximum_depth;
    uint32_t russian_roulette;
    uint32_t roulette_depth;
};

// One job's share of a multi-job wave: a pixel rectangle x sample range of one render, with
// everything the kernels need to trace it (the job's scene, integrator settings and buffers).
struct WaveSegment {
    DeviceScene      scene;
    IntegratorParams p;
    uint32_t         x0, y0, w, h;      // pixel rectangle
    uint32_t         s0, ns;            // samples s0 .. s0+ns, sample-major path slots
    uint32_t         width, height, spp;
    uint32_t         first_path;        // wave slot of the segment's first path
    uint64_t         seed;
    float4*          accumulator;       // the job's (sum, compensation) per pixel
    float*           rgb;               // the job's image; pixels whose last sample resolves here
    unsigned*        error;             // the job's error word
};

constexpr uint32_t kMaxSegments = 1024;

// Device descriptor of a multi-job wave. Segments are sorted by first_path; first_path[] and
// first_pixel[] hold count+1 prefix entries so kernels find a path's or pixel's segment by
// binary search.
struct WaveDesc {
    uint32_t    count;           // paths in the wave
    uint32_t    segments;
    uint32_t    pixels;          // resolve index space: sum of w*h over segments
    uint32_t    sort_threshold;  // queues shorter than this are not sorted by material
    uint32_t    first_path[kMaxSegments + 1];
    uint32_t    first_pixel[kMaxSegments + 1];
    uint32_t    pad[2];
    WaveSegment seg[kMaxSegments];
};

// One field of a record array: element i sits at base + i * STRIDE.
template <typename T, size_t STRIDE>
struct RecordField {
    unsigned char* base = nullptr;  // the field in record 0
    __host__ __device__ __forceinline__ T& operator[](size_t i) const {
        return *reinterpret_cast<T*>(base + i * STRIDE);
    }
    __host__ __device__ explicit operator bool() const { return base != nullptr; }
};

// Path state of `capacity` paths as records: one 128-byte path record and one 64-byte shadow
// record per path slot. Kernels reach paths by slot in queue and bin order, which scatters the
// slots; a record keeps what one kernel reads of a path in whole 32-byte sectors instead of a
// 16-byte piece of a sector in each of a dozen arrays. Path record sectors: the ray (ray_o,
// ray_d: what traversal reads), the hit (hit, hit_slot, flags, segment: what traversal writes),
// throughput and previous vertex (beta, prev), radiance and RNG (radiance, rng). Shading reads
// and writes the four; a shadow test reads the shadow record's ray and, when the segment is clear,
// its contribution and the path's radiance sector.
constexpr size_t kPathRecordBytes   = 128;
constexpr size_t kShadowRecordBytes = 64;

template <typename T>
using PathField = RecordField<T, kPathRecordBytes>;
template <typename T>
using ShadowField = RecordField<T, kShadowRecordBytes>;

struct PathState {
    PathField<float4>     ray_o;     // origin, interval minimum                        (+0)
    PathField<float4>     ray_d;     // direction, interval maximum                     (+16)
    PathField<float4>     hit;       // distance, barycentrics (medium: distance, g)    (+32)
    PathField<uint32_t>   hit_slot;  // triangle slot, kNone on a miss                  (+48)
    PathField<uint32_t>   flags;     // bit 0: previous event was delta                 (+52)
    PathField<uint32_t>   segment;   // multi-job waves: the path's wave segment        (+56)
    PathField<float4>     beta;      // throughput, eta scale                           (+64)
    PathField<float4>     prev;      // previous scattering vertex, previous pdf        (+80)
    PathField<float4>     radiance;  // accumulated radiance                            (+96)
    PathField<ulonglong2> rng;       // PCG state, increment                            (+112)
    ShadowField<float4>   shadow_o;  // shadow origin, segment limit                    (+0)
    ShadowField<float4>   shadow_d;  // shadow direction                                (+16)
    ShadowField<float4>   shadow_c;  // unoccluded contribution                         (+32)

    // Views of `paths` (capacity x 128 bytes) and `shadows` (capacity x 64 bytes), both
    // 128-byte aligned. Without `with_segment` the segment field stays unset (single-job use).
    void view(unsigned char* paths, unsigned char* shadows, bool with_segment) {
        ray_o.base    = paths + 0;
        ray_d.base    = paths + 16;
        hit.base      = paths + 32;
        hit_slot.base = paths + 48;
        flags.base    = paths + 52;
        segment.base  = with_segment ? paths + 56 : nullptr;
        beta.base     = paths + 64;
        prev.base     = paths + 80;
        radiance.base = paths + 96;
        rng.base      = paths + 112;
        shadow_o.base = shadows + 0;
        shadow_d.base = shadows + 16;
        shadow_c.base = shadows + 32;
    }
};

// Coherence sort of the extension and shadow rays between bounces: a counting sort on a key made of where
// the ray starts (the position of its origin's triangle in the tree's leaf order, in 16,384 equal
// ranges; or, for a medium vertex, the Morton code of its cell in the scene's bounds, 4 bits per
// axis) and its direction octant. Leaf order follows the tree, so a range covers a compact piece of geometry
// however the geometry is spread. Waves of fewer paths than kRaySortMinPaths and scenes of fewer
// triangle slots than kRaySortMinSlots are not sorted: their traversal is too cheap for the sort
// to pay.
constexpr int      kSortAxisBits    = 4;
constexpr uint32_t kSortCells       = 1u << 14;  // >= 2^(3 kSortAxisBits)
constexpr uint32_t kSortBuckets     = 8u * kSortCells;
constexpr uint32_t kRaySortMinPaths = 1u << 18;
constexpr uint32_t kRaySortMinSlots = 4096;
// Lanes (workspace + stream) that a plain frame of several waves goes round, so that one wave's
// last bounces overlap the next waves' first (two lanes: 1M-triangle frame -7.0%; three: a
// further -1.7%; four: a further -1.0%).
constexpr uint32_t kFrameLanes = 4;

struct Queues {
    uint32_t*       ext[2];
    uint32_t*       staging;  // this bounce's continuing paths before the sort (null: no sort)
    uint32_t*       keys;     // their sort keys, at the same positions
    uint32_t*       shadow_staging;  // this bounce's shadow rays before the sort
    uint32_t*       shadow_keys;     // their sort keys
    uint32_t*       buckets;  // 2 kSortBuckets counts (extension rays, then shadow rays), then the
                              // 2 kSortBuckets cursors
    uint32_t*       bins;    // kBinCount * capacity
    uint32_t*       shadow;
    BounceCounters* counters;  // maximum_depth + 2 entries
    unsigned long long* stats;  // kStatCount
    unsigned*           error;
};

// Device workspace for `capacity` concurrent paths; pooled and reused across renders.
struct Workspace {
    size_t    capacity     = 0;
    uint32_t  max_bounces  = 0;
    void*     memory       = nullptr;
    size_t    bytes        = 0;
    PathState state{};
    Queues    queues{};
    float4*   accumulator  = nullptr;  // Kahan sum per pixel (sum, compensation) of a frame
    size_t    pixels       = 0;
    int       device       = 0;
    ~Workspace();
};

// Diagnostics: first-bounce shadow rays (2 float4 per path), a flag per path that one was
// traced, and its occlusion result (device buffers of the wave's path count).
struct ShadowCapture {
    float4*  rays;
    uint8_t* has_shadow;
    uint8_t* occluded;
};

// How the paths of one wave start.
enum InitKind : int { kInitCamera = 0, kInitPixelList = 1, kInitRays = 2 };

struct WaveInit {
    InitKind        kind;
    // camera waves: pixel rectangle x0..x0+w, y0..y0+h of a width x height image, samples
    // s0..s0+ns, sample-major slots.
    uint32_t        x0, y0, w, h;
    uint32_t        s0, ns;
    uint32_t        width, height;
    uint64_t        seed;
    // pixel lists / explicit rays
    const uint32_t* pixels;   // x, y pairs (device)
    const uint64_t* samples;  // (device)
    const float4*   rays;     // origin+min, direction+max pairs (device)
    const uint64_t* keys;     // seed, pixel, sample triples (device)
    uint32_t        count;
    float4*         camera_rays_out;  // optional (device), 2 float4 per path
    ShadowCapture*  capture;          // optional diagnostics (host struct of device pointers)
};

// Grid sizes of the persistent kernels of a multi-job wave (blocks of 128 threads).
struct BatchShape {
    int trace_blocks = 0;
    int shade_blocks = 0;
};

class Engine {
  public:
    // Renders one wave on `stream`: initialises `count` paths, runs up to maximum_depth + 1
    // bounces. Path radiance stays in ws.state.radiance (slot order).
    static void run_wave(const Scene& scene, const IntegratorParams& params, const WaveInit& init,
                         Workspace& ws, cudaStream_t stream);

    // Enqueues the paths of one multi-job wave whose descriptor is already in device memory
    // (`wave`): camera paths of every segment and up to maximum_depth + 1 bounces; radiance stays
    // per path. The launch sequence depends only on its arguments, so it can be captured once in
    // a CUDA graph and replayed for every wave of the same depth.
    static void enqueue_batch_paths(const WaveDesc* wave, uint32_t maximum_depth, bool media, bool two,
                                    bool ray_sort, const BatchShape& shape, Workspace& ws,
                                    cudaStream_t stream);

    // Enqueues the per-pixel resolve of a wave's radiance into each job's accumulator and image.
    static void enqueue_batch_resolve(const WaveDesc* wave, Workspace& ws, cudaStream_t stream);

    // Largest grids the batch kernels can keep resident (blocks per SM at 128 threads).
    static void batch_occupancy(int& trace_blocks_per_sm, int& shade_blocks_per_sm);

    // Kernel launches of one wave (paths + resolve).
    static uint64_t batch_wave_launches(uint32_t maximum_depth, bool ray_sort) {
        return 2ull + 2ull * (maximum_depth + 1) + (ray_sort ? 4ull * maximum_depth : 0ull);
    }
};

// Workspace pool (per device).
std::shared_ptr<Workspace> acquire_workspace(size_t capacity, uint32_t max_bounces, size_t pixels);
void                       release_workspace(std::shared_ptr<Workspace> ws);

// Kernel timing for roofline figures (nearest-hit traversal launches).
struct KernelTiming {
    std::mutex         mutex;
    std::atomic<bool>  enabled{false};
    std::atomic<uint64_t> all_launches{0};
    uint64_t           launches = 0;
    double             seconds  = 0;
    mr_trace_statistics counted{};
};
KernelTiming& kernel_timing();

// Counts kernel launches for mr_kernel_timing while timing is enabled.
inline void note_launches(uint64_t n) {
    KernelTiming& t = kernel_timing();
    if (t.enabled.load(std::memory_order_relaxed)) {
        t.all_launches.fetch_add(n, std::memory_order_relaxed);
    }
}

// Frame render into a device image (width*height*3 floats) — used by mr_render(_device) and the
// session. Statistics (optional) are read back after the frame.
// With row_begin/row_end the rows [row_begin, row_end) of the frame are rendered into a
// width*(row_end-row_begin)*3 image; every pixel is the full frame's pixel bit for bit.
void render_frame(const Scene& scene, const IntegratorParams& params, const mr_render_settings& render,
                  float* device_rgb, cudaStream_t stream, mr_path_statistics* statistics,
                  size_t max_paths = 0, uint32_t row_begin = 0, uint32_t row_end = 0xFFFFFFFFu);

// A further workspace and stream that a tile's waves may alternate with the first.
struct TileLane {
    Workspace*   ws     = nullptr;
    cudaStream_t stream = nullptr;
};

// Accumulates the samples [s0, s0+ns) of a pixel rectangle into a caller-owned Kahan
// accumulator (float4 sum + float4 compensation per pixel of the full image).
// The accumulator's first row is image row `accumulator_row0`. With further lanes (`more`)
// consecutive waves go round the lanes (`ws` and `stream` first), so one wave's last, sparse
// bounces overlap the next wave's first; the resolves still run one after the other in wave
// order (per pixel, samples accumulate in order), and `stream` waits for all of it.
void render_tile(const Scene& scene, const IntegratorParams& params, const mr_render_settings& render,
                 uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t s0, uint32_t ns,
                 float4* accumulator, Workspace& ws, cudaStream_t stream, uint32_t accumulator_row0 = 0,
                 const TileLane* more = nullptr, uint32_t more_count = 0);

void read_statistics(Workspace& ws, cudaStream_t stream, mr_path_statistics* out, unsigned* error);
void reset_statistics(Workspace& ws, cudaStream_t stream);
mr_status error_status(unsigned error, std::string& message);

}  // namespace mr
