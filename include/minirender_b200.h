/*
 * minirender_b200.h — C ABI of the B200 offline path tracer.
 *
 * This is the drop-in boundary for MiniRender's CPU offline render call. The reference has no
 * FFI: its callers link the C++ classes `PathTracer` (include/minirender/render/path_tracer.hpp)
 * and `RenderSession` (include/minirender/render/render_session.hpp). Every entry point below
 * replaces one of those calls; the citation beside it names the reference interface
 * (file:line inside the MiniRender source tree).
 *
 * Conventions
 *  - Plain C: pointers, sizes and POD structs. No C++ or torch types cross the boundary.
 *  - Every call returns an `mr_status`. C++ exceptions of the reference map onto status codes
 *    (std::invalid_argument -> MR_INVALID_ARGUMENT, std::overflow_error -> MR_OVERFLOW, ...);
 *    `mr_last_error` returns the message of the calling thread's last failure.
 *  - Host pointers are host memory unless the name says `device`.
 *  - All device arithmetic is FP32. Scene inputs keep the reference's types (float meshes and
 *    matrices, double medium coefficients), so the same descriptor also feeds the CPU oracle.
 *  - The library never falls back to the CPU: without a usable CUDA device every compute entry
 *    point returns MR_CUDA_ERROR.
 */
#ifndef MINIRENDER_B200_H
#define MINIRENDER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MR_ABI_VERSION 1u

typedef enum mr_status {
    MR_OK               = 0,
    MR_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    MR_OUT_OF_RANGE     = 2, /* std::out_of_range */
    MR_OVERFLOW         = 3, /* std::overflow_error: radiance above FLT_MAX */
    MR_RUNTIME_ERROR    = 4, /* std::runtime_error: nonfinite or negative path contribution */
    MR_CANCELLED        = 5, /* OperationCancelled */
    MR_LOGIC_ERROR      = 6, /* std::logic_error: session still active */
    MR_LENGTH_ERROR     = 7, /* std::length_error: index range exceeded */
    MR_CUDA_ERROR       = 8, /* CUDA runtime failure or no device */
    MR_OUT_OF_MEMORY    = 9, /* device allocation failed or HBM budget exceeded */
    MR_TIMEOUT          = 10 /* a bounded device or host wait gave up */
} mr_status;

/* MaterialKind (include/minirender/scene/scene.hpp:106). cloth and subsurface are rejected. */
typedef enum mr_material_kind {
    MR_MATERIAL_DIFFUSE    = 0,
    MR_MATERIAL_CONDUCTOR  = 1,
    MR_MATERIAL_MIRROR     = 2,
    MR_MATERIAL_DIELECTRIC = 3,
    MR_MATERIAL_CLOTH      = 4,
    MR_MATERIAL_SUBSURFACE = 5
} mr_material_kind;

/* SamplingMode (include/minirender/render/path_tracer.hpp:13). */
typedef enum mr_sampling_mode {
    MR_SAMPLING_BSDF  = 0,
    MR_SAMPLING_LIGHT = 1,
    MR_SAMPLING_MIS   = 2
} mr_sampling_mode;

/* RenderState (include/minirender/render/render_session.hpp:12-23). */
typedef enum mr_render_state {
    MR_STATE_IDLE       = 0,
    MR_STATE_PREPARING  = 1,
    MR_STATE_RUNNING    = 2,
    MR_STATE_PAUSING    = 3,
    MR_STATE_PAUSED     = 4,
    MR_STATE_FINALIZING = 5,
    MR_STATE_CANCELLING = 6,
    MR_STATE_CANCELLED  = 7,
    MR_STATE_COMPLETED  = 8,
    MR_STATE_FAILED     = 9
} mr_render_state;

/* Camera (include/minirender/scene/scene.hpp:85-104). */
typedef struct mr_camera {
    float position[3];
    float target[3];
    float up[3];
    float vertical_fov_degrees;
    float near_plane;
    float far_plane;
    float aperture_radius;
    float focus_distance;
} mr_camera;

/* TextureFilter (include/minirender/core/texture.hpp:14). */
typedef enum mr_texture_filter {
    MR_FILTER_NEAREST   = 0,
    MR_FILTER_BILINEAR  = 1,
    MR_FILTER_TRILINEAR = 2
} mr_texture_filter;

/* Material (include/minirender/scene/scene.hpp:113-136), the fields the offline path reads.
 * Textures are 1-based indices into mr_scene_desc.textures, 0 = none (RenderInstance resolves
 * the material's texture ids, include/minirender/scene/scene.hpp:201-209). */
typedef struct mr_material {
    uint32_t kind; /* mr_material_kind */
    float    base_color[3];
    float    emission[3];
    float    roughness;
    float    ior;
    uint32_t double_sided;
    uint32_t base_color_texture; /* multiplies base_color after clamping to [0,1] */
    uint32_t texture_filter;     /* mr_texture_filter of both textures */
    uint32_t normal_texture;     /* tangent-space normals decoded in the triangle's UV frame */
    float    normal_scale;       /* xy scale of the decoded normal; <= 0 disables the map */
    uint32_t normal_flip_y;
} mr_material;

/* A decoded texture (TextureAsset's data, include/minirender/scene/scene.hpp:148-154): linear
 * RGB, width * height * 3 floats, row 0 at the top of the image. */
typedef struct mr_texture {
    const float* rgb;
    uint32_t     width;
    uint32_t     height;
} mr_texture;

/* MeshCorner (include/minirender/scene/scene.hpp:33-37): 24 bytes. */
typedef struct mr_mesh_corner {
    uint32_t position;
    float    normal[3];
    float    uv[2];
} mr_mesh_corner;

/* MeshData (include/minirender/scene/scene.hpp:45-50): positions and 3 corners per triangle. */
typedef struct mr_mesh {
    const float*          positions; /* 3 * position_count */
    uint32_t              position_count;
    const mr_mesh_corner* corners; /* 3 * triangle_count */
    uint32_t              triangle_count;
} mr_mesh;

/* RenderInstance (include/minirender/scene/scene.hpp:201-209). Matrices are column-major
 * (glm layout): object_to_world[4*c + r], normal_to_world[3*c + r]. */
typedef struct mr_instance {
    uint32_t mesh;
    uint32_t material;
    float    object_to_world[16];
    float    normal_to_world[9];
} mr_instance;

/* DirectionalLight (include/minirender/scene/scene.hpp:170-175). */
typedef struct mr_directional_light {
    float direction[3];
    float color[3];
    float intensity;
} mr_directional_light;

/* MediumRegion + HomogeneousMedium (include/minirender/scene/medium.hpp:14-41). */
typedef struct mr_medium_region {
    double   minimum[3];
    double   maximum[3];
    double   absorption[3];
    double   scattering[3];
    double   anisotropy;
    uint32_t enabled;
} mr_medium_region;

/* SceneSnapshot (include/minirender/scene/scene.hpp:220-230). */
typedef struct mr_scene_desc {
    mr_camera                   camera;
    float                       environment[3];
    const mr_mesh*              meshes;
    uint32_t                    mesh_count;
    const mr_material*          materials;
    uint32_t                    material_count;
    const mr_instance*          instances;
    uint32_t                    instance_count;
    const mr_directional_light* directional_lights;
    uint32_t                    directional_light_count;
    const mr_medium_region*     media;
    uint32_t                    medium_count;
    const mr_texture*           textures;
    uint32_t                    texture_count;
    uint32_t                    environment_texture;  /* 1-based lat-long map, 0 = none */
    float                       environment_strength; /* scales the map (not the constant) */
    float                       environment_rotation_degrees; /* about +Y, right-handed */
} mr_scene_desc;

/* SceneBvh::Node (include/minirender/render/bvh.hpp:81-86), the reference's flat node layout.
 * Leaf: count > 0 and [first, first+count) indexes `order`. Interior: count == 0, `first` is
 * the left child and `right` the right child. Primitive ids enumerate instances in order and
 * their triangles in order, as in SceneBvh's constructor (src/render/bvh.cpp:53-89). */
typedef struct mr_bvh_node {
    float    minimum[3];
    float    maximum[3];
    uint32_t first;
    uint32_t right;
    uint32_t count;
} mr_bvh_node;

typedef struct mr_bvh_desc {
    const mr_bvh_node* nodes;
    uint32_t           node_count;
    const uint32_t*    order;
    uint32_t           primitive_count;
} mr_bvh_desc;

/* IntegratorSettings (include/minirender/render/path_tracer.hpp:21-35), path tracing only. */
typedef struct mr_integrator_settings {
    uint32_t mode; /* mr_sampling_mode */
    uint32_t maximum_depth;
    uint32_t russian_roulette;
    uint32_t roulette_depth;
} mr_integrator_settings;

/* RenderSettings (include/minirender/render/path_tracer.hpp:38-49). */
typedef struct mr_render_settings {
    uint64_t width;
    uint64_t height;
    uint32_t samples_per_pixel;
    uint64_t seed;
} mr_render_settings;

/* SessionSettings (include/minirender/render/render_session.hpp:30-38), validated with the
 * reference's limits. batch_samples keeps its meaning: samples added per pixel between two
 * commits (progress, preview, pause and cancel points). The GPU advances the whole image per
 * batch, so `threads` and `tile_size` do not change the schedule; results are bitwise the same
 * for every setting, as in the reference. */
typedef struct mr_session_settings {
    uint32_t threads;
    uint32_t tile_size;
    uint32_t batch_samples;
} mr_session_settings;

/* TraceStatistics (include/minirender/render/bvh.hpp:37-40). */
typedef struct mr_trace_statistics {
    uint64_t bounds_tests;
    uint64_t triangle_tests;
} mr_trace_statistics;

/* PathStatistics (include/minirender/render/path_tracer.hpp:52-68). */
typedef struct mr_path_statistics {
    mr_trace_statistics geometry;
    uint64_t            paths;
    uint64_t            shadow_rays;
    uint64_t            scattering_events;
    uint64_t            roulette_terminations;
    uint64_t            medium_scattering_events;
    uint64_t            subsurface_events;
    double              subsurface_distance;
} mr_path_statistics;

/* BvhBuildStatistics (include/minirender/render/bvh.hpp:29-34). */
typedef struct mr_bvh_statistics {
    uint64_t triangles;
    uint64_t nodes;
    uint64_t leaves;
    uint64_t maximum_depth;
} mr_bvh_statistics;

/* Ray + RayInterval (include/minirender/scene/scene.hpp:27-30,
 * include/minirender/render/intersection.hpp:15-20) in FP32: 32 bytes. */
typedef struct mr_ray {
    float origin[3];
    float direction[3];
    float minimum;
    float maximum; /* +inf allowed */
} mr_ray;

/* The part of SurfaceHit (include/minirender/render/bvh.hpp:15-26) that identifies the hit. */
typedef struct mr_hit {
    float    distance;
    uint32_t instance_index;
    uint32_t triangle_index;
    uint32_t primitive; /* flat primitive id (instance-major), UINT32_MAX on a miss */
    float    barycentric[3];
    uint32_t front_face;
} mr_hit;

/* RenderProgress (include/minirender/render/render_session.hpp:41-65), path tracing part. */
typedef struct mr_render_progress {
    uint32_t           state; /* mr_render_state */
    uint64_t           job_id;
    uint64_t           recorded_samples;
    uint64_t           total_samples;
    uint64_t           completed_pixels;
    uint32_t           worker_count;
    double             elapsed_seconds;
    mr_path_statistics statistics;
    char               error[256];
} mr_render_progress;

/* RenderPreview (include/minirender/render/render_session.hpp:68-77) without the image, which
 * the caller receives in its own buffer. */
typedef struct mr_render_preview {
    uint64_t job_id;
    uint64_t revision;
    uint64_t recorded_samples;
    uint64_t width;
    uint64_t height;
    uint32_t available; /* 0 when the preview lock was busy (reference returns no image) */
} mr_render_preview;

typedef struct mr_scene   mr_scene;
typedef struct mr_session mr_session;

/* ---- library ---------------------------------------------------------------------------- */

/* ABI version of the loaded library (MR_ABI_VERSION). No reference counterpart. */
uint32_t mr_abi_version(void);

/* Copies the calling thread's last error message into `buffer` (always NUL-terminated) and
 * returns its full length. Stands in for the reference's exception `what()` strings. */
size_t mr_last_error(char* buffer, size_t capacity);

/* ---- scene ------------------------------------------------------------------------------ */

/* Validates the snapshot, uploads it to the current CUDA device and builds everything the
 * reference's PathTracer constructor builds (src/render/path_tracer.cpp:111-120): the SceneBvh
 * (src/render/bvh.cpp:31-99; here the GPU binned-SAH builder, or `bvh` when non-null, which
 * must be the reference layout of the same primitives), the LightSampler
 * (src/render/light.cpp:197-264) and the MediumField (src/render/medium.cpp:145-148). */
mr_status mr_scene_create(const mr_scene_desc* desc, const mr_bvh_desc* bvh, mr_scene** scene);

/* Builder options. No reference counterpart: the reference bins whole triangles only. */
typedef struct mr_build_settings {
    uint32_t split_references; /* nonzero: early split clipping. A triangle whose box area exceeds
                                  split_factor x the mean triangle box area enters the build once
                                  per nonempty cell of a grid over its box, with the clipped
                                  bounds. Hits, images and statistics of paths are unchanged (the
                                  same triangles are tested); the tree, its SAH cost and its leaf
                                  slots differ from the reference builder's. */
    float    split_factor;     /* 0 = 16 */
    uint64_t max_references;   /* cap on leaf slots; 0 = max(2 x triangles, triangles + 65536) */
    uint32_t two_level;        /* nonzero: an instance-level tree (TLAS) over one object-space
                                  tree per mesh (BLAS) instead of the reference's flattened
                                  world-space tree (src/render/bvh.cpp:31-99). Triangles are still
                                  tested in world space with the flattening's own arithmetic, so
                                  hits, images and path statistics other than the traversal
                                  counters equal the flattened scene's; a mesh instanced many
                                  times is stored once. Not combinable with split references or
                                  an imported tree. Enables mr_scene_update_instances and
                                  mr_scene_update_mesh. */
} mr_build_settings;

/* mr_scene_create with builder options (`build` NULL = mr_scene_create). A scene built with
 * split references or two levels cannot be exported in the reference layout (MR_LOGIC_ERROR). */
mr_status mr_scene_create_with(const mr_scene_desc* desc, const mr_bvh_desc* bvh,
                               const mr_build_settings* build, mr_scene** scene);

/* Releases every device and host resource of the scene. */
mr_status mr_scene_destroy(mr_scene* scene);

/* Refit of a two-level scene, no reference counterpart (the reference rebuilds its flattened
 * tree for every new snapshot, src/render/bvh.cpp:31-99). Replaces the transforms
 * (object_to_world, normal_to_world) of instances [first, first + count) with those of
 * `instances` (their mesh and material must be unchanged) and rebuilds the instance-level tree;
 * every mesh tree is reused. The scene then renders exactly as a scene created from the updated
 * description. Emissive instances cannot move (their triangles are the scene's area lights):
 * MR_INVALID_ARGUMENT, as for a flattened scene. Not thread-safe against rendering the same
 * scene. */
mr_status mr_scene_update_instances(mr_scene* scene, uint32_t first, uint32_t count,
                                    const mr_instance* instances);

/* Refit of a two-level scene, no reference counterpart: replaces the object-space positions of
 * mesh `mesh` (same position count, same triangles) and refits its tree bottom-up (the topology
 * is kept, the boxes are recomputed), then rebuilds the instance-level tree. Meshes used by an
 * emissive instance cannot change (MR_INVALID_ARGUMENT). */
mr_status mr_scene_update_mesh(mr_scene* scene, uint32_t mesh, const float* positions,
                               uint32_t position_count);

/* Device bytes held by the scene (geometry, trees, light and material tables). No reference
 * counterpart. */
mr_status mr_scene_device_bytes(const mr_scene* scene, uint64_t* bytes);

/* SceneBvh::statistics (include/minirender/render/bvh.hpp:52). */
mr_status mr_scene_bvh_statistics(const mr_scene* scene, mr_bvh_statistics* statistics);

/* Surface-area-heuristic cost of the scene's BVH with the reference builder's constants
 * (C_T = C_I = 1, src/render/bvh.cpp:134-135): sum over interior nodes of A(node)/A(root) plus
 * sum over leaves of count * A(leaf)/A(root). No single reference function computes the
 * whole-tree figure; it is the cost the reference's split search minimises. */
mr_status mr_scene_sah_cost(const mr_scene* scene, double* cost);

/* Copies the scene's BVH out in the reference node layout (mr_bvh_node + order). Either
 * pointer may be null to query the counts only. No reference counterpart (its nodes are
 * private members, include/minirender/render/bvh.hpp:101-107). */
mr_status mr_scene_export_bvh(const mr_scene* scene, mr_bvh_node* nodes, uint32_t node_capacity,
                              uint32_t* order, uint32_t order_capacity, uint32_t* node_count,
                              uint32_t* primitive_count);

/* Seconds the scene's BVH build took on the device (CUDA events around the build kernels),
 * 0 for an imported BVH. No reference counterpart (bvh.cpp has no timer; the CLI's
 * --trace-normals times it, src/app/cli.cpp:60-97). */
mr_status mr_scene_build_seconds(const mr_scene* scene, double* seconds);

/* ---- queries ---------------------------------------------------------------------------- */

/* SceneBvh::intersect (src/render/bvh.cpp:372-378) for `count` rays: nearest hit in the closed
 * interval, ties to the lowest primitive id, single-sided culling. */
mr_status mr_intersect(const mr_scene* scene, const mr_ray* rays, size_t count, mr_hit* hits,
                       mr_trace_statistics* statistics);

/* SceneBvh::occluded (src/render/bvh.cpp:380-384) for `count` rays; occluded[i] is 0 or 1. */
mr_status mr_occluded(const mr_scene* scene, const mr_ray* rays, size_t count, uint8_t* occluded,
                      mr_trace_statistics* statistics);

/* PathTracer::trace (src/render/path_tracer.cpp:153-366) for `count` independent paths. The
 * sampler of path i is Sampler::for_sample(keys[3i], keys[3i+1], keys[3i+2])
 * (src/core/sampling.cpp:43-46); rays[i] carries the primary interval. */
mr_status mr_trace_paths(const mr_scene* scene, const mr_integrator_settings* integrator,
                         const mr_ray* rays, const uint64_t* keys, size_t count,
                         float* radiance, mr_path_statistics* statistics);

/* PathTracer::sample_pixel (src/render/path_tracer.cpp:368-386) for `count` (x, y, sample)
 * triples (`pixels` holds x, y pairs). Writes the radiance and, when `rays` is non-null, the
 * primary camera ray with its clip interval. */
mr_status mr_sample_pixels(const mr_scene* scene, const mr_integrator_settings* integrator,
                           const mr_render_settings* render, const uint32_t* pixels,
                           const uint64_t* samples, size_t count, float* radiance, mr_ray* rays,
                           mr_path_statistics* statistics);

/* Diagnostics for hit-record parity: renders the `count` camera samples like mr_sample_pixels
 * and reports, per sample, the first shadow ray its path traced (origin, direction, interval
 * [0, limit]) in `shadow_rays`, has_shadow[i] = 1 when it traced one, and occluded[i] = the
 * any-hit result. No reference counterpart (the reference traces the same ray inside
 * PathTracer::shadow_transmittance, src/render/path_tracer.cpp:126-151). */
mr_status mr_capture_shadow_rays(const mr_scene* scene, const mr_integrator_settings* integrator,
                                 const mr_render_settings* render, const uint32_t* pixels,
                                 const uint64_t* samples, size_t count, mr_ray* shadow_rays,
                                 uint8_t* has_shadow, uint8_t* occluded);

/* Largest batch mr_trace_paths_static accepts. */
#define MR_STATIC_MAX_PATHS 16384u

/* PathTracer::trace for up to MR_STATIC_MAX_PATHS paths without allocating any memory, for
 * callers that cannot allocate device memory while they render (for example a server that
 * reserves its whole HBM budget in its own pool at start-up, or a loop that must not pay the
 * device synchronisation an allocation can cause). No counterpart in the reference: it is the
 * allocation-free form of mr_trace_paths (same per-path results). `device_rays`, `device_keys`
 * (seed, pixel, sample per path) and `device_radiance` (3 floats per path) are device memory;
 * `stream` is a cudaStream_t (null = legacy default stream); the call returns after the work
 * has finished. The working memory is one fixed array of about 4.3 MB inside the library, held
 * on every GPU that loads it until the process exits. The first call on a device looks up the
 * array's address, which under CUDA's lazy module loading also loads the module and places the
 * array in device memory (an allocation and a synchronisation): warm up each device with a call
 * of count 0 (null buffers allowed) before any stream capture and before the phase that must not
 * allocate. The address is cached per device and must not be used across a cudaDeviceReset.
 * Calls share that array: it is cleared at the start of each call, and calls whose GPU work
 * overlaps race. Larger batches are rejected with MR_INVALID_ARGUMENT. */
mr_status mr_trace_paths_static(const mr_scene* scene, const mr_integrator_settings* integrator,
                                const mr_ray* device_rays, const uint64_t* device_keys,
                                size_t count, float* device_radiance, void* stream);

/* ---- render ----------------------------------------------------------------------------- */

/* PathTracer::render (src/render/path_tracer.cpp:388-405): writes width*height*3 floats of
 * linear RGB, row-major, origin top-left (include/minirender/core/image.hpp). Host buffer.
 * A frame renders in waves of at most 8,388,608 paths (pixels x samples); a frame of several
 * waves sends them round several pooled path-state workspaces (about 2 GB each at full size),
 * each with its own stream, so that one wave's last bounces overlap the next waves' first (a
 * workspace that does not fit in device memory is left out; the image is the same). The same
 * holds for mr_render_device and mr_render_rows. */
mr_status mr_render(const mr_scene* scene, const mr_integrator_settings* integrator,
                    const mr_render_settings* render, float* rgb, mr_path_statistics* statistics);

/* PathTracer::render with the image left in device memory: `device_rgb` is a device pointer
 * to width*height*3 floats and `stream` a cudaStream_t (null = the legacy default stream). The
 * work runs on `stream`; the call returns once it has finished (it reads the frame's error
 * words and statistics back). */
mr_status mr_render_device(const mr_scene* scene, const mr_integrator_settings* integrator,
                           const mr_render_settings* render, float* device_rgb, void* stream,
                           mr_path_statistics* statistics);

/* Rows [row_begin, row_end) of PathTracer::render's image into `rgb` (width*(row_end-row_begin)*3
 * host floats). Every pixel equals the full render's pixel bit for bit (each pixel's samples are
 * its own streams, summed in sample order), so ranks can render row bands of one frame and
 * gather them. No reference counterpart: the reference's tile loop is internal to
 * RenderSession (src/render/render_session.cpp:363-459). Statistics cover the band. */
mr_status mr_render_rows(const mr_scene* scene, const mr_integrator_settings* integrator,
                         const mr_render_settings* render, uint64_t row_begin, uint64_t row_end,
                         float* rgb, mr_path_statistics* statistics);

/* display_image (src/render/path_tracer.cpp:407-424): exposure + Reinhard on a host image. */
mr_status mr_display_image(const float* linear, uint64_t width, uint64_t height, double exposure,
                           float* display);

/* Kernel timing for roofline figures: when enabled, the library records CUDA events around
 * every launch of the nearest-hit traversal kernel on its launching stream; `mr_kernel_timing`
 * returns the number of those launches, their summed device time in seconds, the summed
 * bounds/triangle test counters of those launches, and the number of all kernels the library
 * launched while timing was enabled. Enabling resets the figures. While it is enabled each wave
 * of a plain render waits for the host to read its events, so the waves of a frame no longer
 * overlap on the frame's lanes: time the render itself with timing disabled. No reference
 * counterpart. */
mr_status mr_set_kernel_timing(int enabled);
mr_status mr_kernel_timing(uint64_t* launches, double* seconds, mr_trace_statistics* counted,
                           uint64_t* all_launches);

/* ---- session ---------------------------------------------------------------------------- */

/* RenderSession::RenderSession / ~RenderSession (render_session.hpp:84-87). */
mr_status mr_session_create(mr_session** session);
mr_status mr_session_destroy(mr_session* session);

/* RenderSession::start (include/minirender/render/render_session.hpp:91-92). The scene must
 * outlive the job. MR_LOGIC_ERROR while a job is active. */
mr_status mr_session_start(mr_session* session, const mr_scene* scene,
                           const mr_render_settings* render,
                           const mr_integrator_settings* integrator,
                           const mr_session_settings* settings);

/* RenderSession::pause / resume (render_session.hpp:93-96): `accepted` receives the bool. */
mr_status mr_session_pause(mr_session* session, int* accepted);
mr_status mr_session_resume(mr_session* session, int* accepted);

/* RenderSession::cancel / wait / wait_for (render_session.hpp:97-102). */
mr_status mr_session_cancel(mr_session* session);
mr_status mr_session_wait(mr_session* session);
mr_status mr_session_wait_for(mr_session* session, uint32_t milliseconds, int* terminal);

/* RenderSession::progress (render_session.hpp:104). */
mr_status mr_session_progress(const mr_session* session, mr_render_progress* progress);

/* RenderSession::preview (render_session.hpp:105-107): fills `rgb` (capacity in floats) with
 * the preview image of at most `maximum_dimension` on its longer side (0 = full size). */
mr_status mr_session_preview(const mr_session* session, uint64_t maximum_dimension, float* rgb,
                             size_t capacity, mr_render_preview* preview);

/* RenderSession::result (render_session.hpp:109): MR_OUT_OF_RANGE unless the job completed. */
mr_status mr_session_result(const mr_session* session, float* rgb, size_t capacity,
                            uint64_t* width, uint64_t* height);

/* ---- batching and serving ------------------------------------------------------------------
 * No reference counterpart: MiniRender renders one job per PathTracer::render or
 * RenderSession::start call (path_tracer.hpp:82-93, render_session.hpp:91-92). These entry points
 * render many jobs together. Their samples are packed into shared waves of GPU paths (one CUDA
 * graph launch per wave), so small jobs fill the GPU and per-job launch and copy costs overlap.
 * Every job's image is bitwise the image mr_render returns for the same scene and settings: the
 * estimator, the RNG streams and the per-pixel summation order are the same. */

/* Wave shape of the multi-job engine. Zero fields take the defaults (or the autotuner's pick). */
typedef struct mr_batch_settings {
    uint64_t wave_paths;          /* paths per wave; 0 = 1<<22 */
    uint32_t trace_blocks_per_sm; /* resident traversal blocks (128 threads) per SM; 0 = maximum */
    uint32_t shade_blocks_per_sm; /* resident shading blocks per SM; 0 = maximum */
    uint32_t sort_threshold;      /* bounce queues shorter than this skip the material sort;
                                     0 = always sort */
    uint32_t use_graphs;          /* nonzero: each wave is one launch of a captured CUDA graph */
    uint32_t concurrent_waves;    /* waves that run at once on separate streams (each with its own
                                     path state), so one wave's slow last rays overlap another's
                                     work; 0 = 2, at most 4 */
} mr_batch_settings;

/* One render of a batch: PathTracer::render's arguments plus the host image it fills. */
typedef struct mr_batch_job {
    const mr_scene*        scene;
    mr_integrator_settings integrator;
    mr_render_settings     render;
    float*                 rgb;    /* host image, width*height*3 floats; NULL = not copied back */
    mr_status              status; /* out: the job's own outcome */
} mr_batch_job;

typedef struct mr_batch_statistics {
    uint64_t           waves;
    uint64_t           segments;        /* job pieces carried by the waves */
    uint64_t           samples;         /* camera samples rendered */
    uint64_t           kernel_launches; /* device kernels run (inside graphs or not) */
    uint64_t           graph_launches;
    double             seconds;         /* wall time from the first submission to the last image */
    double             busy_seconds;    /* device time of the waves, summed over the lanes */
    double             device_seconds;  /* CUDA events on the engine's streams: before the first
                                           wave to after the last resolve */
    mr_path_statistics paths;           /* summed over all jobs */
} mr_batch_statistics;

/* Renders `count` jobs together. Returns MR_OK when every job completed; otherwise the first
 * failing job's status (each job's own status is in jobs[i].status, jobs that completed keep
 * their images). */
mr_status mr_render_batch(mr_batch_job* jobs, size_t count, const mr_batch_settings* settings,
                          mr_batch_statistics* statistics);

/* Autotuner: renders the calibration jobs once per candidate wave shape (paths per wave,
 * concurrent waves, sort threshold), then renders the three fastest shapes, each also with fewer
 * resident traversal blocks, twice more; writes the shape of the best run to `best` together with
 * the samples/s (per device second) it reached. Images are not copied back. */
mr_status mr_batch_autotune(const mr_batch_job* jobs, size_t count, mr_batch_settings* best,
                            double* samples_per_second);

/* Render server: a request loop that admits jobs as they arrive, within an HBM budget for
 * their accumulation buffers and images, keeps those buffers resident until the job ends, and
 * packs the samples of every admitted job into shared waves (continuous batching: a job that
 * arrives while others render joins the next wave). Scenes stay resident in their mr_scene
 * handles, which must outlive the jobs submitted with them. */
typedef enum mr_schedule_policy {
    MR_SCHEDULE_SHORTEST_FIRST = 0, /* fewest remaining samples first */
    MR_SCHEDULE_ARRIVAL        = 1  /* submission order */
} mr_schedule_policy;

typedef struct mr_server_settings {
    uint64_t          hbm_budget_bytes; /* job buffers admitted at once; 0 = half the free memory */
    uint32_t          max_jobs;         /* jobs admitted at once; 0 = 1024 */
    uint32_t          policy;           /* mr_schedule_policy */
    mr_batch_settings batch;
} mr_server_settings;

typedef enum mr_job_state {
    MR_JOB_QUEUED    = 0, /* waiting for HBM budget */
    MR_JOB_RUNNING   = 1,
    MR_JOB_PAUSED    = 2,
    MR_JOB_COMPLETED = 3, /* image in host memory */
    MR_JOB_CANCELLED = 4,
    MR_JOB_FAILED    = 5
} mr_job_state;

typedef struct mr_job_info {
    uint32_t state;             /* mr_job_state */
    uint32_t status;            /* mr_status of a failed job */
    uint64_t total_samples;     /* width * height * samples_per_pixel */
    uint64_t completed_samples; /* samples resolved into the accumulator */
    double   submitted_seconds; /* server clock: seconds since mr_server_create */
    double   admitted_seconds;  /* 0 until admitted */
    double   finished_seconds;  /* completed, cancelled or failed; 0 before */
    char     error[256];
} mr_job_info;

typedef struct mr_server_statistics {
    uint64_t submitted, admitted, completed, cancelled, failed;
    uint64_t waves, segments, samples, kernel_launches, graph_launches;
    uint64_t resident_bytes; /* job buffers held now */
    double   busy_seconds;   /* device time of the waves */
    double   elapsed_seconds;
} mr_server_statistics;

typedef struct mr_server mr_server;

mr_status mr_server_create(const mr_server_settings* settings, mr_server** server);
/* Cancels the jobs that have not finished, waits for the device and frees everything. */
mr_status mr_server_destroy(mr_server* server);
/* Validates like mr_render; MR_OUT_OF_MEMORY when the job alone exceeds the budget. */
mr_status mr_server_submit(mr_server* server, const mr_scene* scene, const mr_render_settings* render,
                           const mr_integrator_settings* integrator, uint64_t* job);
/* Pause/resume take effect at the next wave; `accepted` as RenderSession::pause/resume. */
mr_status mr_server_pause(mr_server* server, uint64_t job, int* accepted);
mr_status mr_server_resume(mr_server* server, uint64_t job, int* accepted);
mr_status mr_server_cancel(mr_server* server, uint64_t job);
/* Waits up to `milliseconds` for the job to complete, fail or be cancelled. */
mr_status mr_server_wait(mr_server* server, uint64_t job, uint32_t milliseconds, int* finished);
mr_status mr_server_job_info(mr_server* server, uint64_t job, mr_job_info* info);
/* The completed image (capacity in floats); MR_OUT_OF_RANGE unless the job completed. */
mr_status mr_server_result(mr_server* server, uint64_t job, float* rgb, size_t capacity);
/* Progressive image of the samples issued so far (mean per pixel); `samples` receives the
 * sample passes every pixel has. */
mr_status mr_server_preview(mr_server* server, uint64_t job, float* rgb, size_t capacity,
                            uint64_t* samples);
/* Forgets a finished job and its host image. */
mr_status mr_server_release(mr_server* server, uint64_t job);
mr_status mr_server_get_statistics(mr_server* server, mr_server_statistics* statistics);

#ifdef __cplusplus
}
#endif

#endif /* MINIRENDER_B200_H */
