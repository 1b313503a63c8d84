/*
 * gpt_b200.h — C ABI of the B200 wavefront path tracer.
 *
 * Drop-in boundary for KrzystekMatej/gpu-path-tracer's CUDA renderer
 * (Core::Graphics::Cuda::Renderer, Core/Include/Core/Graphics/Cuda/PathTracing/Renderer.hpp:42-189)
 * and its kernel launchers (Core/Include/Core/Graphics/Cuda/PathTracing/Kernels/Launchers.hpp:20-145).
 * Plain C types only: opaque handles, raw pointers, sizes. Every call returns an int
 * status (GPT_OK = 0); no exception crosses the boundary. The message of the last
 * failure is kept per renderer (gpt_peek_last_error / gpt_consume_last_error), as the
 * reference keeps m_LastError (Renderer.cpp:453-459, 308-320).
 */
#ifndef GPT_B200_H
#define GPT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define GPT_OK 0
#define GPT_ERR_INVALID_ARGUMENT 1
#define GPT_ERR_CUDA 2
#define GPT_ERR_OUT_OF_MEMORY 3
#define GPT_ERR_STATE 4          /* e.g. "Renderer is already rendering" (Renderer.cpp:347-348) */
#define GPT_ERR_NO_SCENE 5
#define GPT_ERR_CAPACITY 6       /* a size above a documented limit */
#define GPT_ERR_TIMEOUT 7        /* a bounded device wait ran out */
#define GPT_ERR_DEVICE_FAULT 8   /* a kernel reported an internal error flag */

/* GlobalShadingModel (Core/Include/Core/Graphics/Cuda/PathTracing/Material.hpp:8-17). */
enum gpt_shading_model {
    GPT_MODEL_NORMAL = 0,
    GPT_MODEL_DIFFUSE = 1,
    GPT_MODEL_MIRROR = 2,
    GPT_MODEL_PHONG = 3,
    GPT_MODEL_GGX = 4,
    GPT_MODEL_EMISSIVE = 5,
    GPT_MODEL_COUNT = 6
};

/*
 * Constant material: the values the reference's 1x1 material textures return
 * (Material.hpp:73-87; Manager.cpp:321-380 encodes MTL constants into those texels).
 * 80 bytes.
 */
typedef struct gpt_material {
    uint32_t model;        /* gpt_shading_model */
    float color[3];        /* albedo / base colour, linear */
    float specular[3];     /* Phong specular / mirror reflectance, linear */
    float shininess;       /* normalised shininess texel t in [0,1]; exponent = t*999+1 (MaterialEval.cu:405-408) */
    float rma[3];          /* roughness, metallic, ambient occlusion */
    float emission[3];     /* radiance of emissive triangles */
    float normal[3];       /* tangent-space normal-map texel in [0,1]; (128,128,255)/255 is the default map */
    float ior;
    float transmission;
    float reserved;
} gpt_material;

/*
 * Image texture of a material slot (Texture::Create2D, Core/Source/Graphics/Cuda/Resources/Texture.cpp:65-189):
 * sampled with normalised coordinates, clamp addressing and bilinear filtering; u8 texels are read as
 * normalised floats, with hardware sRGB decode for GPT_TEXEL_U8_SRGB; 3-channel images are expanded
 * to 4 channels (alpha 255 / 1.0). Rows are stored top row first, width * channels texels each.
 */
enum gpt_texel_format { GPT_TEXEL_U8_SRGB = 0, GPT_TEXEL_U8_LINEAR = 1, GPT_TEXEL_F32 = 2 };
typedef struct gpt_texture_desc {
    uint32_t width;
    uint32_t height;
    uint32_t channels;            /* 1, 3 or 4 */
    uint32_t format;              /* gpt_texel_format */
    const void* data;
} gpt_texture_desc;

/* Texture slots of a material (Material.hpp:73-87). */
enum gpt_texture_slot {
    GPT_TEX_COLOR = 0, GPT_TEX_SPECULAR = 1, GPT_TEX_SHININESS = 2, GPT_TEX_RMA = 3, GPT_TEX_EMISSION = 4,
    GPT_TEX_NORMAL = 5, GPT_TEX_SLOTS = 6
};

/*
 * Scene upload, replacing InitializeSceneBuffers(entt::registry, Assets::Storage)
 * (Renderer.hpp:115, Renderer.cpp:292-306). The arrays are the output of the
 * reference's BuildTriangles (Renderer.cpp:159-213): world-space per-triangle
 * vertex data, already transformed. All pointers are host memory.
 */
typedef struct gpt_scene_desc {
    uint32_t triangle_count;       /* at most 2^24 (16,777,216) */
    const float* positions;       /* [T][3][3] world positions */
    const float* normals;         /* [T][3][3] world normals */
    const float* tangents;        /* [T][3][4] world tangent xyz + handedness sign */
    const float* uvs;             /* [T][3][2] */
    const uint32_t* material_ids; /* [T] index into materials */
    uint32_t material_count;
    const gpt_material* materials;
    uint32_t texture_count;       /* optional image textures (0 = constant materials only) */
    const gpt_texture_desc* textures;
    const int32_t* material_textures; /* [material_count][GPT_TEX_SLOTS] texture index, -1 = the material's constant */
} gpt_scene_desc;

/* DeviceCamera (Core/Include/Core/Graphics/Cuda/PathTracing/DeviceCamera.hpp:5-11). */
typedef struct gpt_device_camera {
    float origin[3];
    float lower_left[3];
    float horizontal[3];
    float vertical[3];
} gpt_device_camera;

/* Capture::MotionState (Core/Include/Core/Capture/Sample.hpp:6-10): position, quaternion (w, x, y, z). */
typedef struct gpt_motion_state {
    float position[3];
    float rotation[4];
} gpt_motion_state;

/* Capture::MotionSample (Core/Include/Core/Capture/Sample.hpp:12-16): a recorded state and its time (s). */
typedef struct gpt_motion_sample {
    gpt_motion_state state;
    float time;
} gpt_motion_sample;

/* Per-frame settings of StartSimulation (Renderer.cpp:330-376) plus B200 tuning knobs. */
typedef struct gpt_render_settings {
    uint32_t width;
    uint32_t height;
    uint32_t samples_per_pixel;   /* rounded down to a square, as Renderer.cpp:366-367 */
    uint32_t path_depth;          /* clamped to [1, 100] (PathTracerDefaults.hpp:15-17) */
    uint32_t use_nee;             /* next-event estimation */
    uint32_t pool_size;           /* path slots; 0 = 1,048,576 (PathTracerDefaults.hpp:9) */
    uint64_t max_samples;         /* 0 = the whole frame; else render only sample indices [0, max_samples) */
    uint32_t trace_block;         /* 0 = default threads per block of the traversal kernels (64 or 128) */
    uint32_t trace_refill;        /* idle lanes a traversal warp waits for before fetching new rays: bits 0-7 for
                                     closest-hit rays (0 = 16), bits 8-15 for shadow rays (0 = half the former) */
    uint64_t rng_offset;          /* added to every sample index to form its Philox subsequence (0 = the reference's streams) */
    uint32_t loop_mode;           /* GPT_LOOP_GRAPH (default): the whole frame is one CUDA graph whose conditional WHILE
                                     node repeats the iteration on the device; GPT_LOOP_HOST: the host launches each
                                     iteration and reads the loop condition after it (the reference's structure) */
    uint32_t trace_occupancy;     /* traversal kernel variant: 0/1 = registers unconstrained, 10 or 12 = that many
                                     resident 128-thread blocks per SM targeted (fewer registers, more warps) */
    uint32_t bvh_format;          /* GPT_BVH8_Q8 (default): 8-wide BVH, 8-bit quantised child boxes, 128-B nodes;
                                     GPT_BVH2_FP32: the binary BVH it is collapsed from, FP32 child boxes, 64-B nodes,
                                     local-memory stack (the plain format; same hits, bit for bit) */
    uint32_t wavefront_layout;    /* GPT_WAVEFRONT_B200 (default): finished slots are regenerated from a bitmap in
                                     slot order and the per-model shading kernels run side by side;
                                     GPT_WAVEFRONT_QUEUES: the reference's structure, a queue of finished slots in the
                                     order paths ended (RegenQueue, PathGeneration.cu:74-102) and the shading kernels
                                     one after another (Renderer.cpp:540-566). Same results, bit for bit. */
    uint32_t rng_policy;          /* GPT_RNG_PHILOX (default): the reference's streams, cuRAND Philox4_32_10 with seed
                                     1234 and subsequence = sample index (PathData.hpp:37-73); GPT_RNG_PCG32: one PCG32
                                     stream per sample, seeded by a hash of (seed, pixel, sample) */
    uint32_t light_sampling;      /* GPT_LIGHTS_AREA (default): NEE picks an emitter with probability proportional to
                                     its area, the reference's light sampler (LightSampler.cpp:16-19); GPT_LIGHTS_POWER:
                                     proportional to area x luminance of its emission (the production mode; the alias
                                     table is built from an FP64 prefix sum by a parallel split on the device) */
    uint32_t max_iterations;      /* 0 = the automatic bound of the device loop, depth x (ceil(samples / pool) + 2) + 64;
                                     else at most this many wavefront iterations: a frame that still has paths in flight
                                     then ends with GPT_ERR_DEVICE_FAULT (the loop's bounded wait running out) */
    uint32_t trace_stack;         /* 0 = traversal stack sized to the BVH8 depth; else at most this many entries (1-64)
                                     per ray: a stack shallower than the tree can overflow, and a ray that would push
                                     beyond it stops traversing and the frame ends with GPT_ERR_DEVICE_FAULT */
} gpt_render_settings;

#define GPT_LOOP_GRAPH 0u
#define GPT_LOOP_HOST 1u
#define GPT_BVH8_Q8 0u
#define GPT_BVH2_FP32 1u
#define GPT_WAVEFRONT_B200 0u
#define GPT_WAVEFRONT_QUEUES 1u
#define GPT_RNG_PHILOX 0u
#define GPT_RNG_PCG32 1u
#define GPT_LIGHTS_AREA 0u
#define GPT_LIGHTS_POWER 1u

typedef struct gpt_frame_stats {
    uint32_t iterations;          /* wavefront iterations (Renderer.cpp:517-623) */
    uint32_t kernel_launches;     /* kernels the frame graph launched */
    uint64_t samples;             /* paths rendered */
    uint64_t rays;                /* extension + camera rays traced (closest hit) */
    uint64_t shadow_rays;         /* NEE shadow rays traced (any hit) */
    uint64_t node_visits[2];      /* BVH nodes visited (of the frame's bvh_format): [0] closest-hit, [1] shadow traversal */
    uint64_t triangle_tests[2];   /* triangles tested:   [0] closest-hit, [1] shadow traversal */
    float device_ms;              /* CUDA-event time of the frame graph on the render stream */
    float phase_ms[4];            /* device time per phase, summed over iterations: closest-hit traversal,
                                     shading (all models), shadow traversal, regeneration */
    float trace_event_ms;         /* GPT_LOOP_HOST only: CUDA-event time of the closest-hit traversal launches */
} gpt_frame_stats;

typedef struct gpt_renderer gpt_renderer;

const char* gpt_status_string(int status);

/* Renderer lifetime; device = CUDA ordinal. Renderer() / ~Renderer() (Renderer.hpp:105-106). */
int gpt_create(gpt_renderer** out, int device);
void gpt_destroy(gpt_renderer* renderer);

/* Renderer::InitializeRenderingBuffers (Renderer.hpp:114, Renderer.cpp:265-290). */
int gpt_init_rendering_buffers(gpt_renderer* renderer, uint32_t width, uint32_t height);
/* Renderer::InitializeSceneBuffers (Renderer.hpp:115, Renderer.cpp:292-306). */
int gpt_init_scene_buffers(gpt_renderer* renderer, const gpt_scene_desc* scene);
/* Renderer::Clear (Renderer.hpp:117, Renderer.cpp:322-328, 677-687). */
int gpt_clear(gpt_renderer* renderer, uint8_t r, uint8_t g, uint8_t b, uint8_t a);

/*
 * Renderer::StartSimulation (Renderer.hpp:118-126, Renderer.cpp:330-399): renders one frame per
 * motion state on a worker thread. fov_y in radians (Graphics::Ecs::Camera::fovY). When
 * output_folder is not NULL each finished frame is written as frame_NNNN.png there
 * (Renderer.cpp:645-675), flipped vertically like the reference.
 */
int gpt_start_simulation(gpt_renderer* renderer, uint32_t width, uint32_t height, float fov_y,
                         const gpt_motion_state* motion_states, uint32_t motion_state_count,
                         uint32_t samples_per_pixel, uint32_t path_depth, const char* output_folder, int use_nee);
/* Renderer::ResumeSimulation (Renderer.hpp:127, Renderer.cpp:401-427). */
int gpt_resume_simulation(gpt_renderer* renderer, uint32_t start_frame);
/* Renderer::StopRendering (Renderer.hpp:128, Renderer.cpp:429-440). */
int gpt_stop_rendering(gpt_renderer* renderer);
/* Progress getters (Renderer.hpp:131-140). */
int gpt_is_rendering(const gpt_renderer* renderer);
uint32_t gpt_get_done_frames(const gpt_renderer* renderer);
uint32_t gpt_get_total_frames(const gpt_renderer* renderer);
uint64_t gpt_get_done_samples(const gpt_renderer* renderer);
uint64_t gpt_get_total_samples(const gpt_renderer* renderer);
uint32_t gpt_get_width(const gpt_renderer* renderer);
uint32_t gpt_get_height(const gpt_renderer* renderer);

/* GetFrameView().Lock() (Renderer.hpp:45-103,130): the host RGBA8 frame, held until unlock. */
int gpt_lock_frame(gpt_renderer* renderer, const uint32_t** data, size_t* size, size_t* element_size);
int gpt_unlock_frame(gpt_renderer* renderer);

/* PeekLastError / ConsumeLastError (Renderer.hpp:142-143). Writes a NUL-terminated message; returns
 * 1 when an error was present, 0 otherwise. */
int gpt_peek_last_error(const gpt_renderer* renderer, char* buffer, size_t length);
int gpt_consume_last_error(gpt_renderer* renderer, char* buffer, size_t length);

/*
 * One frame, synchronously, on the calling thread: Renderer::RenderFrame (Renderer.cpp:468-647)
 * without the worker thread or PNG output. The frame runs as one CUDA graph (device-driven
 * wavefront loop, no host synchronisation per iteration). Results stay on the device until read.
 */
int gpt_render_frame(gpt_renderer* renderer, const gpt_device_camera* camera,
                     const gpt_render_settings* settings, gpt_frame_stats* stats);
/*
 * Autotuner: measures the frame's tuning knobs (pool_size = path slots and queue capacities,
 * trace_occupancy, trace_refill, trace_block) on reduced frames of the same workload (whole
 * image; per pool candidate, the smallest square spp of at least 4, and at most the frame's spp,
 * that holds two pool-fulls of samples) and writes the combination with the lowest device time
 * per sample into *best (the other fields copied from *base); *best_ms is that time scaled to the
 * full frame. Results of a frame do not depend on these knobs, only its speed.
 * No counterpart in the reference, whose launch shapes are compile-time constants
 * (Kernels/LaunchUtils.cuh:7-17, PathTracerDefaults.hpp:9).
 */
int gpt_autotune(gpt_renderer* renderer, const gpt_device_camera* camera, const gpt_render_settings* base,
                 gpt_render_settings* best, float* best_ms, uint32_t* candidates);

/* Copies of the last frame's results to host memory. */
int gpt_read_framebuffer(gpt_renderer* renderer, uint32_t* rgba, size_t pixel_count);
int gpt_read_accumulation(gpt_renderer* renderer, float* rgba32f, size_t pixel_count);
/* Per-sample (per-path) radiance of the last frame, [samples][3], in sample-index order. */
int gpt_read_sample_radiance(gpt_renderer* renderer, float* rgb, uint64_t sample_count);
/* The last frame's float4 accumulation into a device buffer of the same GPU (for a collective across
 * ranks without a round trip through host memory). stream NULL: the renderer's stream, synchronised
 * before returning; else the copy is queued on `stream` after the frame (gpt_render_frame returns
 * only after its frame has finished). */
int gpt_copy_accumulation_device(gpt_renderer* renderer, float* device_rgba32f, size_t pixel_count, void* stream);
/* The last frame's FP64 reference accumulation: per pixel, its samples' radiance summed in FP64 on
 * the device in sample order, [pixels][3] doubles, for measuring the FP32 Kahan accumulation against
 * it. No counterpart in the reference, which accumulates with float atomics (Common.hpp:8-16). */
int gpt_read_accumulation_fp64(gpt_renderer* renderer, double* rgb64, size_t pixel_count);
/* Per-iteration queue sizes of the last frame: rows of 9 words (rays, 6 material queues,
 * shadow rays, regenerated/terminated paths), as the reference's queues hold them. */
int gpt_read_queue_log(gpt_renderer* renderer, uint32_t* rows, uint32_t max_rows, uint32_t* row_count);

/*
 * Ray-batch traversal on the current scene (Kernels::IntersectRaysWithScene and
 * Kernels::IntersectShadowRaysWithScene, Launchers.hpp:60-80 / Intersect.cu:216-295, with the
 * queue plumbing replaced by plain arrays). Device pointers; stream may be NULL (the renderer's
 * stream). rays: [n][8] float = origin xyz, direction xyz, tMin, tMax.
 * Closest: tri_out [n] = original triangle index or 0xFFFFFFFF; uvt_out [n][3] = u, v, t.
 * Any: occluded_out [n] = 1 if any triangle hits with tMin <= t < tMax.
 */
int gpt_intersect_closest(gpt_renderer* renderer, const float* rays, uint32_t n, uint32_t* tri_out,
                          float* uvt_out, void* stream);
int gpt_intersect_any(gpt_renderer* renderer, const float* rays, uint32_t n, uint8_t* occluded_out,
                      void* stream);

/* The same queries against the binary FP32 BVH of the scene (the plain format; GPT_BVH2_FP32).
 * They return the same triangles, (u, v, t) and occlusion bits as the BVH8 queries. */
int gpt_intersect_closest_binary(gpt_renderer* renderer, const float* rays, uint32_t n, uint32_t* tri_out,
                                 float* uvt_out, void* stream);
int gpt_intersect_any_binary(gpt_renderer* renderer, const float* rays, uint32_t n, uint8_t* occluded_out,
                             void* stream);

/* Scene statistics after upload: BVH8 node count, tree depth, light count, triangle count. */
int gpt_scene_info(const gpt_renderer* renderer, uint32_t* node_count, uint32_t* depth, uint32_t* light_count,
                   uint32_t* triangle_count);
/* Node count and depth of the scene's binary FP32 BVH (HostBvh.cpp:22-100 builds the reference's
 * binary tree by median splits; this one is the binned-SAH tree the BVH8 is collapsed from). */
int gpt_scene_info_binary(const gpt_renderer* renderer, uint32_t* node_count, uint32_t* depth);
/* Wall-clock seconds of the last scene upload: the BVH build (on the host: binned SAH, 8-wide
 * collapse, quantisation on all host threads; or on the device, gpt_set_bvh_build) and the whole
 * gpt_init_scene_buffers call, which adds validation,
 * textures, host-to-device copies and the device-built shading records, lights and alias tables
 * (Renderer.cpp:292-306 is the reference's upload; it reports no timings). */
int gpt_scene_upload_times(const gpt_renderer* renderer, double* bvh_build_seconds, double* upload_seconds);

/* Where the next gpt_init_scene_buffers builds the BVH8 (the reference builds it on the host,
 * HostBvh.cpp, with median splits). GPT_BVH_BUILD_HOST (default): binned SAH on all host threads,
 * plus the binary FP32 BVH of GPT_BVH2_FP32. GPT_BVH_BUILD_DEVICE: on the GPU (Morton order,
 * clustering of nearest neighbours, the same 8-wide collapse and quantisation), no binary BVH (frames
 * with GPT_BVH2_FP32 are refused). Hits, and so frames, do not depend on the builder; traversal work
 * does. */
#define GPT_BVH_BUILD_HOST 0u
#define GPT_BVH_BUILD_DEVICE 1u
int gpt_set_bvh_build(gpt_renderer* renderer, uint32_t build);
/* Structural check of the uploaded BVH8 against the scene's positions ([n][3][3], the ones uploaded),
 * on the host: quantised child boxes not containing their subtree (exact arithmetic), triangles not
 * referenced exactly once, and triangles in leaves. */
int gpt_check_bvh(gpt_renderer* renderer, const float* positions, uint32_t triangle_count, uint64_t* containment_violations,
                  uint64_t* triangles_not_exactly_once, uint64_t* leaf_triangles);
/* The light alias table built on the device, [lights][4] words (q, p, alias, value)
 * (AliasTableView.hpp:8-14). */
int gpt_read_alias_table(gpt_renderer* renderer, uint32_t* bins, uint32_t count);
/* The power-weighted alias table of GPT_LIGHTS_POWER (area x emission luminance, FP64 prefix sums,
 * parallel split on the device), same layout. No counterpart in the reference, whose light sampler
 * weights by area only (LightSampler.cpp:16-19). */
int gpt_read_alias_table_power(gpt_renderer* renderer, uint32_t* bins, uint32_t count);

/*
 * Fault-injection hook for tests of the error paths (no counterpart in the reference): the
 * after-th device allocation made by this library from now on (1 = the next one) fails as if the
 * device were out of memory, on the host, before cudaMalloc is called; 0 disarms. Calls that fail
 * this way return GPT_ERR_OUT_OF_MEMORY and leave the renderer or server as it was before the call.
 */
int gpt_inject_allocation_failure(uint32_t after);

/*
 * Host-side validation of the BVH builder (no device work): builds the wide BVH and the binary FP32
 * BVH for a scene and checks in exact arithmetic that every quantised BVH8 child box and every
 * binary child box contains its subtree, and that every triangle sits in exactly one leaf of each
 * tree (violations and misplaced triangles of both trees are summed). Replaces nothing in the
 * reference; it pins the structural guarantee behind HostBvh.cpp:37-48's padded bounds.
 */
int gpt_bvh8_check(const gpt_scene_desc* scene, uint32_t* node_count, uint32_t* depth,
                   uint64_t* containment_violations, uint64_t* misplaced_triangles);

/*
 * Allocation-free alias-table build. This entry point has no counterpart in the reference; it
 * exists for callers that must not allocate device memory when they build a light sampler
 * (a fixed per-frame memory budget, an engine that owns every allocation through its own pool,
 * or code that cannot afford cudaMalloc/cudaFree stalls, since cudaFree synchronises the device).
 * It builds the same table as the scene upload (AliasTable.hpp:22-84 semantics: FP64 sum of the
 * weights, p = w / sum, the reference's sequential pairing) from light_count float weights into
 * bins ([light_count][4] uint32 = q, p, alias, value). Both pointers are device memory; bins must be
 * 16-byte aligned and weights 4-byte aligned (GPT_ERR_INVALID_ARGUMENT otherwise). The weights must
 * be finite and non-negative with a positive sum; other weights give NaN or infinite entries.
 * light_count 0 returns GPT_OK and touches nothing. stream may be NULL (the legacy default
 * stream); the call is asynchronous on it.
 * Working memory is a fixed array of about 2 MiB compiled into the library, held by every GPU that
 * loads it until the process exits; light_count above GPT_NOALLOC_MAX_LIGHTS returns
 * GPT_ERR_CAPACITY. The first call on a device looks up that array's device address (set-up),
 * so make the first call before any stream capture; that address is kept for the process, so a
 * device reset (cudaDeviceReset) after the first call is not supported. All calls share the
 * array: calls that can overlap on the GPU race and must be ordered by the caller.
 */
#define GPT_NOALLOC_MAX_LIGHTS 65536u
int gpt_build_alias_table_noalloc(const float* weights, uint32_t light_count, uint32_t* bins, void* stream);

/*
 * Per-vertex tangents of an indexed triangle mesh by Mikkelsen's method, the tangent space the
 * reference generates for imported meshes (GenerateTangentSpace, Core/Source/Utils/Math/TangentSpace.cpp:
 * 66-89, MikkTSpace with its default 180-degree threshold): positions [V][3], normals [V][3] (unit),
 * uvs [V][2], indices [T][3]; tangents [V][4] = unit tangent xyz and handedness sign (+1 where the uv
 * mapping preserves orientation). A vertex takes the frame of the last triangle corner naming it.
 */
int gpt_generate_tangents(const float* positions, const float* normals, const float* uvs, uint32_t vertex_count,
                          const uint32_t* indices, uint32_t triangle_count, float* tangents);

/*
 * Headless OBJ/MTL ingest (the reference's LoadObj + GenerateTangentSpace + Manager::ImportMaterial +
 * BuildTriangles: Core/Source/Import/ObjLoader.cpp:67-234, Core/Source/Assets/Manager.cpp:311-412,
 * Renderer.cpp:116-213). Produces the arrays of a gpt_scene_desc: triangles grouped per shape and
 * material, vertex normals and uvs required, tangents from uv derivatives, constant materials
 * encoded as the reference's texels. transform: optional column-major 4x4 world matrix (NULL =
 * identity). The scene object owns the arrays gpt_obj_scene_desc points into.
 */
typedef struct gpt_obj_scene gpt_obj_scene;
int gpt_obj_load(const char* path, const float* transform, gpt_obj_scene** out);
int gpt_obj_scene_desc(const gpt_obj_scene* scene, gpt_scene_desc* desc);
int gpt_obj_material_name(const gpt_obj_scene* scene, uint32_t index, char* buffer, size_t length);
void gpt_obj_free(gpt_obj_scene* scene);

/*
 * Job server: continuous batching of render jobs over device-resident scenes. The reference renders
 * one job at a time through Renderer (RenderFrame per camera, Renderer.cpp:401-647); the server keeps
 * several scenes resident (gpt_server_add_scene), admits submitted jobs while others run, as long as
 * a job-table entry and the HBM budget allow, and traces the paths of all admitted jobs together in
 * one device loop (one CUDA graph per scheduling slice). Every job renders progressively in passes of
 * one sample per pixel; its image equals the one gpt_render_frame produces for the same scene,
 * camera and settings, bit for bit, alone or mixed with other jobs.
 *
 * Admission accounting per job: 64 bytes per path the job may have in flight (min(ring passes x
 * pixels, pool)) plus its framebuffers (pass ring 12 B, Kahan accumulator 32 B, RGBA8 4 B per
 * pixel and pass). Jobs are admitted in submission order; a job larger than the whole budget is
 * refused at submission with GPT_ERR_CAPACITY. Among admitted jobs, idle path slots go to short
 * jobs first, then to the others in submission order (or as gpt_server_config.schedule says); the
 * order changes which job finishes first, never an image. All gpt_server_* calls are thread-safe.
 */
typedef struct gpt_server gpt_server;

typedef struct gpt_server_config {
    uint32_t pool_size;            /* path slots shared by all jobs, <= 2^24 (0 = 4,194,304) */
    uint32_t max_jobs;             /* job-table entries: jobs admitted at the same time (0 = 256) */
    uint32_t max_active_jobs;      /* 0 = as many as fit; 1 = one job at a time (the plain loop) */
    uint32_t ring_passes;          /* pass buffers per job, <= 256 (0 = chosen from pool and image size) */
    uint64_t hbm_budget_bytes;     /* admission budget (0 = 16 GiB); also the size of the job arena */
    uint32_t trace_block;          /* traversal tuning, as in gpt_render_settings (0 = defaults) */
    uint32_t trace_refill;
    uint32_t trace_occupancy;
    uint32_t max_slice_iterations; /* wavefront iterations per graph launch at most (0 = 4096) */
    uint32_t schedule;             /* which active job gets idle path slots first: 0/GPT_SCHEDULE_TWO_CLASS = jobs whose
                                      render time alone (samples / the server's measured paths per second) is below
                                      short_job_seconds first, fewest samples left first, then the other jobs in
                                      submission order; GPT_SCHEDULE_SHORTEST_FIRST = the job with the fewest samples
                                      left; GPT_SCHEDULE_OLDEST_FIRST = submission order;
                                      GPT_SCHEDULE_DEADLINE = the earliest deadline, submit time + deadline_slowdown x the
                                      job's samples / the server's measured paths per second (small jobs still go
                                      first, and a large job is not passed over past its deadline) */
    float deadline_slowdown;       /* GPT_SCHEDULE_DEADLINE: deadline in units of the job's own render time (0 = 4) */
    float short_job_seconds;       /* GPT_SCHEDULE_TWO_CLASS: render time alone below which a job is short (0 = 0.05) */
    uint32_t bvh_build;            /* where gpt_server_add_scene builds a scene's BVH8: GPT_BVH_BUILD_HOST (0) or
                                      GPT_BVH_BUILD_DEVICE (see gpt_set_bvh_build) */
} gpt_server_config;

#define GPT_SCHEDULE_SHORTEST_FIRST 1u
#define GPT_SCHEDULE_OLDEST_FIRST 2u
#define GPT_SCHEDULE_DEADLINE 3u
#define GPT_SCHEDULE_TWO_CLASS 4u

typedef struct gpt_job_desc {
    uint32_t scene;                /* id from gpt_server_add_scene */
    uint32_t width, height;
    uint32_t samples_per_pixel;    /* rounded down to a square, as StartSimulation does */
    uint32_t path_depth;
    uint32_t use_nee;
    uint64_t rng_offset;           /* added to the sample index to form the Philox subsequence */
    gpt_device_camera camera;
    uint32_t keep_accumulation;    /* nonzero: keep the float4 accumulation for gpt_server_read */
    uint32_t rng_policy;           /* GPT_RNG_PHILOX (default) or GPT_RNG_PCG32, as in gpt_render_settings */
    uint32_t light_sampling;       /* GPT_LIGHTS_AREA (default) or GPT_LIGHTS_POWER, as in gpt_render_settings */
    uint32_t reserved;
} gpt_job_desc;

#define GPT_JOB_QUEUED 0
#define GPT_JOB_RUNNING 1
#define GPT_JOB_DONE 2
#define GPT_JOB_CANCELLED 3
#define GPT_JOB_FAILED 4

typedef struct gpt_job_status {
    uint32_t state;                /* GPT_JOB_* */
    uint32_t passes_done;          /* samples per pixel folded into the image so far */
    uint32_t passes_total;
    uint32_t reserved;
    uint64_t samples_total;
    uint64_t admitted_bytes;
    double submit_s, admit_s, done_s; /* seconds since gpt_server_create; -1 = not yet */
} gpt_job_status;

typedef struct gpt_server_stats {
    uint64_t slices;               /* graph launches */
    uint64_t iterations;           /* wavefront iterations */
    uint64_t samples;              /* samples (paths) launched */
    uint64_t rays, shadow_rays;
    uint64_t admitted_bytes, admitted_high_water, budget_bytes;
    uint32_t active_jobs, queued_jobs, completed_jobs, scenes;
    double device_ms;              /* sum of the slices' device times */
    float phase_ms[4];             /* as gpt_frame_stats.phase_ms, summed over all slices */
} gpt_server_stats;

int gpt_server_create(gpt_server** out, int device, const gpt_server_config* config);
int gpt_server_destroy(gpt_server* server);
/* Only while no job is queued or running. */
int gpt_server_add_scene(gpt_server* server, const gpt_scene_desc* scene, uint32_t* scene_id);
int gpt_server_submit(gpt_server* server, const gpt_job_desc* job, uint64_t* job_id);
int gpt_server_poll(gpt_server* server, uint64_t job_id, gpt_job_status* status);
/* GPT_OK once the job is done, cancelled or failed; GPT_ERR_TIMEOUT after timeout_s seconds. */
int gpt_server_wait(gpt_server* server, uint64_t job_id, double timeout_s);
/* After GPT_JOB_DONE: rgba [height][width] uint32; accumulation [height][width][4] float or NULL. */
int gpt_server_read(gpt_server* server, uint64_t job_id, uint32_t* rgba, float* accumulation);
/* Forgets a finished job (its host copy of the image). */
int gpt_server_release(gpt_server* server, uint64_t job_id);
/* A queued job is dropped; a running one launches no more samples and ends as GPT_JOB_CANCELLED
 * (without an image) once its paths in flight finish. */
int gpt_server_cancel(gpt_server* server, uint64_t job_id);
/* How the server runs a slice: GPT_LOOP_GRAPH (default) as one CUDA graph whose conditional WHILE node
 * repeats the engine iteration on the device, GPT_LOOP_HOST as one launch per kernel with the loop
 * condition read on the host after every iteration (slower; for profilers, which do not profile kernel
 * nodes of graphs with conditional nodes). Takes effect from the next slice; results do not change.
 * No counterpart in the reference, which has no job server. */
int gpt_server_set_loop_mode(gpt_server* server, uint32_t mode);
int gpt_server_get_stats(gpt_server* server, gpt_server_stats* stats);
int gpt_server_peek_last_error(gpt_server* server, char* buffer, size_t length);

/* sizeof() of the public structs as compiled into this library, in the order gpt_material,
 * gpt_scene_desc, gpt_device_camera, gpt_motion_state, gpt_render_settings, gpt_frame_stats,
 * gpt_texture_desc, gpt_server_config, gpt_job_desc, gpt_job_status, gpt_server_stats,
 * gpt_motion_sample (for binding checks from other languages). */
int gpt_abi_struct_sizes(uint32_t* sizes, uint32_t count);

/* DeviceCamera from fov_y (radians), aspect and a motion state: MakeDeviceCamera (Renderer.cpp:237-257). */
int gpt_make_device_camera(float fov_y, float aspect, const gpt_motion_state* state, gpt_device_camera* out);

/*
 * Capture::ResampleMotion (Core/Source/Capture/Resampling.cpp:17-55): a recorded camera path (samples
 * at strictly increasing times) to one state per frame at a fixed interval from the first sample's
 * time: position linearly interpolated, rotation by spherical linear interpolation along the shorter
 * arc and renormalised (Utils/Math/Interpolation.hpp SlerpShortest). The states feed
 * gpt_start_simulation. *state_count receives the number of states; if it exceeds capacity nothing
 * is written and GPT_ERR_CAPACITY is returned. interval <= 0 or times that do not increase:
 * GPT_ERR_INVALID_ARGUMENT. No samples give no states; one sample gives its own state.
 */
int gpt_resample_motion(const gpt_motion_sample* samples, uint32_t sample_count, float interval,
                        gpt_motion_state* states, uint32_t capacity, uint32_t* state_count);

#ifdef __cplusplus
}
#endif

#endif /* GPT_B200_H */
