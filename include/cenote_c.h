/*
 * cenote_c.h — the C ABI of the B200 wavefront path tracer.
 *
 * This is the boundary a host (the reference's Rust crate through a bindgen'd
 * `cenote-sys`, the C++ CLI, or Python through ctypes) binds. It replaces the
 * `cenote` crate's scene/renderer API:
 *
 *   Scene::new(&Context, &[Object], Camera, &Environment)   crates/cenote/src/scene/mod.rs:254
 *   Renderer::with_max_bounces(&Context, u32)               crates/cenote/src/render/mod.rs:151
 *   Renderer::render(&self, &Context, &Scene, w, h)         crates/cenote/src/render/mod.rs:209
 *   Renderer::accumulate(&self, &Context, &Scene, &mut Film) crates/cenote/src/render/mod.rs:245
 *   Film::{new, reset, samples, averages}                   crates/cenote/src/render/film.rs:102-217
 *   Wavefront::trace(&Context, &Scene, &Buffer, w, h, sample) crates/cenote/src/wavefront.rs:568
 *   LightSampling {Mis, BsdfOnly, NeeOnly}                  crates/cenote/src/wavefront.rs (LIGHT_SAMPLING_* in shaders/lights.slang:32-34)
 *
 * Conventions (bindgen-friendly): opaque handles, POD structs, every call
 * returns an int32_t status (0 ok, negative = cenote error). A caller bug that
 * the reference catches with `assert!` (zero-sized target, bounce cap outside
 * 1..=255, empty scene, non-invertible transform) returns
 * CENOTE_E_INVALID_ARGUMENT instead of aborting. cenote_last_error() returns
 * the calling thread's last message. Output buffers are caller-owned host
 * memory unless a name says "device". A handle is not thread-safe by itself;
 * every handle created from one context shares that context's CUDA stream.
 */
#ifndef CENOTE_C_H
#define CENOTE_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, mirroring cenote::Error (crates/cenote/src/error.rs:10-72). */
#define CENOTE_OK 0
#define CENOTE_E_INVALID_ARGUMENT (-1)
#define CENOTE_E_DEVICE (-2)        /* CUDA runtime error (the reference's Error::Vulkan) */
#define CENOTE_E_NO_CAPABLE_GPU (-3) /* Error::NoCapableGpu */
#define CENOTE_E_ALLOCATION (-4)    /* Error::Allocation */
#define CENOTE_E_SCENE (-5)         /* Error::Scene */
#define CENOTE_E_TIMEOUT (-6)       /* a bounded device wait gave up */
#define CENOTE_E_OVERFLOW (-7)      /* a device-side bound (stack, queue) was exceeded */
#define CENOTE_E_BUDGET (-8)        /* a job does not fit the server's HBM budget */

/* LightSampling (wavefront.rs; LIGHT_SAMPLING_* in shaders/lights.slang:32-34). */
#define CENOTE_LIGHT_SAMPLING_MIS 0u
#define CENOTE_LIGHT_SAMPLING_BSDF 1u
#define CENOTE_LIGHT_SAMPLING_NEE 2u

/* "No texture" in a material's texture slots (material.rs TEXTURE_NONE). */
#define CENOTE_TEXTURE_NONE 0xffffffffu

/* Delta-light kinds (lights.rs KIND_*). */
#define CENOTE_LIGHT_DISTANT 1u
#define CENOTE_LIGHT_POINT 2u

typedef struct cenote_context cenote_context;
typedef struct cenote_scene cenote_scene;
typedef struct cenote_renderer cenote_renderer;
typedef struct cenote_film cenote_film;

/* The 144-byte OpenPBR record, field for field crates/cenote/src/material.rs:28-109. */
typedef struct cenote_material {
    float base_color[3];
    float base_roughness;
    float emission[3];
    float metalness;
    float specular_weight;
    float specular_roughness;
    float specular_ior;
    float transmission_weight;
    float transmission_color[3];
    float transmission_depth;
    float coat_color[3];
    float coat_weight;
    float coat_roughness;
    float coat_ior;
    float coat_darkening;
    float fuzz_weight;
    float fuzz_color[3];
    float fuzz_roughness;
    float opacity;
    uint32_t thin_walled;
    uint32_t base_color_texture;
    uint32_t specular_roughness_texture;
    uint32_t metalness_texture;
    uint32_t emission_texture;
    uint32_t opacity_texture;
    uint32_t normal_texture;
} cenote_material;

/* One scene object: mesh + placement + surface (scene/mod.rs:61-86).
 * positions/normals are 3 floats per vertex, uvs 2 floats, indices 3 per
 * triangle (counter-clockwise outward); transform = rows of the 3×4
 * object-to-world matrix. The library copies everything it needs. */
typedef struct cenote_object {
    const float* positions;
    const float* normals;
    const float* uvs;
    const uint32_t* indices;
    uint32_t vertex_count;
    uint32_t triangle_count;
    float transform[12];
    cenote_material material;
    uint32_t camera_visible; /* 0: camera rays pass it (ray_mask::CAMERA) */
    uint32_t pad;
} cenote_object;

/* Camera (scene/mod.rs:392-422); aperture_radius 0 is a pinhole. */
typedef struct cenote_camera {
    float position[3];
    float look_at[3];
    float up[3];
    float vfov_degrees;
    float aperture_radius;
    float focus_distance;
} cenote_camera;

/* A material texture of the bindless table (crates/cenote/src/texture.rs,
 * shaders/textures.slang): one level, bilinear, repeat addressing. Materials
 * name it by its index in the array given to cenote_scene_create_textured.
 * Usages: colour slots read RGB (sRGB storage decoded per texel, then
 * Rec.709 -> ACEScg), scalar slots read R, normal maps read R/G as x/y. */
#define CENOTE_TEXTURE_RGBA8_SRGB 1u  /* 8-bit RGBA, colour in sRGB transfer */
#define CENOTE_TEXTURE_RGBA8_UNORM 2u /* 8-bit RGBA, linear */
#define CENOTE_TEXTURE_RGBA32F 3u     /* float RGBA, linear (HDR colour) */
#define CENOTE_TEXTURE_BC1_SRGB 4u    /* BC1 blocks, colour in sRGB transfer */
#define CENOTE_TEXTURE_BC1_UNORM 5u   /* BC1 blocks, linear */
#define CENOTE_TEXTURE_BC4_UNORM 6u   /* BC4 blocks: one channel (scalar masks) */
#define CENOTE_TEXTURE_BC5_UNORM 7u   /* BC5 blocks: two channels (tangent-space normals) */
#define CENOTE_TEXTURE_BC7_SRGB 8u    /* BC7 blocks, RGBA colour in sRGB transfer (texture.rs:249-281) */
#define CENOTE_TEXTURE_BC7_UNORM 9u   /* BC7 blocks, RGBA linear */
#define CENOTE_TEXTURE_BC6H_UF16 10u  /* BC6H blocks, unsigned FP16 RGB (HDR colour, texture.rs:283-306) */
#define CENOTE_TEXTURE_BC6H_SF16 11u  /* BC6H blocks, signed FP16 RGB */

typedef struct cenote_texture {
    uint32_t format; /* CENOTE_TEXTURE_* */
    uint32_t width;  /* texels; a multiple of 4 for the BC formats */
    uint32_t height;
    uint32_t pad;
    /* Row 0 first: w·h texels, or the 4x4 blocks row-major over w/4 x h/4
     * (8 bytes per BC1/BC4 block, 16 per BC5/BC6H/BC7 block). */
    const void* data;
} cenote_texture;

/* Bytes of `data` for a texture of this format and size; 0 if invalid. */
uint64_t cenote_texture_bytes(uint32_t format, uint32_t width, uint32_t height);
/* Encode RGBA8 texels (w·h·4 bytes, row 0 first) into BC1 (RGB), BC4 (R),
 * BC5 (R, G) or BC7 (RGBA; the bytes as stored, so an sRGB texture is
 * encoded in its stored space) blocks: `out` holds
 * cenote_texture_bytes(format, w, h) bytes.
 * Host work, no device needed (the prep step of texture.rs:221-405). */
int32_t cenote_texture_encode(uint32_t format, const uint8_t* rgba8, uint32_t width, uint32_t height, void* out);
/* Encode RGBA float texels (w·h·4 floats, row 0 first) into BC6H unsigned
 * blocks (CENOTE_TEXTURE_BC6H_UF16: RGB, negatives clamp to zero, alpha is
 * dropped), as texture.rs:283-306 prepares float colour. Host work. */
int32_t cenote_texture_encode_float(uint32_t format, const float* rgba32f, uint32_t width, uint32_t height,
                                    void* out);

/* Equirect environment, RGBA f32 ACEScg, row 0 = +Y (environment.rs:33-79). */
typedef struct cenote_environment {
    uint32_t width;
    uint32_t height;
    const float* texels;
} cenote_environment;

/* A delta light (lights.rs:57-73): kind CENOTE_LIGHT_DISTANT with anchor =
 * unit travel direction and emission = irradiance, or CENOTE_LIGHT_POINT with
 * anchor = position and emission = intensity. ACEScg. */
typedef struct cenote_delta_light {
    uint32_t kind;
    float anchor[3];
    float emission[3];
} cenote_delta_light;

typedef struct cenote_options {
    int32_t device; /* CUDA ordinal */
} cenote_options;

/* Per-renderer counters of the last accumulate/render call. */
typedef struct cenote_stats {
    uint64_t extension_rays;  /* camera + scattered rays traced */
    uint64_t shadow_rays;
    uint64_t samples;         /* pixel samples completed */
    uint64_t node_visits;     /* wide BVH nodes visited (CENOTE_PROFILE_COUNTS only) */
    uint64_t triangle_tests;  /* ray-triangle tests (CENOTE_PROFILE_COUNTS only) */
    float gpu_ms;             /* device time of the call's waves */
    float raygen_ms;          /* per-stage device time (CENOTE_PROFILE_TIMING only) */
    float intersect_ms;
    float shade_ms;
    float shadow_ms;
    float film_ms;
    uint32_t kernel_launches; /* kernels this library launched in the call */
    uint32_t waves;
    uint32_t samples_per_wave;
    uint32_t overflow;        /* nonzero: a device-side bound was hit */
    uint64_t surface_hits;    /* extension rays whose closest hit is a surface (CENOTE_PROFILE_COUNTS only) */
} cenote_stats;

/* Profiling switches for subsequent calls (bit flags). TIMING records CUDA
 * events around every stage launch; COUNTS runs the instrumented traversal
 * that tallies node visits and triangle tests (slower: keep it out of timed
 * runs). */
#define CENOTE_PROFILE_TIMING 1u
#define CENOTE_PROFILE_COUNTS 2u

/* ---- context -------------------------------------------------------------- */

const char* cenote_last_error(void);
int32_t cenote_context_create(const cenote_options* options, cenote_context** out);
void cenote_context_destroy(cenote_context* ctx);
/* The context's cudaStream_t, for callers that time or order work on it. */
void* cenote_context_stream(cenote_context* ctx);
int32_t cenote_synchronize(cenote_context* ctx);
/* How scenes created from now on build their BVH. Every builder's binary
 * tree is collapsed by the same cost-optimal programme into 8-wide nodes, and
 * every tree gives the same closest hits.
 *   HOST_SAH: on the host; binned SAH above 65,536 triangles per range, the
 *             exact SAH sweep below.
 *   GPU_PLOC: on the device; PLOC over the Morton order.
 *   GPU_SAH:  on the device; binned SAH (32 bins per axis) at every level.
 *   AUTO:     (the default) GPU_SAH for scenes of at least 2^20 triangles,
 *             where the host build takes seconds and binning loses nothing,
 *             else HOST_SAH, whose exact sweep suits small scenes. */
#define CENOTE_BVH_HOST_SAH 0u
#define CENOTE_BVH_GPU_PLOC 1u
#define CENOTE_BVH_GPU_SAH 2u
#define CENOTE_BVH_AUTO 3u
#define CENOTE_BVH_AUTO_GPU_MIN_TRIANGLES (1u << 20)
int32_t cenote_context_set_bvh_builder(cenote_context* ctx, uint32_t builder);

/* ---- scene (Scene::new, scene/mod.rs:254) ------------------------------------ */

int32_t cenote_scene_create(cenote_context* ctx, const cenote_object* objects, uint32_t object_count,
                            const cenote_camera* camera, const cenote_environment* environment,
                            const cenote_delta_light* deltas, uint32_t delta_count, cenote_scene** out);
/* Scene::prep with material textures (scene/prep.rs, lower.rs:92-206): every
 * texture slot a material names must index `textures`. */
int32_t cenote_scene_create_textured(cenote_context* ctx, const cenote_object* objects, uint32_t object_count,
                                     const cenote_camera* camera, const cenote_environment* environment,
                                     const cenote_delta_light* deltas, uint32_t delta_count,
                                     const cenote_texture* textures, uint32_t texture_count, cenote_scene** out);
void cenote_scene_destroy(cenote_scene* scene);
/* Append a delta light (lights.rs:57-73) to a built scene: the light list,
 * its alias table and the environment/light selection probability are rebuilt
 * as if the scene had been created with it last among `deltas`. Renders
 * already queued, and serving jobs already admitted, keep the old list. */
int32_t cenote_scene_add_delta_light(cenote_scene* scene, const cenote_delta_light* light);
/* Replace the camera (the viewer's orbit control writes Scene::camera_mut). */
int32_t cenote_scene_set_camera(cenote_scene* scene, const cenote_camera* camera);
/* Scene-prep timings (ms): [0] BVH build, [1] env tables on the GPU, [2] total. */
int32_t cenote_scene_prep_times(cenote_scene* scene, float* ms3);
/* Device bytes the scene holds (BVH + triangles + records + textures + env). */
uint64_t cenote_scene_device_bytes(cenote_scene* scene);
/* The builder the scene's BVH came from (CENOTE_BVH_HOST_SAH, _GPU_PLOC or
 * _GPU_SAH: AUTO resolved by the scene's triangle count). */
uint32_t cenote_scene_bvh_builder(cenote_scene* scene);
/* The light list as built (80-byte records of lights.rs:79-109), and its length. */
int32_t cenote_scene_light_records(cenote_scene* scene, void* out_records, uint32_t* out_count);
/* The environment tables built on the device (environment.rs:221-233 layout),
 * the emitted power and the environment selection probability. Any output may
 * be NULL. */
int32_t cenote_scene_env_tables(cenote_scene* scene, float* marginal, float* conditional, float* pdfs,
                                double* power, float* select_prob);

/* ---- renderer (Renderer::with_max_bounces, render/mod.rs:151) ----------------- */

/* capacity = paths in flight per wave (0 = one full sample of the largest
 * target seen, grown on demand). */
int32_t cenote_renderer_create(cenote_context* ctx, uint32_t max_bounces, uint32_t light_sampling,
                               uint32_t capacity, cenote_renderer** out);
void cenote_renderer_destroy(cenote_renderer* r);
/* Samples traced per wave: 0 picks automatically; 1 is the reference's
 * one-sample waves. Results are bitwise identical for every setting. */
int32_t cenote_renderer_set_samples_per_wave(cenote_renderer* r, uint32_t samples_per_wave);
int32_t cenote_renderer_stats(cenote_renderer* r, cenote_stats* out);
/* Material sort before shading: the bounce's paths are counting-sorted by
 * the hit's material slot (misses first) and shaded in that order. Only the
 * order of work changes: without online guide training (whose batches follow
 * the order records are made in) the results are bitwise the same. */
#define CENOTE_SORT_NONE 0u
#define CENOTE_SORT_ALL 1u
#define CENOTE_SORT_SECONDARY 2u /* every bounce but the camera rays' */
/* A new renderer sorts every bounce (CENOTE_SORT_ALL). */
int32_t cenote_renderer_set_material_sort(cenote_renderer* r, uint32_t mode);
/* The per-scene launch knobs. None changes a result: every setting renders
 * the same film bit for bit. */
typedef struct cenote_tuning {
    uint32_t material_sort;    /* CENOTE_SORT_* */
    uint32_t samples_per_wave; /* samples of every pixel one wave carries (0 = automatic); sets the queue capacity */
    uint32_t refill_idle;      /* idle lanes (1..32) before a traversal warp takes new rays (0 = default 8) */
    uint32_t top_nodes;        /* BVH top-level nodes staged in shared memory per traversal block (0..320) */
    uint32_t l2_window;        /* 1: the BVH nodes are a persisting L2 access-policy window during the waves */
    uint32_t per_lane_triangles; /* 1: each traversal lane tests its own triangles; 0: a warp shares its
                                  * pending triangle tests through a queue (scenes whose triangles are all
                                  * opaque; scenes with fractional opacity always test per lane) */
    float ms_per_sample;       /* autotune: device time of one sample of every pixel at the chosen setting */
    uint32_t block_size;       /* traversal threads per block: 128 or 256 (0 = 128) */
    uint32_t stack_depth;      /* traversal stack entries per lane: 16 or 32 (0 = 32); 16 falls back to 32
                                * for a tree whose node groups could need more */
    uint32_t sort_by_location; /* 1: the material sort orders a bounce's hits on layer-free materials by
                                * where they lie (a 32 x 32 Morton cell of the scene's x/z extent) rather
                                * than by instance, so the next bounce's rays leave nearby points together */
} cenote_tuning;
int32_t cenote_renderer_set_tuning(cenote_renderer* r, const cenote_tuning* tuning);
int32_t cenote_renderer_get_tuning(cenote_renderer* r, cenote_tuning* out);
/* Time candidate settings on `scene` at width x height (a scratch film, a few
 * hundred ms of device time at 1080p) by coordinate descent over the sort
 * mode, samples per wave, refill threshold, shared-memory top levels, the
 * L2 persistence window, per-lane or queued triangle tests, the
 * traversal's block size and stack depth and the sort's key (instance or
 * location);
 * apply the fastest to `r` and
 * report it in `out` (nullable). The renderer's stats afterwards describe the
 * last probe. */
int32_t cenote_renderer_autotune(cenote_renderer* r, cenote_scene* scene, uint32_t width, uint32_t height,
                                 cenote_tuning* out);
int32_t cenote_renderer_set_profiling(cenote_renderer* r, uint32_t flags);

/* Renderer::render: one wave at sample index `sample`, RGBA f32 row-major,
 * pixel (0,0) top-left, into caller-owned host memory (w·h·4 floats). */
int32_t cenote_render_once(cenote_renderer* r, cenote_scene* scene, uint32_t width, uint32_t height,
                           uint32_t sample, float* rgba_out);

/* ---- film (render/film.rs) -------------------------------------------------------- */

int32_t cenote_film_create(cenote_context* ctx, uint32_t width, uint32_t height, cenote_film** out);
void cenote_film_destroy(cenote_film* film);
int32_t cenote_film_reset(cenote_film* film);
uint32_t cenote_film_samples(cenote_film* film);
/* Renderer::accumulate: trace the film's next sample and add it (non-finite guarded). */
int32_t cenote_accumulate(cenote_renderer* r, cenote_scene* scene, cenote_film* film);
/* `count` consecutive accumulate calls in one submission (bitwise identical). */
int32_t cenote_accumulate_n(cenote_renderer* r, cenote_scene* scene, cenote_film* film, uint32_t count);
/* Accumulate the samples first_sample .. first_sample + count - 1 of every
 * pixel (Wavefront::trace's explicit sample index, wavefront.rs:568) instead
 * of the film's own count: independent estimates of one image, e.g. a
 * reference that shares no samples with the render it judges. */
int32_t cenote_accumulate_range(cenote_renderer* r, cenote_scene* scene, cenote_film* film, uint32_t first_sample,
                                uint32_t count);
/* Film::averages: sums / samples into host memory; any pointer may be NULL.
 * beauty/albedo/normal are w·h·4 floats, depth w·h floats. */
int32_t cenote_film_averages(cenote_film* film, float* beauty, float* albedo, float* normal, float* depth);
/* The display frame (crates/cenote/shaders/tonemap.slang, headless): the
 * beauty average exposed by 2^exposure_stops, through the ACES RRT+ODT fit
 * and the sRGB transfer, packed RGBA8 (R in the low byte), w·h words into
 * host memory. The _device form writes device memory on the context's stream
 * and returns without waiting (a serving preview). */
int32_t cenote_film_tonemap(cenote_film* film, float exposure_stops, uint32_t* rgba8);
int32_t cenote_film_tonemap_device(cenote_film* film, float exposure_stops, void* rgba8);
/* The raw running beauty sums (w·h·4 floats). */
int32_t cenote_film_sums(cenote_film* film, float* beauty_sum);
/* Device pointer to the beauty sums (float4 per pixel). */
void* cenote_film_device_sums(cenote_film* film);
/* Resume accumulation from a checkpoint: the film takes `beauty_sum` (w·h·4
 * floats, as cenote_film_sums returned them) and `samples`; the guide sums
 * restart at zero. */
int32_t cenote_film_restore(cenote_film* film, const float* beauty_sum, uint32_t samples);

/* ---- probes (test entry points; rng_test.slang and friends) ------------------------- */

/* Sampler dump (shaders/rng_test.slang:23): sample_2d and sample_1d for sample
 * indices 0..count-1 of one (pixel, dimension). points: 2·count floats. */
int32_t cenote_probe_sampler(cenote_context* ctx, uint32_t pixel, uint32_t dimension, uint32_t count,
                             float* points, float* values);
/* Closure eval + pdf for n (wo, wi) pairs in the shading frame, FP32 on the
 * device: f = 3 floats per pair, pdf = 1. */
int32_t cenote_probe_bsdf(cenote_context* ctx, const cenote_material* material, const float* wo,
                          const float* wi, uint32_t n, uint32_t exiting, float* f, float* pdf);
/* Closure sampling: u = (u_lobe, u.x, u.y) per entry; wi = 3 floats, pdf, lobe. */
int32_t cenote_probe_bsdf_sample(cenote_context* ctx, const cenote_material* material, const float* wo,
                                 const float* u, uint32_t n, uint32_t exiting, float* wi, float* pdf,
                                 uint32_t* lobe);
/* Closest hit for n rays (all instances visible): hits = (instance, primitive,
 * b1 bits, b2 bits) per ray, instance 0xffffffff on a miss; t = hit distance. */
int32_t cenote_probe_intersect(cenote_scene* scene, const float* origins, const float* directions, uint32_t n,
                               uint32_t* hits, float* t);
/* The same query through the warp triangle queue the wavefront uses for
 * all-opaque scenes (every lane of a warp tests the warp's pending
 * triangles); results equal cenote_probe_intersect's bit for bit. */
int32_t cenote_probe_intersect_queued(cenote_scene* scene, const float* origins, const float* directions,
                                      uint32_t n, uint32_t* hits, float* t);
/* Shadow query: attenuation ≥ 0 when the (instance, primitive) target — or
 * nothing, for target instance 0xffffffff — is the closest hit within tmax;
 * -1 when occluded. */
int32_t cenote_probe_shadow(cenote_scene* scene, const float* origins, const float* directions,
                            const float* tmax, const uint32_t* targets, uint32_t n, float* out);
/* The same query through the warp triangle queue the wavefront uses for
 * all-opaque scenes (CENOTE_E_INVALID_ARGUMENT for a scene with fractional
 * opacity); results equal cenote_probe_shadow's bit for bit. */
int32_t cenote_probe_shadow_queued(cenote_scene* scene, const float* origins, const float* directions,
                                   const float* tmax, const uint32_t* targets, uint32_t n, float* out);
/* Environment importance sampling (environment.slang:94-107) for n uniform
 * pairs: direction (3 floats), pdf, and the sampled (row, column). */
int32_t cenote_probe_env_sample(cenote_scene* scene, const float* u, uint32_t n, float* directions,
                                float* pdf, uint32_t* row_col);
/* Environment pdf for n directions (environment.slang:111-120). */
int32_t cenote_probe_env_pdf(cenote_scene* scene, const float* directions, uint32_t n, float* pdf);
/* n taps of bindless slot `index` at uv (n·2 floats) into rgba (n·4 floats):
 * mode 0 the filtered texel, 1 sampleColor, 2 sampleScalar, 3 sampleNormal
 * (textures.slang:24-64). */
int32_t cenote_probe_texture(cenote_scene* scene, uint32_t index, uint32_t mode, const float* uv, uint32_t n,
                             float* rgba);

/* ---- serving: progressive jobs over one device ------------------------------------- */

/* A request loop with no counterpart in the reference (which renders one
 * view per render::Session, crates/cenote/src/render/session.rs:416): jobs
 * of uneven scenes, sizes and sample counts are admitted in arrival order
 * against an HBM budget, kept resident, and advanced in chunks of
 * `frame_spp` samples over `slots` CUDA streams (each with its own path
 * pool), a progressive frame after every chunk. A job's result is bitwise
 * identical alone and in any mix. Scenes must outlive their jobs. */
typedef struct cenote_server cenote_server;

typedef struct cenote_server_options {
    uint32_t slots;          /* lanes (path pool + streams, one wave in flight each), 1 or 2 (0: 2) */
    uint32_t frame_spp;      /* samples per progressive frame (0: 4) */
    uint32_t max_active;     /* jobs resident at once (0: 64) */
    uint32_t pool_paths;     /* each lane's path pool capacity (0: 2^24); a job's image must fit it */
    uint32_t light_sampling; /* CENOTE_LIGHT_SAMPLING_* */
    uint32_t no_graphs;      /* 1: launch every wave directly instead of replaying its group's captured graph */
} cenote_server_options;

#define CENOTE_JOB_QUEUED 0u
#define CENOTE_JOB_RUNNING 1u
#define CENOTE_JOB_DONE 2u
#define CENOTE_JOB_FAILED 3u

/* Called on the server thread after each progressive frame: `rgba`
 * (width·height·4 linear averages over `samples`) is valid only during the
 * call. */
typedef void (*cenote_frame_fn)(void* user, uint64_t job, uint32_t samples, uint32_t target_spp, const float* rgba,
                                uint32_t width, uint32_t height);

typedef struct cenote_job_status {
    uint32_t state;   /* CENOTE_JOB_* */
    uint32_t samples; /* completed */
    uint32_t target;
    int32_t error;    /* status code when FAILED */
    /* Milliseconds on the server's clock; -1 until reached. */
    double submit_ms, admit_ms, first_frame_ms, done_ms;
} cenote_job_status;

typedef struct cenote_server_counters {
    uint64_t submitted, completed, failed, queued, active;
    uint64_t samples;      /* pixel samples finished */
    uint64_t bytes_in_use; /* bytes counted against the budget: pools, resident jobs, and finished
                            * jobs' film buffers cached for reuse */
    uint64_t budget;
    double wall_ms;        /* since creation */
    uint64_t waves;        /* waves finished */
    uint64_t first_waves;  /* of those, waves that opened with first frames */
    uint64_t wave_paths;   /* camera paths traced by those waves */
    double busy_ms;        /* their device time (CUDA events around each wave) */
} cenote_server_counters;

/* The serving loop: jobs of any scenes, sizes and sample counts traced
 * together as one wavefront of job-tagged paths (each wave: the jobs of one
 * scene and bounce count, first frames first). `hbm_budget` bounds the path
 * pool, every resident scene's device bytes and every admitted job's film;
 * the pool is allocated here (CENOTE_E_BUDGET if it alone exceeds it). */
int32_t cenote_server_create(cenote_context* ctx, uint64_t hbm_budget, const cenote_server_options* options,
                             cenote_server** out);
/* Stops the loop after the chunks in flight; queued jobs are dropped. */
void cenote_server_destroy(cenote_server* server);
/* Queue a job (CENOTE_E_BUDGET if it could never fit with its scene,
 * CENOTE_E_INVALID_ARGUMENT if its image exceeds the pool); `fn` may be NULL. */
int32_t cenote_job_submit(cenote_server* server, cenote_scene* scene, uint32_t width, uint32_t height,
                          uint32_t target_spp, uint32_t max_bounces, cenote_frame_fn fn, void* user, uint64_t* job);
int32_t cenote_job_poll(cenote_server* server, uint64_t job, cenote_job_status* status);
/* Block until the job is done or failed, at most `timeout_ms` (CENOTE_E_TIMEOUT). */
int32_t cenote_job_wait(cenote_server* server, uint64_t job, double timeout_ms);
/* The finished job's averages (width·height·4 floats). */
int32_t cenote_job_result(cenote_server* server, uint64_t job, float* rgba);
/* Forget a finished job and its result. */
int32_t cenote_job_release(cenote_server* server, uint64_t job);
int32_t cenote_server_stats(cenote_server* server, cenote_server_counters* stats);

/* ---- the learned directional guide ----------------------------------------------- */

/* A small MLP (96 encoded inputs: position in 12 frequency bands, normal,
 * outgoing direction; 3 hidden layers of 64 ReLU; 40 outputs = 8 von
 * Mises-Fisher lobes of raw direction, concentration and weight logit) run
 * and trained by tcgen05 tensor-core kernels in BF16 with FP32 accumulation.
 * No counterpart in the reference. Parameters are 17,128 floats: W1 [64][96],
 * b1, W2 [64][64], b2, W3 [64][64], b3, W4 [40][64], b4. */
typedef struct cenote_guide cenote_guide;

int32_t cenote_guide_create(cenote_context* ctx, uint64_t seed, cenote_guide** out);
void cenote_guide_destroy(cenote_guide* guide);
int32_t cenote_guide_params(cenote_guide* guide, float* params);
int32_t cenote_guide_set_params(cenote_guide* guide, const float* params);
/* outputs (n x 40) for features (n x 96, rounded to BF16 on the device). */
int32_t cenote_guide_forward(cenote_guide* guide, const float* features, uint32_t n, float* outputs);
/* One step on the loss mean_s -weights_s log q(dirs_s): the loss and, when
 * `grads` is non-NULL, the gradient before the update; lr > 0 applies Adam
 * (beta 0.9 / 0.999, eps 1e-8), lr = 0 only evaluates. */
int32_t cenote_guide_train_step(cenote_guide* guide, const float* features, const float* dirs, const float* weights,
                                uint32_t n, float lr, float* loss, float* grads);
/* Guided sampling in a renderer (NULL detaches): every surface vertex that is
 * not near-specular draws its direction from the guide's mixture with
 * probability `fraction`, else from the BSDF, and weighs by the combined pdf
 * (one-sample MIS, so the estimate stays unbiased whatever the network says);
 * next-event MIS uses the same combined pdf. With train_steps > 0 the renderer
 * records a sample of its guided vertices each wave and runs that many Adam
 * steps (batch 65,536, learning rate `lr`) on them after the wave. The guide
 * must outlive its use by the renderer. */
int32_t cenote_renderer_set_guide(cenote_renderer* renderer, cenote_guide* guide, float fraction,
                                  uint32_t train_steps, float lr);

/* ---- environment tables without device allocation --------------------------------- */

/* The environment's sampling tables (the same bits cenote_scene_create
 * builds: marginal h+1, conditional h·(w+1) and pdf w·h floats, plus the
 * emitted power) for callers that cannot allocate device memory: a host that
 * hands the library a fixed arena and accounts for every byte of HBM, code
 * that must not stall the device on cudaMalloc/cudaFree (a per-frame
 * environment edit in an interactive loop), or a binding that only holds
 * memory another runtime owns. This entry point has no counterpart in the
 * reference, which builds these tables on the host. `texels` (RGBA f32, w·h)
 * and the three outputs are device pointers the caller owns; `power` is host
 * memory (may be NULL). The FP64 scratch lives in one static device array per
 * device, sized for at most 262,144 texels and 1,024 rows; larger inputs are
 * rejected with CENOTE_E_INVALID_ARGUMENT. The call allocates nothing on the
 * device and returns when the tables are written. Every call on a device
 * shares that scratch, so calls whose GPU work overlaps (from different
 * contexts, or threads bypassing one context) race. A call that returns
 * CENOTE_E_TIMEOUT leaves its work running; the next call on that device
 * first waits for it (and returns CENOTE_E_TIMEOUT itself if it is still
 * running after the same bound) before touching the scratch. The first call on a
 * device looks up the scratch's device address and may load the kernels, so
 * make it before any stream capture. */
int32_t cenote_env_tables_static(cenote_context* ctx, const float* texels, uint32_t width, uint32_t height,
                                 float* marginal, float* conditional, float* pdfs, double* power);

#ifdef __cplusplus
}
#endif

#endif /* CENOTE_C_H */
