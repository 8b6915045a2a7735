// The C ABI (include/cenote_c.h): context, scene prep, renderer, film and
// probes. Host arithmetic that feeds bit-exact tables is compiled with
// -ffp-contract=off so every a·b + c rounds twice, as the reference's Rust does.
#include <algorithm>
#include <utility>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cenote_c.h"
#include "bvh_build.h"
#include "bvh_gpu.h"
#include "records.h"
#include "runtime.h"
#include "texture_prep.h"
#include "wavefront.h"

namespace cn {
void launch_env_cuts(const float* marginal, const float* conditional, uint32_t w, uint32_t h, uint32_t* cut,
                     cudaStream_t stream);
void launch_env_tables(const float4* texels, const double* sin_theta, const double* solid, uint32_t w, uint32_t h,
                       double* scratch, float* marginal, float* conditional, float* pdfs, double* totals,
                       cudaStream_t stream);
void probe_sampler(uint32_t pixel, uint32_t dim, uint32_t count, float2* points, float* values, cudaStream_t s);
void probe_bsdf(const float* tables, const Material& m, const float3* wo, const float3* wi, uint32_t n,
                uint32_t exiting, float3* f, float* pdf, cudaStream_t s);
void probe_bsdf_sample(const float* tables, const Material& m, const float3* wo, const float3* u, uint32_t n,
                       uint32_t exiting, float3* wi, float* pdf, uint32_t* lobe, cudaStream_t s);
void probe_intersect(const DeviceScene& scene, const float3* org, const float3* dir, uint32_t n, uint4* hits, float* t,
                     uint32_t* flag, cudaStream_t s);
void probe_intersect_queued(const DeviceScene& scene, const float3* org, const float3* dir, uint32_t n, uint4* hits,
                            float* t, uint32_t* flag, cudaStream_t s);
void probe_shadow(const DeviceScene& scene, const float3* org, const float3* dir, const float* tmax,
                  const uint2* targets, uint32_t n, float* out, uint32_t* flag, cudaStream_t s);
void probe_shadow_queued(const DeviceScene& scene, const float3* org, const float3* dir, const float* tmax,
                         const uint2* targets, uint32_t n, float* out, uint32_t* flag, cudaStream_t s);
void probe_env_sample(const DeviceScene& scene, const float2* u, uint32_t n, float3* dir, float* pdf, uint2* rc,
                      cudaStream_t s);
void probe_env_pdf(const DeviceScene& scene, const float3* d, uint32_t n, float* pdf, cudaStream_t s);
void probe_texture(const DeviceScene& scene, uint32_t index, uint32_t mode, const float2* uv, uint32_t n, float4* out,
                   cudaStream_t s);
cudaError_t static_env_scratch(int device, double** out, size_t* max_texels, uint32_t* max_rows, cudaEvent_t* done);
bool static_env_pending(int device);
void static_env_set_pending(int device, bool pending);
}  // namespace cn

using namespace cn;


namespace {

// The BSDF lookup tables (ggx_energy.bin ++ ltc_sheen.bin, the layout of
// crates/cenote/src/tables.rs:51-80), embedded at build time.
const uint32_t kTables[] = {
#include "tables_blob.inc"
};
static_assert(sizeof(kTables) == 16928 * 4, "BSDF tables are 16,928 floats");

struct V3 {
    float x, y, z;
};
V3 v3(const float* f) { return {f[0], f[1], f[2]}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float dotv(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 crossv(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
float lengthv(V3 a) { return std::sqrt(dotv(a, a)); }

// color.rs:367-369
float luminance(V3 c) { return c.x * 0.2722287f + c.y * 0.6740818f + c.z * 0.0536895f; }

// glam's transform_point3 over the top three rows: ((x·p.x + y·p.y) + z·p.z) + w.
V3 transform_point(const float m[12], V3 p) {
    return {m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
            m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
}

// Inverse of an affine 3×4 (rows), in double, rounded to f32.
bool invert_affine(const float m[12], float out[3][4]) {
    double a[3][3], t[3];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) a[r][c] = m[4 * r + c];
        t[r] = m[4 * r + 3];
    }
    double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                 a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) out[r][c] = float(inv[r][c]);
        out[r][3] = float(-(inv[r][0] * t[0] + inv[r][1] * t[1] + inv[r][2] * t[2]));
    }
    return true;
}

// ---- the light list: crates/cenote/src/lights.rs:123-275 -----------------------

struct TriLight {
    V3 c[3];
    V3 emission;
    uint32_t instance, primitive;
};

LightRecord make_record(uint32_t kind, V3 anchor, V3 e1, V3 e2, V3 em, uint32_t inst, uint32_t prim) {
    LightRecord r;
    std::memset(&r, 0, sizeof r);
    r.anchor[0] = anchor.x; r.anchor[1] = anchor.y; r.anchor[2] = anchor.z;
    r.edge1[0] = e1.x; r.edge1[1] = e1.y; r.edge1[2] = e1.z;
    r.edge2[0] = e2.x; r.edge2[1] = e2.y; r.edge2[2] = e2.z;
    r.emission[0] = em.x; r.emission[1] = em.y; r.emission[2] = em.z;
    r.pdf = 0.0f;
    r.alias_threshold = 1.0f;
    r.alias_index = 0;
    r.instance = inst;
    r.kind = kind;
    r.primitive = prim;
    return r;
}

double record_area(const LightRecord& r) { return double(lengthv(crossv(v3(r.edge1), v3(r.edge2)))) / 2.0; }

double record_power(const LightRecord& r) {
    double luma = double(luminance(v3(r.emission)));
    if (r.kind == KIND_TRIANGLE) return 3.141592653589793 * luma * record_area(r);
    if (r.kind == KIND_DISTANT) return luma;
    return 4.0 * 3.141592653589793 * luma;
}

// Walker/Vose over f64 shares: stable small/large partition, both popped
// from the back, leftovers keep threshold 1.
// Fills every record's pdf and alias entry from its power; returns the total.
double alias_lights(std::vector<LightRecord>& recs) {
    std::vector<double> power(recs.size());
    double total = 0.0;
    for (size_t i = 0; i < recs.size(); ++i) {
        power[i] = record_power(recs[i]);
        total += power[i];
    }
    if (total <= 0.0) return total;
    for (size_t i = 0; i < recs.size(); ++i) {
        double sel = power[i] / total;
        if (recs[i].kind == KIND_TRIANGLE) {
            double area = record_area(recs[i]);
            recs[i].pdf = area > 0.0 ? float(sel / area) : 0.0f;
        } else {
            recs[i].pdf = float(sel);
        }
    }
    const double n = double(recs.size());
    std::vector<double> share(recs.size());
    std::vector<uint32_t> small, large;
    for (size_t i = 0; i < recs.size(); ++i) {
        share[i] = power[i] * n / total;
        (share[i] < 1.0 ? small : large).push_back(uint32_t(i));
    }
    while (!small.empty() && !large.empty()) {
        uint32_t poor = small.back(), rich = large.back();
        small.pop_back();
        large.pop_back();
        recs[poor].alias_threshold = float(share[poor]);
        recs[poor].alias_index = rich;
        share[rich] -= 1.0 - share[poor];
        (share[rich] < 1.0 ? small : large).push_back(rich);
    }
    return total;
}

LightRecord delta_record(const cenote_delta_light& d) {
    return make_record(d.kind, v3(d.anchor), {0, 0, 0}, {0, 0, 0}, v3(d.emission), LIGHT_NONE, 0);
}

// lights.rs:175-227: triangle records first, then the delta lights, in order.
std::vector<LightRecord> build_lights(const std::vector<TriLight>& tris, const cenote_delta_light* deltas,
                                      uint32_t n_deltas, double* total_out) {
    std::vector<LightRecord> recs;
    recs.reserve(tris.size() + n_deltas);
    for (const TriLight& t : tris)
        recs.push_back(make_record(KIND_TRIANGLE, t.c[0], t.c[1] - t.c[0], t.c[2] - t.c[0], t.emission, t.instance,
                                   t.primitive));
    for (uint32_t i = 0; i < n_deltas; ++i) recs.push_back(delta_record(deltas[i]));
    *total_out = alias_lights(recs);
    return recs;
}

// scene/mod.rs:665-671
float select_probability(double env_power, double light_power) {
    if (light_power == 0.0) return env_power > 0.0 ? 1.0f : 0.0f;
    return float(env_power / (env_power + light_power));
}

// Camera::basis (scene/mod.rs:448-460), scaled to the focal plane when the
// lens is open (wavefront.rs:633-650).
bool camera_valid(const cenote_camera& cam) {
    V3 pos = v3(cam.position), look = v3(cam.look_at), up = v3(cam.up);
    V3 d = look - pos;
    float l = lengthv(d);
    if (!(l > 0.0f) || !std::isfinite(l)) return false;
    V3 c = crossv(d * (1.0f / l), up);
    float cl = lengthv(c);
    return cl > 0.0f && std::isfinite(cl) && cam.vfov_degrees > 0.0f && cam.vfov_degrees < 180.0f &&
           !(cam.aperture_radius > 0.0f && !(cam.focus_distance > 0.0f));
}

}  // namespace

namespace cn {
// Camera::basis (crates/cenote/src/scene/mod.rs:448-460) for the wave's
// aspect ratio, pre-scaled to the focal plane when the lens is open.
void camera_basis(const cenote_camera& cam, float aspect, WaveParams& wp) {
    V3 pos = v3(cam.position), look = v3(cam.look_at), up = v3(cam.up);
    V3 d = look - pos;
    V3 f = d * (1.0f / lengthv(d));
    V3 c = crossv(f, up);
    V3 r = c * (1.0f / lengthv(c));
    V3 u = crossv(r, f);
    float half_h = std::tan(cam.vfov_degrees * (3.14159265358979323846f / 180.0f) / 2.0f);
    V3 right = r * half_h * aspect, upv = u * half_h, fwd = f;
    if (cam.aperture_radius > 0.0f) {
        right = right * cam.focus_distance;
        upv = upv * cam.focus_distance;
        fwd = fwd * cam.focus_distance;
    }
    wp.cam_pos = make_float3(pos.x, pos.y, pos.z);
    wp.cam_right = make_float3(right.x, right.y, right.z);
    wp.cam_up = make_float3(upv.x, upv.y, upv.z);
    wp.cam_fwd = make_float3(fwd.x, fwd.y, fwd.z);
    wp.aperture = cam.aperture_radius;
}
}  // namespace cn

extern "C" {

const char* cenote_last_error(void) { return cn::last_error(); }

int32_t cenote_context_create(const cenote_options* options, cenote_context** out) {
    CN_CHECK(out, CENOTE_E_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(CENOTE_E_NO_CAPABLE_GPU, "no CUDA device is visible");
    int dev = options ? options->device : 0;
    CN_CHECK(dev >= 0 && dev < count, CENOTE_E_INVALID_ARGUMENT, "device ordinal out of range");
    cudaDeviceProp prop;
    CN_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) return fail(CENOTE_E_NO_CAPABLE_GPU, "the kernels are built for sm_100a (B200)");
    CN_CUDA(cudaSetDevice(dev));
    auto ctx = std::make_unique<cenote_context>();
    ctx->device = dev;
    CN_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CN_CUDA(cudaEventCreateWithFlags(&ctx->sync_ev, cudaEventDisableTiming));
    CN_CUDA(cudaEventCreate(&ctx->t0));
    CN_CUDA(cudaEventCreate(&ctx->t1));
    ctx->shape = launch_shape(dev);
    ctx->l2_persist_max = size_t(prop.persistingL2CacheMaxSize);
    ctx->l2_window_max = size_t(prop.accessPolicyMaxWindowSize);
    CN_CUDA(ctx->tables.alloc(sizeof(kTables)));
    CN_CUDA(cudaMemcpy(ctx->tables.ptr, kTables, sizeof(kTables), cudaMemcpyHostToDevice));
    *out = ctx.release();
    return CENOTE_OK;
}

void cenote_context_destroy(cenote_context* ctx) {
    if (ctx) release(ctx);
}

void* cenote_context_stream(cenote_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int32_t cenote_context_set_bvh_builder(cenote_context* ctx, uint32_t builder) {
    CN_CHECK(ctx, CENOTE_E_INVALID_ARGUMENT, "null context");
    CN_CHECK(builder <= CENOTE_BVH_AUTO, CENOTE_E_INVALID_ARGUMENT, "unknown BVH builder");
    ctx->bvh_builder = builder;
    return CENOTE_OK;
}

int32_t cenote_synchronize(cenote_context* ctx) {
    CN_CHECK(ctx, CENOTE_E_INVALID_ARGUMENT, "null context");
    return wait_stream(ctx->stream, ctx->sync_ev, 600000.0);
}

// ---- scene -------------------------------------------------------------------------

}  // extern "C"

namespace {

// One bindless slot: a CUDA array holding the texels (BC formats: an array
// of the block-compressed channel kind, texel extents, filled one block row
// at a time) and a bilinear, repeat-addressed texture object over normalised
// coordinates.
cudaError_t upload_texture(const cenote_texture& t, cudaStream_t stream, cudaArray_t* arr, cudaTextureObject_t* obj,
                           uint64_t* bytes) {
    const uint32_t w = t.width, h = t.height;
    cudaChannelFormatDesc fmt{};
    size_t row = 0, rows = h;
    bool block = false;
    switch (t.format) {
    case CENOTE_TEXTURE_RGBA8_SRGB:
    case CENOTE_TEXTURE_RGBA8_UNORM:
        fmt = cudaCreateChannelDesc<uchar4>();
        row = size_t(w) * 4;
        break;
    case CENOTE_TEXTURE_RGBA32F:
        fmt = cudaCreateChannelDesc<float4>();
        row = size_t(w) * 16;
        break;
    case CENOTE_TEXTURE_BC1_SRGB:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindUnsignedBlockCompressed1SRGB>();
        block = true;
        break;
    case CENOTE_TEXTURE_BC1_UNORM:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindUnsignedBlockCompressed1>();
        block = true;
        break;
    case CENOTE_TEXTURE_BC4_UNORM:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindUnsignedBlockCompressed4>();
        block = true;
        break;
    case CENOTE_TEXTURE_BC5_UNORM:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindUnsignedBlockCompressed5>();
        block = true;
        break;
    case CENOTE_TEXTURE_BC7_SRGB:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindUnsignedBlockCompressed7SRGB>();
        block = true;
        break;
    case CENOTE_TEXTURE_BC7_UNORM:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindUnsignedBlockCompressed7>();
        block = true;
        break;
    case CENOTE_TEXTURE_BC6H_UF16:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindUnsignedBlockCompressed6H>();
        block = true;
        break;
    case CENOTE_TEXTURE_BC6H_SF16:
        fmt = cudaCreateChannelDesc<cudaChannelFormatKindSignedBlockCompressed6H>();
        block = true;
        break;
    default:
        return cudaErrorInvalidValue;
    }
    if (block) {
        const bool wide = t.format == CENOTE_TEXTURE_BC5_UNORM || t.format == CENOTE_TEXTURE_BC7_SRGB ||
                          t.format == CENOTE_TEXTURE_BC7_UNORM || t.format == CENOTE_TEXTURE_BC6H_UF16 ||
                          t.format == CENOTE_TEXTURE_BC6H_SF16;
        row = size_t(w / 4) * (wide ? 16 : 8);
        rows = h / 4;
    }
    cudaError_t e = cudaMallocArray(arr, &fmt, w, h);
    if (e != cudaSuccess) return e;
    *bytes += row * rows;
    e = cudaMemcpy2DToArrayAsync(*arr, 0, 0, t.data, row, row, rows, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    cudaResourceDesc res{};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = *arr;
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.normalizedCoords = 1;
    td.sRGB = (t.format == CENOTE_TEXTURE_RGBA8_SRGB || t.format == CENOTE_TEXTURE_BC1_SRGB ||
               t.format == CENOTE_TEXTURE_BC7_SRGB)
                  ? 1
                  : 0;
    const bool floats = t.format == CENOTE_TEXTURE_RGBA32F || t.format == CENOTE_TEXTURE_BC6H_UF16 ||
                        t.format == CENOTE_TEXTURE_BC6H_SF16;
    td.readMode = floats ? cudaReadModeElementType : cudaReadModeNormalizedFloat;
    e = cudaCreateTextureObject(obj, &res, &td, nullptr);
    if (e != cudaSuccess && block) {
        // Block formats decode to unorm floats by themselves; accept the
        // element-type read mode where the runtime asks for it.
        cudaGetLastError();
        td.readMode = cudaReadModeElementType;
        e = cudaCreateTextureObject(obj, &res, &td, nullptr);
    }
    return e;
}

}  // namespace

extern "C" {

int32_t cenote_scene_create(cenote_context* ctx, const cenote_object* objects, uint32_t object_count,
                            const cenote_camera* camera, const cenote_environment* env,
                            const cenote_delta_light* deltas, uint32_t delta_count, cenote_scene** out) {
    return cenote_scene_create_textured(ctx, objects, object_count, camera, env, deltas, delta_count, nullptr, 0, out);
}

int32_t cenote_scene_create_textured(cenote_context* ctx, const cenote_object* objects, uint32_t object_count,
                                     const cenote_camera* camera, const cenote_environment* env,
                                     const cenote_delta_light* deltas, uint32_t delta_count,
                                     const cenote_texture* textures, uint32_t texture_count, cenote_scene** out) {
    CN_CHECK(ctx && out, CENOTE_E_INVALID_ARGUMENT, "null context or output handle");
    *out = nullptr;
    CN_CHECK(objects && object_count > 0, CENOTE_E_INVALID_ARGUMENT, "a scene needs at least one object");
    CN_CHECK(object_count < 0xffffffu, CENOTE_E_INVALID_ARGUMENT, "instance index exceeds 24 bits");
    CN_CHECK(camera && camera_valid(*camera), CENOTE_E_INVALID_ARGUMENT, "degenerate camera");
    CN_CHECK(env && env->width > 0 && env->height > 0 && env->texels, CENOTE_E_INVALID_ARGUMENT,
             "environment needs width, height and texels");
    CN_CHECK(delta_count == 0 || deltas, CENOTE_E_INVALID_ARGUMENT, "null delta-light array");
    for (uint32_t i = 0; i < delta_count; ++i)
        CN_CHECK(deltas[i].kind == KIND_DISTANT || deltas[i].kind == KIND_POINT, CENOTE_E_INVALID_ARGUMENT,
                 "unknown delta-light kind");
    CN_CHECK(texture_count == 0 || textures, CENOTE_E_INVALID_ARGUMENT, "null texture array");
    for (uint32_t k = 0; k < texture_count; ++k)
        CN_CHECK(textures[k].data && texture_bytes(textures[k].format, textures[k].width, textures[k].height) > 0,
                 CENOTE_E_INVALID_ARGUMENT, "texture " + std::to_string(k) + " has an unknown format, no data, or a "
                 "size its format cannot take");
    for (uint32_t i = 0; i < object_count; ++i) {
        const cenote_material& m = objects[i].material;
        for (uint32_t slot : {m.base_color_texture, m.specular_roughness_texture, m.metalness_texture,
                              m.emission_texture, m.opacity_texture, m.normal_texture})
            CN_CHECK(slot == TEXTURE_NONE || slot < texture_count, CENOTE_E_SCENE,
                     "object " + std::to_string(i) + " names texture slot " + std::to_string(slot) + " of " +
                         std::to_string(texture_count));
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    auto t_start = std::chrono::steady_clock::now();
    auto sc = std::make_unique<cenote_scene>();
    sc->ctx = ctx;
    sc->camera = *camera;
    cudaError_t err = cudaSuccess;

    std::vector<GeomRecord> geoms(object_count);
    std::vector<Material> mats(object_count);
    std::vector<BuildTri> tris;
    std::vector<TriLight> tri_lights;
    size_t total_tris = 0;
    for (uint32_t i = 0; i < object_count; ++i) total_tris += objects[i].triangle_count;
    tris.reserve(total_tris);
    bool nonopaque = false, layered = false;
    for (uint32_t i = 0; i < object_count; ++i) {
        const cenote_object& o = objects[i];
        CN_CHECK(o.positions && o.normals && o.uvs && o.indices && o.vertex_count > 0, CENOTE_E_INVALID_ARGUMENT,
                 "object " + std::to_string(i) + " lacks attributes");
        for (uint64_t k = 0; k < uint64_t(o.triangle_count) * 3; ++k)
            CN_CHECK(o.indices[k] < o.vertex_count, CENOTE_E_SCENE,
                     "object " + std::to_string(i) + " indexes past its vertices");
        GeomRecord& g = geoms[i];
        std::memset(&g, 0, sizeof g);
        std::memcpy(g.o2w, o.transform, sizeof g.o2w);
        CN_CHECK(invert_affine(o.transform, g.w2o), CENOTE_E_INVALID_ARGUMENT,
                 "object " + std::to_string(i) + " transform is not invertible");
        g.light = LIGHT_NONE;
        DeviceBuffer* bp = sc->add(size_t(o.vertex_count) * 12, &err);
        CN_CUDA(err);
        DeviceBuffer* bn = sc->add(size_t(o.vertex_count) * 12, &err);
        CN_CUDA(err);
        DeviceBuffer* bu = sc->add(size_t(o.vertex_count) * 8, &err);
        CN_CUDA(err);
        DeviceBuffer* bi = sc->add(size_t(o.triangle_count) * 12, &err);
        CN_CUDA(err);
        CN_CUDA(cudaMemcpyAsync(bp->ptr, o.positions, size_t(o.vertex_count) * 12, cudaMemcpyHostToDevice, ctx->stream));
        CN_CUDA(cudaMemcpyAsync(bn->ptr, o.normals, size_t(o.vertex_count) * 12, cudaMemcpyHostToDevice, ctx->stream));
        CN_CUDA(cudaMemcpyAsync(bu->ptr, o.uvs, size_t(o.vertex_count) * 8, cudaMemcpyHostToDevice, ctx->stream));
        if (o.triangle_count)
            CN_CUDA(cudaMemcpyAsync(bi->ptr, o.indices, size_t(o.triangle_count) * 12, cudaMemcpyHostToDevice,
                                    ctx->stream));
        g.positions = bp->as<float>();
        g.normals = bn->as<float>();
        g.uvs = bu->as<float>();
        g.indices = bi->as<uint32_t>();
        mats[i] = o.material;
        V3 em = v3(o.material.emission);
        bool emissive = em.x != 0.0f || em.y != 0.0f || em.z != 0.0f;
        bool opaque = o.material.opacity >= 1.0f && o.material.opacity_texture == TEXTURE_NONE;
        nonopaque = nonopaque || !opaque;
        layered = layered || o.material.coat_weight != 0.0f || o.material.fuzz_weight != 0.0f ||
                  o.material.transmission_weight != 0.0f || o.material.thin_walled != 0u;
        uint32_t flags = (o.camera_visible ? RAY_MASK_ALL : (RAY_MASK_ALL & ~RAY_MASK_CAMERA)) | (opaque ? TRI_OPAQUE : 0u);
        for (uint32_t t = 0; t < o.triangle_count; ++t) {
            BuildTri bt;
            V3 c[3];
            for (int k = 0; k < 3; ++k) {
                uint32_t vi = o.indices[3 * t + k];
                c[k] = transform_point(o.transform, v3(o.positions + 3 * size_t(vi)));
                bt.v[k][0] = c[k].x;
                bt.v[k][1] = c[k].y;
                bt.v[k][2] = c[k].z;
            }
            bt.instance = i;
            bt.primitive = t;
            bt.flags = flags;
            tris.push_back(bt);
            if (emissive) {
                if (g.light == LIGHT_NONE) g.light = uint32_t(tri_lights.size());
                tri_lights.push_back({{c[0], c[1], c[2]}, em, i, t});
            }
        }
    }
    double light_power = 0.0;
    sc->lights = build_lights(tri_lights, deltas, delta_count, &light_power);
    // World bounds of every triangle, for the learned guide's position encoding.
    float bmin[3] = {1e30f, 1e30f, 1e30f}, bmax[3] = {-1e30f, -1e30f, -1e30f};
    for (const BuildTri& t : tris)
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) {
                bmin[a] = std::min(bmin[a], t.v[k][a]);
                bmax[a] = std::max(bmax[a], t.v[k][a]);
            }

    auto t_bvh = std::chrono::steady_clock::now();
    DeviceBuffer* bnodes = nullptr;
    DeviceBuffer* btris = nullptr;
    uint32_t node_count = 0;
    const uint32_t tri_count = uint32_t(tris.size());
    DeviceBuffer* bgeo = sc->add(geoms.size() * sizeof(GeomRecord), &err);
    CN_CUDA(err);
    CN_CUDA(cudaMemcpyAsync(bgeo->ptr, geoms.data(), geoms.size() * sizeof(GeomRecord), cudaMemcpyHostToDevice,
                            ctx->stream));
    DeviceBuffer* bleaf = sc->add(std::max<size_t>(1, sc->lights.size()) * 4, &err);
    CN_CUDA(err);
    std::vector<uint8_t> layers(std::max<size_t>(1, mats.size()), 0);
    for (size_t i = 0; i < mats.size(); ++i)
        layers[i] = (mats[i].coat_weight != 0.0f || mats[i].fuzz_weight != 0.0f || mats[i].transmission_weight != 0.0f ||
                     mats[i].thin_walled != 0u) ? 1 : 0;
    DeviceBuffer* blayers = sc->add(layers.size(), &err);
    CN_CUDA(err);
    CN_CUDA(cudaMemcpyAsync(blayers->ptr, layers.data(), layers.size(), cudaMemcpyHostToDevice, ctx->stream));
    CN_CUDA(cudaMemsetAsync(bleaf->ptr, 0xff, std::max<size_t>(1, sc->lights.size()) * 4, ctx->stream));
    uint32_t bvh_depth = 0;  // stack entries the tree's node groups may take
    uint32_t builder = ctx->bvh_builder;
    if (builder == CENOTE_BVH_AUTO)
        builder = tris.size() >= CENOTE_BVH_AUTO_GPU_MIN_TRIANGLES ? CENOTE_BVH_GPU_SAH : CENOTE_BVH_HOST_SAH;
    sc->bvh_builder = builder;
    if (builder != CENOTE_BVH_HOST_SAH && !tris.empty()) {
        // Triangles in input order, identity in the w lanes; the device
        // builds the binary tree, collapses it and lays out the leaves.
        std::vector<float> packed(tris.size() * 12);
        for (size_t i = 0; i < tris.size(); ++i) {
            float* rec = &packed[12 * i];
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 3; ++a) rec[4 * k + a] = tris[i].v[k][a];
            std::memcpy(&rec[3], &tris[i].instance, 4);
            std::memcpy(&rec[7], &tris[i].primitive, 4);
            std::memcpy(&rec[11], &tris[i].flags, 4);
        }
        DeviceBuffer staged;
        CN_CUDA(staged.alloc(packed.size() * 4));
        CN_CUDA(cudaMemcpyAsync(staged.ptr, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
        GpuBvh g{};
        CN_CUDA(build_wide_bvh_gpu(staged.as<float4>(), tri_count, &g, ctx->stream, builder == CENOTE_BVH_GPU_SAH));
        bnodes = sc->adopt(g.nodes, size_t(g.node_count) * sizeof(WideNode));
        btris = sc->adopt(g.tris, size_t(tri_count) * 48);
        node_count = g.node_count;
        bvh_depth = g.depth;  // bounds the node groups a walk pushes
        CN_CHECK(g.depth < uint32_t(TRAVERSAL_STACK_DEPTH), CENOTE_E_SCENE,
                 "the scene's BVH needs a deeper traversal stack than the walks hold");
    } else {
        WideBvh bvh = build_wide_bvh(tris, std::max(1u, std::thread::hardware_concurrency()));
        CN_CHECK(bvh.stack_need < uint32_t(TRAVERSAL_STACK_DEPTH), CENOTE_E_SCENE,
                 "the scene's BVH needs a deeper traversal stack than the walks hold");
        bvh_depth = bvh.stack_need;
        bnodes = sc->add(bvh.nodes.size() * sizeof(WideNode), &err);
        CN_CUDA(err);
        btris = sc->add(bvh.tris.size() * 4, &err);
        CN_CUDA(err);
        if (!bvh.nodes.empty()) {
            CN_CUDA(cudaMemcpyAsync(bnodes->ptr, bvh.nodes.data(), bvh.nodes.size() * sizeof(WideNode),
                                    cudaMemcpyHostToDevice, ctx->stream));
            CN_CUDA(cudaMemcpyAsync(btris->ptr, bvh.tris.data(), bvh.tris.size() * 4, cudaMemcpyHostToDevice,
                                    ctx->stream));
        }
        node_count = uint32_t(bvh.nodes.size());
        // wait for the uploads before the host vectors go
        CN_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    // Each emissive triangle's leaf index, for the shadow query's target test.
    launch_light_leaves(btris->as<float4>(), tri_count, bgeo->as<GeomRecord>(), bleaf->as<uint32_t>(), ctx->stream);
    CN_CUDA(cudaGetLastError());
    CN_CUDA(cudaStreamSynchronize(ctx->stream));
    sc->prep_ms[0] = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_bvh).count());
    DeviceBuffer* bmat = sc->add(mats.size() * sizeof(Material), &err);
    CN_CUDA(err);
    CN_CUDA(cudaMemcpyAsync(bmat->ptr, mats.data(), mats.size() * sizeof(Material), cudaMemcpyHostToDevice, ctx->stream));
    DeviceBuffer* blights = sc->add(std::max<size_t>(1, sc->lights.size()) * sizeof(LightRecord), &err);
    CN_CUDA(err);
    if (!sc->lights.empty())
        CN_CUDA(cudaMemcpyAsync(blights->ptr, sc->lights.data(), sc->lights.size() * sizeof(LightRecord),
                                cudaMemcpyHostToDevice, ctx->stream));

    // Environment: texels → device, FP64 tables on the device, texture object.
    auto t_env = std::chrono::steady_clock::now();
    const uint32_t ew = env->width, eh = env->height;
    const size_t en = size_t(ew) * eh;
    sc->env_w = ew;
    sc->env_h = eh;
    DeviceBuffer* btex = sc->add(en * 16, &err);
    CN_CUDA(err);
    CN_CUDA(cudaMemcpyAsync(btex->ptr, env->texels, en * 16, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<double> rowc(2 * size_t(eh));
    const double PI = 3.141592653589793;
    for (uint32_t r = 0; r < eh; ++r) {
        rowc[r] = std::sin((double(r) + 0.5) / double(eh) * PI);
        double th0 = double(r) / double(eh) * PI, th1 = double(r + 1) / double(eh) * PI;
        rowc[eh + r] = 2.0 * PI / double(ew) * (std::cos(th0) - std::cos(th1));
    }
    DeviceBuffer* brow = sc->add(rowc.size() * 8, &err);
    CN_CUDA(err);
    CN_CUDA(cudaMemcpyAsync(brow->ptr, rowc.data(), rowc.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    DeviceBuffer scratch;
    CN_CUDA(scratch.alloc((2 * en + 2 * size_t(eh) + 4) * 8));
    sc->env_marginal = sc->add((eh + 1) * 4, &err);
    CN_CUDA(err);
    sc->env_conditional = sc->add(size_t(eh) * (ew + 1) * 4, &err);
    CN_CUDA(err);
    sc->env_pdfs = sc->add(en * 4, &err);
    CN_CUDA(err);
    sc->env_cut = sc->add(size_t(eh + 1) * (ENV_CUTS + 1) * 4, &err);
    CN_CUDA(err);
    double* totals = scratch.as<double>() + 2 * en + 2 * size_t(eh);
    launch_env_tables(btex->as<float4>(), brow->as<double>(), brow->as<double>() + eh, ew, eh, scratch.as<double>(),
                      sc->env_marginal->as<float>(), sc->env_conditional->as<float>(), sc->env_pdfs->as<float>(), totals,
                      ctx->stream);
    launch_env_cuts(sc->env_marginal->as<float>(), sc->env_conditional->as<float>(), ew, eh, sc->env_cut->as<uint32_t>(),
                    ctx->stream);
    CN_CUDA(cudaGetLastError());
    double host_totals[2] = {0, 0};
    CN_CUDA(cudaMemcpyAsync(host_totals, totals, 16, cudaMemcpyDeviceToHost, ctx->stream));
    cudaChannelFormatDesc fmt = cudaCreateChannelDesc<float4>();
    CN_CUDA(cudaMallocArray(&sc->env_array, &fmt, ew, eh));
    sc->device_bytes += en * 16;
    CN_CUDA(cudaMemcpy2DToArrayAsync(sc->env_array, 0, 0, env->texels, size_t(ew) * 16, size_t(ew) * 16, eh,
                                     cudaMemcpyHostToDevice, ctx->stream));
    int32_t rc = wait_stream(ctx->stream, ctx->sync_ev, 600000.0);
    if (rc != CENOTE_OK) return rc;
    sc->prep_ms[1] = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_env).count());
    sc->env_power = host_totals[1];
    sc->select_prob = select_probability(sc->env_power, light_power);
    cudaResourceDesc res;
    std::memset(&res, 0, sizeof res);
    res.resType = cudaResourceTypeArray;
    res.res.array.array = sc->env_array;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof td);
    td.addressMode[0] = cudaAddressModeWrap;   // u wraps in azimuth
    td.addressMode[1] = cudaAddressModeClamp;  // v clamps at the poles
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    CN_CUDA(cudaCreateTextureObject(&sc->env_tex, &res, &td, nullptr));

    // The bindless table.
    sc->tex_arrays.assign(texture_count, nullptr);
    sc->tex_objects.assign(texture_count, 0);
    for (uint32_t k = 0; k < texture_count; ++k) {
        cudaError_t te = upload_texture(textures[k], ctx->stream, &sc->tex_arrays[k], &sc->tex_objects[k],
                                        &sc->device_bytes);
        if (te != cudaSuccess) {
            cudaGetLastError();
            return fail(CENOTE_E_DEVICE, "texture " + std::to_string(k) + ": " + cudaGetErrorString(te));
        }
    }
    DeviceBuffer* btexs = sc->add(std::max<size_t>(1, texture_count) * 8, &err);
    CN_CUDA(err);
    if (texture_count)
        CN_CUDA(cudaMemcpyAsync(btexs->ptr, sc->tex_objects.data(), size_t(texture_count) * 8, cudaMemcpyHostToDevice,
                                ctx->stream));
    CN_CUDA(cudaStreamSynchronize(ctx->stream));

    DeviceScene& ds = sc->ds;
    ds.textures = btexs->as<unsigned long long>();
    ds.texture_count = texture_count;
    ds.nodes = bnodes->as<WideNode>();
    ds.tris = btris->as<float4>();
    ds.geometry = bgeo->as<GeomRecord>();
    ds.materials = bmat->as<Material>();
    ds.lights = blights->as<LightRecord>();
    ds.bsdf_tables = ctx->tables.as<float>();
    ds.env_marginal = sc->env_marginal->as<float>();
    ds.env_conditional = sc->env_conditional->as<float>();
    ds.env_cut = sc->env_cut->as<uint32_t>();
    ds.env_pdfs = sc->env_pdfs->as<float>();
    ds.env_tex = sc->env_tex;
    ds.env_w = ew;
    ds.env_h = eh;
    ds.select_prob = sc->select_prob;
    ds.light_count = uint32_t(sc->lights.size());
    ds.node_count = node_count;
    ds.tri_count = tri_count;
    ds.stack_room = uint32_t(TRAVERSAL_STACK_DEPTH) - bvh_depth;
    ds.has_nonopaque = nonopaque ? 1u : 0u;
    ds.has_layers = layered ? 1u : 0u;
    const float extent = std::max({bmax[0] - bmin[0], bmax[1] - bmin[1], bmax[2] - bmin[2], 1e-6f});
    for (int a = 0; a < 3; ++a) ds.bbox_min[a] = tris.empty() ? 0.0f : bmin[a];
    ds.bbox_inv = tris.empty() ? 1.0f : 1.0f / extent;
    ds.light_leaf = bleaf->as<uint32_t>();
    ds.instance_layers = blayers->as<uint8_t>();
    sc->prep_ms[2] = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
    retain(ctx);
    *out = sc.release();
    return CENOTE_OK;
}

void cenote_scene_destroy(cenote_scene* scene) {
    if (!scene) return;
    cenote_context* ctx = scene->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete scene;
    release(ctx);
}

int32_t cenote_scene_set_camera(cenote_scene* scene, const cenote_camera* camera) {
    CN_CHECK(scene && camera && camera_valid(*camera), CENOTE_E_INVALID_ARGUMENT, "degenerate camera");
    scene->camera = *camera;
    return CENOTE_OK;
}

int32_t cenote_scene_add_delta_light(cenote_scene* scene, const cenote_delta_light* light) {
    CN_CHECK(scene && light, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(light->kind == KIND_DISTANT || light->kind == KIND_POINT, CENOTE_E_INVALID_ARGUMENT,
             "unknown delta-light kind");
    for (int a = 0; a < 3; ++a)
        CN_CHECK(std::isfinite(light->anchor[a]) && std::isfinite(light->emission[a]), CENOTE_E_INVALID_ARGUMENT,
                 "non-finite delta light");
    std::lock_guard<std::mutex> lock(scene->ctx->mu);
    CN_CUDA(cudaSetDevice(scene->ctx->device));
    // The records rebuilt from scratch: the same list a scene created with the
    // light among its deltas holds, bit for bit.
    std::vector<LightRecord> recs = scene->lights;
    for (LightRecord& r : recs) {
        r.pdf = 0.0f;
        r.alias_threshold = 1.0f;
        r.alias_index = 0;
    }
    recs.push_back(delta_record(*light));
    const double power = alias_lights(recs);
    cudaError_t err = cudaSuccess;
    // A new buffer: launches already queued (and graphs already captured)
    // keep reading the old one, which the scene keeps until it is destroyed.
    DeviceBuffer* b = scene->add(recs.size() * sizeof(LightRecord), &err);
    CN_CUDA(err);
    CN_CUDA(cudaMemcpyAsync(b->ptr, recs.data(), recs.size() * sizeof(LightRecord), cudaMemcpyHostToDevice,
                            scene->ctx->stream));
    int32_t rc = wait_stream(scene->ctx->stream, scene->ctx->sync_ev, 600000.0);
    if (rc != CENOTE_OK) return rc;
    scene->lights = std::move(recs);
    scene->select_prob = select_probability(scene->env_power, power);
    scene->ds.lights = b->as<LightRecord>();
    scene->ds.light_count = uint32_t(scene->lights.size());
    scene->ds.select_prob = scene->select_prob;
    return CENOTE_OK;
}

int32_t cenote_scene_prep_times(cenote_scene* scene, float* ms3) {
    CN_CHECK(scene && ms3, CENOTE_E_INVALID_ARGUMENT, "null argument");
    std::memcpy(ms3, scene->prep_ms, sizeof scene->prep_ms);
    return CENOTE_OK;
}

uint64_t cenote_scene_device_bytes(cenote_scene* scene) { return scene ? scene->device_bytes : 0; }

uint32_t cenote_scene_bvh_builder(cenote_scene* scene) { return scene ? scene->bvh_builder : CENOTE_BVH_HOST_SAH; }

int32_t cenote_scene_light_records(cenote_scene* scene, void* out_records, uint32_t* out_count) {
    CN_CHECK(scene && out_count, CENOTE_E_INVALID_ARGUMENT, "null argument");
    *out_count = uint32_t(scene->lights.size());
    if (out_records && !scene->lights.empty()) {
        CN_CUDA(cudaSetDevice(scene->ctx->device));
        CN_CUDA(cudaMemcpy(out_records, scene->ds.lights, scene->lights.size() * sizeof(LightRecord),
                           cudaMemcpyDeviceToHost));
    }
    return CENOTE_OK;
}

int32_t cenote_scene_env_tables(cenote_scene* scene, float* marginal, float* conditional, float* pdfs, double* power,
                                float* select_prob) {
    CN_CHECK(scene, CENOTE_E_INVALID_ARGUMENT, "null scene");
    CN_CUDA(cudaSetDevice(scene->ctx->device));
    if (marginal)
        CN_CUDA(cudaMemcpy(marginal, scene->env_marginal->ptr, (scene->env_h + 1) * 4, cudaMemcpyDeviceToHost));
    if (conditional)
        CN_CUDA(cudaMemcpy(conditional, scene->env_conditional->ptr, size_t(scene->env_h) * (scene->env_w + 1) * 4,
                           cudaMemcpyDeviceToHost));
    if (pdfs)
        CN_CUDA(cudaMemcpy(pdfs, scene->env_pdfs->ptr, size_t(scene->env_h) * scene->env_w * 4, cudaMemcpyDeviceToHost));
    if (power) *power = scene->env_power;
    if (select_prob) *select_prob = scene->select_prob;
    return CENOTE_OK;
}

// ---- renderer and film -------------------------------------------------------------------

int32_t cenote_renderer_create(cenote_context* ctx, uint32_t max_bounces, uint32_t light_sampling, uint32_t capacity,
                               cenote_renderer** out) {
    CN_CHECK(ctx && out, CENOTE_E_INVALID_ARGUMENT, "null context or output handle");
    *out = nullptr;
    CN_CHECK(max_bounces >= 1 && max_bounces <= MAX_BOUNCES, CENOTE_E_INVALID_ARGUMENT,
             "bounce cap outside 1..=255");
    CN_CHECK(light_sampling <= CENOTE_LIGHT_SAMPLING_NEE, CENOTE_E_INVALID_ARGUMENT, "unknown light-sampling mode");
    CN_CUDA(cudaSetDevice(ctx->device));
    auto r = std::make_unique<cenote_renderer>();
    r->ctx = ctx;
    r->max_bounces = max_bounces;
    r->light_sampling = light_sampling;
    r->capacity_req = capacity;
    CN_CUDA(r->counters.alloc(CTR_COUNT * 4));
    CN_CUDA(r->tally.alloc(8 * 8));
    CN_CUDA(cudaMemset(r->tally.ptr, 0, 64));
    r->pool.counters = r->counters.as<uint32_t>();
    retain(ctx);
    *out = r.release();
    return CENOTE_OK;
}

void cenote_renderer_destroy(cenote_renderer* r) {
    if (!r) return;
    cenote_context* ctx = r->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete r;
    release(ctx);
}

int32_t cenote_renderer_set_samples_per_wave(cenote_renderer* r, uint32_t spw) {
    CN_CHECK(r, CENOTE_E_INVALID_ARGUMENT, "null renderer");
    r->samples_per_wave = spw;
    return CENOTE_OK;
}

int32_t cenote_renderer_set_guide(cenote_renderer* r, cenote_guide* g, float fraction, uint32_t train_steps,
                                  float lr) {
    CN_CHECK(r, CENOTE_E_INVALID_ARGUMENT, "null renderer");
    CN_CHECK(!g || g->ctx == r->ctx, CENOTE_E_INVALID_ARGUMENT, "guide from another context");
    CN_CHECK(!g || (fraction >= 0.0f && fraction < 1.0f), CENOTE_E_INVALID_ARGUMENT, "fraction outside [0, 1)");
    CN_CHECK(!g || (lr >= 0.0f && lr < 1.0f), CENOTE_E_INVALID_ARGUMENT, "learning rate outside [0, 1)");
    r->guide = g;
    r->guide_fraction = fraction;
    r->guide_steps = train_steps;
    r->guide_lr = lr;
    return CENOTE_OK;
}

int32_t cenote_renderer_set_material_sort(cenote_renderer* r, uint32_t mode) {
    CN_CHECK(r, CENOTE_E_INVALID_ARGUMENT, "null renderer");
    CN_CHECK(mode <= CENOTE_SORT_SECONDARY, CENOTE_E_INVALID_ARGUMENT, "unknown material-sort mode");
    r->material_sort = mode;
    return CENOTE_OK;
}

// The traversal variant of a block size and stack depth (0 = defaults).
static uint32_t trav_variant_of(uint32_t block, uint32_t stack) {
    return (block == 256 ? 2u : 0u) + (stack == 16 ? 1u : 0u);
}

int32_t cenote_renderer_set_tuning(cenote_renderer* r, const cenote_tuning* t) {
    CN_CHECK(r && t, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(t->material_sort <= CENOTE_SORT_SECONDARY, CENOTE_E_INVALID_ARGUMENT, "unknown material-sort mode");
    CN_CHECK(t->refill_idle <= 32, CENOTE_E_INVALID_ARGUMENT, "refill threshold above a warp");
    CN_CHECK(t->top_nodes <= TOP_NODES_MAX, CENOTE_E_INVALID_ARGUMENT, "more top-level nodes than shared memory holds");
    CN_CHECK(t->l2_window <= 1, CENOTE_E_INVALID_ARGUMENT, "l2_window is 0 or 1");
    CN_CHECK(t->per_lane_triangles <= 1, CENOTE_E_INVALID_ARGUMENT, "per_lane_triangles is 0 or 1");
    CN_CHECK(t->block_size == 0 || t->block_size == 128 || t->block_size == 256, CENOTE_E_INVALID_ARGUMENT,
             "block_size is 128 or 256");
    CN_CHECK(t->stack_depth == 0 || t->stack_depth == 16 || t->stack_depth == 32, CENOTE_E_INVALID_ARGUMENT,
             "stack_depth is 16 or 32");
    CN_CHECK(t->sort_by_location <= 1, CENOTE_E_INVALID_ARGUMENT, "sort_by_location is 0 or 1");
    r->material_sort = t->material_sort;
    r->samples_per_wave = t->samples_per_wave;
    r->refill_idle = t->refill_idle;
    r->top_nodes = t->top_nodes;
    r->l2_window = t->l2_window;
    r->per_lane_triangles = t->per_lane_triangles;
    r->trav_variant = trav_variant_of(t->block_size, t->stack_depth);
    r->sort_by_location = t->sort_by_location;
    return CENOTE_OK;
}

int32_t cenote_renderer_get_tuning(cenote_renderer* r, cenote_tuning* out) {
    CN_CHECK(r && out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    out->material_sort = r->material_sort;
    out->samples_per_wave = r->samples_per_wave;
    out->refill_idle = r->refill_idle;
    out->top_nodes = r->top_nodes;
    out->l2_window = r->l2_window;
    out->per_lane_triangles = r->per_lane_triangles;
    out->ms_per_sample = r->tuned_ms_per_sample;
    out->block_size = uint32_t(TRAV_VARIANT_BLOCK[r->trav_variant]);
    out->stack_depth = uint32_t(TRAV_VARIANT_STACK[r->trav_variant]);
    out->sort_by_location = r->sort_by_location;
    return CENOTE_OK;
}

int32_t cenote_renderer_set_profiling(cenote_renderer* r, uint32_t flags) {
    CN_CHECK(r, CENOTE_E_INVALID_ARGUMENT, "null renderer");
    CN_CHECK((flags & ~3u) == 0, CENOTE_E_INVALID_ARGUMENT, "unknown profiling flag");
    r->profiling = flags;
    return CENOTE_OK;
}

int32_t cenote_renderer_stats(cenote_renderer* r, cenote_stats* out) {
    CN_CHECK(r && out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    *out = r->stats;
    return CENOTE_OK;
}

int32_t cenote_film_create(cenote_context* ctx, uint32_t width, uint32_t height, cenote_film** out) {
    CN_CHECK(ctx && out, CENOTE_E_INVALID_ARGUMENT, "null context or output handle");
    *out = nullptr;
    CN_CHECK(width > 0 && height > 0, CENOTE_E_INVALID_ARGUMENT, "zero-sized film");
    CN_CHECK(uint64_t(width) * height < (1ull << 31), CENOTE_E_INVALID_ARGUMENT, "film too large");
    CN_CUDA(cudaSetDevice(ctx->device));
    auto f = std::make_unique<cenote_film>();
    f->ctx = ctx;
    f->width = width;
    f->height = height;
    size_t px = size_t(width) * height;
    CN_CUDA(f->sum.alloc(px * 16));
    CN_CUDA(f->avg.alloc(px * 16));
    CN_CUDA(f->albedo.alloc(px * 16));
    CN_CUDA(f->normal.alloc(px * 16));
    CN_CUDA(f->depth.alloc(px * 4));
    CN_CUDA(cudaMemsetAsync(f->sum.ptr, 0, px * 16, ctx->stream));
    CN_CUDA(cudaMemsetAsync(f->albedo.ptr, 0, px * 16, ctx->stream));
    CN_CUDA(cudaMemsetAsync(f->normal.ptr, 0, px * 16, ctx->stream));
    CN_CUDA(cudaMemsetAsync(f->depth.ptr, 0, px * 4, ctx->stream));
    retain(ctx);
    *out = f.release();
    return CENOTE_OK;
}

void cenote_film_destroy(cenote_film* film) {
    if (!film) return;
    cenote_context* ctx = film->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete film;
    release(ctx);
}

int32_t cenote_film_reset(cenote_film* film) {
    CN_CHECK(film, CENOTE_E_INVALID_ARGUMENT, "null film");
    CN_CUDA(cudaSetDevice(film->ctx->device));
    // The next sample overwrites the sums (film.rs:140-145); clearing them
    // too keeps a read of an empty film's sums at zero.
    const size_t px = size_t(film->width) * film->height;
    CN_CUDA(cudaMemsetAsync(film->sum.ptr, 0, px * 16, film->ctx->stream));
    CN_CUDA(cudaMemsetAsync(film->albedo.ptr, 0, px * 16, film->ctx->stream));
    CN_CUDA(cudaMemsetAsync(film->normal.ptr, 0, px * 16, film->ctx->stream));
    CN_CUDA(cudaMemsetAsync(film->depth.ptr, 0, px * 4, film->ctx->stream));
    film->samples = 0;
    return CENOTE_OK;
}

uint32_t cenote_film_samples(cenote_film* film) { return film ? film->samples : 0; }

void* cenote_film_device_sums(cenote_film* film) { return film ? film->sum.ptr : nullptr; }

namespace {

// The blocking form behind cenote_accumulate_n and cenote_render_once: plan,
// enqueue on the context's stream, wait, then fold the counters and stage
// timings into the renderer's stats.
// While alive, the scene's wide BVH nodes are a persisting access-policy
// window on the context's stream: the waves' streaming path state does not
// evict them from L2. The window is cleared on exit; the persisting lines
// (a device-wide state) are released once no window of this process is
// active on the device, so a renderer finishing does not evict the window
// of another renderer or serving slot still running.
std::mutex g_l2_mutex;
int g_l2_active[64] = {};

struct L2Window {
    cudaStream_t stream = nullptr;
    int device = -1;
    L2Window(cenote_context* ctx, const cenote_scene* sc, bool on) {
        const size_t bytes = std::min(size_t(sc->ds.node_count) * sizeof(WideNode), ctx->l2_window_max);
        if (!on || bytes == 0 || ctx->l2_persist_max == 0) return;
        const size_t want = std::min(bytes, ctx->l2_persist_max);
        if (ctx->l2_set_aside < want) {
            if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
                cudaGetLastError();
                return;
            }
            ctx->l2_set_aside = want;
        }
        cudaStreamAttrValue a{};
        a.accessPolicyWindow.base_ptr = const_cast<WideNode*>(sc->ds.nodes);
        a.accessPolicyWindow.num_bytes = bytes;
        a.accessPolicyWindow.hitRatio = std::min(1.0f, float(ctx->l2_set_aside) / float(bytes));
        a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        if (cudaStreamSetAttribute(ctx->stream, cudaStreamAttributeAccessPolicyWindow, &a) == cudaSuccess) {
            stream = ctx->stream;
            if (ctx->device >= 0 && ctx->device < 64) {
                device = ctx->device;
                std::lock_guard<std::mutex> lock(g_l2_mutex);
                g_l2_active[device]++;
            }
        } else {
            cudaGetLastError();
        }
    }
    ~L2Window() {
        if (!stream) return;
        cudaStreamAttrValue a{};
        a.accessPolicyWindow.num_bytes = 0;
        cudaStreamSetAttribute(stream, cudaStreamAttributeAccessPolicyWindow, &a);
        bool last = true;
        if (device >= 0) {
            std::lock_guard<std::mutex> lock(g_l2_mutex);
            last = --g_l2_active[device] == 0;
        }
        if (last) cudaCtxResetPersistingL2Cache();
    }
};

int32_t run_waves(cenote_renderer* r, cenote_scene* sc, uint32_t width, uint32_t height, uint32_t sample0,
                  uint32_t count, cenote_film* film, float4* oneshot) {
    cenote_context* ctx = r->ctx;
    L2Window l2(ctx, sc, r->l2_window != 0);
    const uint64_t pixels = uint64_t(width) * height;
    WavePlan plan = plan_waves(r, pixels, count, oneshot != nullptr);
    CN_CHECK(plan.need < (1ull << 31), CENOTE_E_INVALID_ARGUMENT, "wave too large");
    CN_CUDA(r->ensure(plan.need));
    // Films trace the guides (Renderer::accumulate); one-shot renders do not.
    CN_CUDA(r->set_guides(film != nullptr));
    CN_CUDA(r->set_learned_guide(r->guide != nullptr));
    if (r->guide) CN_CUDA(r->guide->ensure(cenote_renderer::GUIDE_BATCH));

    const bool timing = (r->profiling & CENOTE_PROFILE_TIMING) != 0;
    const bool counting = (r->profiling & CENOTE_PROFILE_COUNTS) != 0;
    // Stage event layout per wave: [begin, after raygen, (after isect, shade, shadow) × bounces, after film].
    const size_t per_wave = 3 + 3 * size_t(r->max_bounces);
    WaveCounts wc;
    CN_CUDA(cudaEventRecord(ctx->t0, ctx->stream));
    FilmTargets targets{};
    if (film) targets = film->targets();
    CN_CUDA(enqueue_waves(r, sc, width, height, sample0, count, r->max_bounces, plan, film ? &targets : nullptr,
                          film && film->samples == 0, oneshot, nullptr, ctx->stream, timing, counting, &wc));
    CN_CUDA(cudaEventRecord(ctx->t1, ctx->stream));
    int32_t rc = wait_stream(ctx->stream, ctx->sync_ev, 600000.0);
    if (rc != CENOTE_OK) return rc;
    unsigned long long t[6];
    CN_CUDA(cudaMemcpy(t, r->tally.ptr, sizeof t, cudaMemcpyDeviceToHost));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ctx->t0, ctx->t1);
    cenote_stats st{};
    st.extension_rays = t[0] - r->tally_prev[0];
    st.shadow_rays = t[1] - r->tally_prev[1];
    st.overflow = uint32_t(t[2]);
    st.node_visits = t[3] - r->tally_prev[3];
    st.triangle_tests = t[4] - r->tally_prev[4];
    st.surface_hits = t[5] - r->tally_prev[5];
    st.samples = pixels * count;
    st.gpu_ms = ms;
    st.kernel_launches = wc.launches;
    st.waves = wc.waves;
    st.samples_per_wave = plan.spw;
    if (timing) {
        for (size_t w = 0; w + per_wave <= wc.events; w += per_wave) {
            auto el = [&](size_t a) {
                float x = 0.0f;
                cudaEventElapsedTime(&x, r->events[w + a], r->events[w + a + 1]);
                return x;
            };
            st.raygen_ms += el(0);
            for (uint32_t b = 0; b < r->max_bounces; ++b) {
                st.intersect_ms += el(1 + 3 * b);
                st.shade_ms += el(2 + 3 * b);
                st.shadow_ms += el(3 + 3 * b);
            }
            st.film_ms += el(1 + 3 * r->max_bounces);
        }
    }
    r->stats = st;
    for (int k = 0; k < 6; ++k) r->tally_prev[k] = t[k];
    if (t[2]) return fail(CENOTE_E_OVERFLOW, "a traversal stack or queue bound was exceeded");
    return CENOTE_OK;
}

}  // namespace

int32_t cenote_renderer_autotune(cenote_renderer* r, cenote_scene* scene, uint32_t width, uint32_t height,
                                 cenote_tuning* out) {
    CN_CHECK(r && scene && width > 0 && height > 0, CENOTE_E_INVALID_ARGUMENT, "null handle or empty target");
    CN_CHECK(r->ctx == scene->ctx, CENOTE_E_INVALID_ARGUMENT, "handles from different contexts");
    cenote_film* film = nullptr;
    int32_t rc = cenote_film_create(r->ctx, width, height, &film);
    if (rc != CENOTE_OK) return rc;
    std::unique_ptr<cenote_film, void (*)(cenote_film*)> hold(film, cenote_film_destroy);
    std::lock_guard<std::mutex> lock(r->ctx->mu);
    CN_CUDA(cudaSetDevice(r->ctx->device));
    const uint64_t pixels = uint64_t(width) * height;
    // The automatic wave size (plan_waves), its half, and 2x, 4x and 8x,
    // bounded by 64 M paths (about 16 GB of path state).
    const uint32_t auto_spw = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>((uint64_t(1) << 24) / pixels, 64)));
    const uint32_t spw_cap = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>((uint64_t(1) << 26) / pixels, 256)));
    const uint32_t spws[5] = {0, std::max(1u, auto_spw / 2), std::min(spw_cap, auto_spw * 2),
                              std::min(spw_cap, auto_spw * 4), std::min(spw_cap, auto_spw * 8)};
    // Probe length: two waves of the largest candidate, at most ~128 M samples.
    uint32_t probe = std::max(2u, 2 * spws[4]);
    while (probe > 2 && pixels * probe > (uint64_t(1) << 27)) probe /= 2;
    const uint32_t saved_profiling = r->profiling;
    r->profiling = 0;
    cenote_tuning best{r->material_sort,
                       r->samples_per_wave,
                       r->refill_idle,
                       r->top_nodes,
                       r->l2_window,
                       r->per_lane_triangles,
                       0.0f,
                       uint32_t(TRAV_VARIANT_BLOCK[r->trav_variant]),
                       uint32_t(TRAV_VARIANT_STACK[r->trav_variant]),
                       r->sort_by_location};
    auto apply = [&](const cenote_tuning& t) {
        r->material_sort = t.material_sort;
        r->samples_per_wave = t.samples_per_wave;
        r->refill_idle = t.refill_idle;
        r->top_nodes = t.top_nodes;
        r->l2_window = t.l2_window;
        r->per_lane_triangles = t.per_lane_triangles;
        r->trav_variant = trav_variant_of(t.block_size, t.stack_depth);
        r->sort_by_location = t.sort_by_location;
    };
    // Device time of `probe` samples, the better of two runs (the first run of
    // a new wave size also allocates).
    auto measure = [&](const cenote_tuning& t, float* ms) -> int32_t {
        apply(t);
        float m = 1e30f;
        for (int k = 0; k < 2; ++k) {
            int32_t e = run_waves(r, scene, width, height, 1u << 30, probe, film, nullptr);
            if (e != CENOTE_OK) return e;
            m = std::min(m, r->stats.gpu_ms);
        }
        *ms = m;
        return CENOTE_OK;
    };
    float best_ms = 0.0f;
    rc = measure(best, &best_ms);
    // An all-opaque scene chooses between the warp triangle queue and per-lane
    // tests (fractional opacity always tests per lane); the 16-entry stack is
    // a candidate only when the tree's node groups fit it.
    const bool short_stack = TRAVERSAL_STACK_DEPTH - int(scene->ds.stack_room) < 16;
    // The sort mode and the sort's key are searched together (the key
    // changes which mode pays): none, every bounce or from the first bounce
    // on, each sorted mode keyed by instance or by location.
    for (int knob = 0; knob < 8 && rc == CENOTE_OK; ++knob) {
        if (knob == 5 && scene->ds.has_nonopaque) continue;
        if (knob == 7 && !short_stack) continue;
        for (int c = 0; c < (knob == 0 ? 5 : (knob == 1 ? 5 : (knob >= 4 ? 2 : 3))) && rc == CENOTE_OK; ++c) {
            cenote_tuning t = best;
            if (knob == 0) {
                t.material_sort = c == 0 ? CENOTE_SORT_NONE : (c % 2 ? CENOTE_SORT_ALL : CENOTE_SORT_SECONDARY);
                t.sort_by_location = c >= 3 ? 1u : 0u;
            }
            if (knob == 1) t.samples_per_wave = spws[c];
            if (knob == 2) t.refill_idle = c == 0 ? 4u : (c == 1 ? 8u : 16u);
            if (knob == 3) t.top_nodes = c == 0 ? 0u : (c == 1 ? 80u : TOP_NODES_MAX);
            if (knob == 4) t.l2_window = uint32_t(c);
            if (knob == 5) t.per_lane_triangles = uint32_t(c);
            if (knob == 6) t.block_size = c == 0 ? 128u : 256u;
            if (knob == 7) t.stack_depth = c == 0 ? 32u : 16u;
            if (t.material_sort == best.material_sort && t.samples_per_wave == best.samples_per_wave &&
                t.refill_idle == best.refill_idle && t.top_nodes == best.top_nodes && t.l2_window == best.l2_window &&
                t.per_lane_triangles == best.per_lane_triangles && t.block_size == best.block_size &&
                t.stack_depth == best.stack_depth && t.sort_by_location == best.sort_by_location)
                continue;
            float ms = 0.0f;
            rc = measure(t, &ms);
            if (rc == CENOTE_OK && ms < best_ms) {
                best = t;
                best_ms = ms;
            }
        }
    }
    r->profiling = saved_profiling;
    apply(best);
    if (rc != CENOTE_OK) return rc;
    best.ms_per_sample = best_ms / float(probe);
    r->tuned_ms_per_sample = best.ms_per_sample;
    if (out) *out = best;
    return CENOTE_OK;
}

int32_t cenote_accumulate_n(cenote_renderer* r, cenote_scene* scene, cenote_film* film, uint32_t count) {
    CN_CHECK(r && scene && film, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(r->ctx == scene->ctx && r->ctx == film->ctx, CENOTE_E_INVALID_ARGUMENT, "handles from different contexts");
    if (count == 0) return CENOTE_OK;
    std::lock_guard<std::mutex> lock(r->ctx->mu);
    CN_CUDA(cudaSetDevice(r->ctx->device));
    int32_t rc = run_waves(r, scene, film->width, film->height, film->samples, count, film, nullptr);
    if (rc == CENOTE_OK) film->samples += count;
    return rc;
}

int32_t cenote_accumulate_range(cenote_renderer* r, cenote_scene* scene, cenote_film* film, uint32_t first_sample,
                                uint32_t count) {
    CN_CHECK(r && scene && film, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(r->ctx == scene->ctx && r->ctx == film->ctx, CENOTE_E_INVALID_ARGUMENT, "handles from different contexts");
    CN_CHECK(uint64_t(first_sample) + count <= 0xffffffffull, CENOTE_E_INVALID_ARGUMENT, "sample index overflow");
    if (count == 0) return CENOTE_OK;
    std::lock_guard<std::mutex> lock(r->ctx->mu);
    CN_CUDA(cudaSetDevice(r->ctx->device));
    int32_t rc = run_waves(r, scene, film->width, film->height, first_sample, count, film, nullptr);
    if (rc == CENOTE_OK) film->samples += count;
    return rc;
}

int32_t cenote_accumulate(cenote_renderer* r, cenote_scene* scene, cenote_film* film) {
    return cenote_accumulate_n(r, scene, film, 1);
}

int32_t cenote_render_once(cenote_renderer* r, cenote_scene* scene, uint32_t width, uint32_t height, uint32_t sample,
                           float* rgba_out) {
    CN_CHECK(r && scene && rgba_out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(width > 0 && height > 0, CENOTE_E_INVALID_ARGUMENT, "zero-sized trace target");
    CN_CHECK(uint64_t(width) * height < (1ull << 31), CENOTE_E_INVALID_ARGUMENT, "target too large");
    std::lock_guard<std::mutex> lock(r->ctx->mu);
    CN_CUDA(cudaSetDevice(r->ctx->device));
    DeviceBuffer out;
    size_t bytes = size_t(width) * height * 16;
    CN_CUDA(out.alloc(bytes));
    int32_t rc = run_waves(r, scene, width, height, sample, 1, nullptr, out.as<float4>());
    if (rc != CENOTE_OK) return rc;
    CN_CUDA(cudaMemcpy(rgba_out, out.ptr, bytes, cudaMemcpyDeviceToHost));
    return CENOTE_OK;
}

int32_t cenote_film_averages(cenote_film* film, float* beauty, float* albedo, float* normal, float* depth) {
    CN_CHECK(film, CENOTE_E_INVALID_ARGUMENT, "null film");
    std::lock_guard<std::mutex> lock(film->ctx->mu);
    CN_CUDA(cudaSetDevice(film->ctx->device));
    size_t px = size_t(film->width) * film->height;
    if (beauty) {
        launch_resolve(film->sum.as<float4>(), film->avg.as<float4>(), uint32_t(px), float(std::max(1u, film->samples)),
                       film->ctx->stream);
        CN_CUDA(cudaGetLastError());
        CN_CUDA(cudaMemcpyAsync(beauty, film->avg.ptr, px * 16, cudaMemcpyDeviceToHost, film->ctx->stream));
    }
    const float n = float(std::max(1u, film->samples));
    float4* avg = film->avg.as<float4>();
    for (auto [src, dst] : {std::pair<float4*, float*>{film->albedo.as<float4>(), albedo},
                            std::pair<float4*, float*>{film->normal.as<float4>(), normal}}) {
        if (!dst) continue;
        launch_resolve(src, avg, uint32_t(px), n, film->ctx->stream);
        CN_CUDA(cudaGetLastError());
        CN_CUDA(cudaMemcpyAsync(dst, avg, px * 16, cudaMemcpyDeviceToHost, film->ctx->stream));
    }
    if (depth) {
        launch_resolve1(film->depth.as<float>(), film->avg.as<float>(), uint32_t(px), n, film->ctx->stream);
        CN_CUDA(cudaGetLastError());
        CN_CUDA(cudaMemcpyAsync(depth, film->avg.ptr, px * 4, cudaMemcpyDeviceToHost, film->ctx->stream));
    }
    return wait_stream(film->ctx->stream, film->ctx->sync_ev, 600000.0);
}

int32_t cenote_film_tonemap_device(cenote_film* film, float exposure_stops, void* rgba8) {
    CN_CHECK(film && rgba8, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(film->samples > 0, CENOTE_E_INVALID_ARGUMENT, "tonemapping an empty film");
    CN_CUDA(cudaSetDevice(film->ctx->device));
    const uint32_t px = film->width * film->height;
    launch_resolve(film->sum.as<float4>(), film->avg.as<float4>(), px, float(film->samples), film->ctx->stream);
    launch_tonemap(film->avg.as<float4>(), static_cast<uint32_t*>(rgba8), px, std::exp2(exposure_stops),
                   film->ctx->stream);
    CN_CUDA(cudaGetLastError());
    return CENOTE_OK;
}

int32_t cenote_film_tonemap(cenote_film* film, float exposure_stops, uint32_t* rgba8) {
    CN_CHECK(film && rgba8, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(film->samples > 0, CENOTE_E_INVALID_ARGUMENT, "tonemapping an empty film");
    std::lock_guard<std::mutex> lock(film->ctx->mu);
    CN_CUDA(cudaSetDevice(film->ctx->device));
    const size_t px = size_t(film->width) * film->height;
    DeviceBuffer out;
    CN_CUDA(out.alloc(px * 4));
    int32_t rc = cenote_film_tonemap_device(film, exposure_stops, out.ptr);
    if (rc != CENOTE_OK) return rc;
    CN_CUDA(cudaMemcpyAsync(rgba8, out.ptr, px * 4, cudaMemcpyDeviceToHost, film->ctx->stream));
    return wait_stream(film->ctx->stream, film->ctx->sync_ev, 600000.0);
}

int32_t cenote_film_sums(cenote_film* film, float* beauty_sum) {
    CN_CHECK(film && beauty_sum, CENOTE_E_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(film->ctx->mu);
    CN_CUDA(cudaSetDevice(film->ctx->device));
    CN_CUDA(cudaMemcpyAsync(beauty_sum, film->sum.ptr, size_t(film->width) * film->height * 16, cudaMemcpyDeviceToHost,
                            film->ctx->stream));
    return wait_stream(film->ctx->stream, film->ctx->sync_ev, 600000.0);
}

int32_t cenote_film_restore(cenote_film* film, const float* beauty_sum, uint32_t samples) {
    CN_CHECK(film && beauty_sum, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(samples > 0, CENOTE_E_INVALID_ARGUMENT, "a restored film holds at least one sample");
    std::lock_guard<std::mutex> lock(film->ctx->mu);
    int32_t rc = cenote_film_reset(film);
    if (rc != CENOTE_OK) return rc;
    CN_CUDA(cudaMemcpyAsync(film->sum.ptr, beauty_sum, size_t(film->width) * film->height * 16, cudaMemcpyHostToDevice,
                            film->ctx->stream));
    rc = wait_stream(film->ctx->stream, film->ctx->sync_ev, 600000.0);
    if (rc == CENOTE_OK) film->samples = samples;
    return rc;
}

// ---- probes ------------------------------------------------------------------------------

}  // extern "C"

namespace {
template <class F>
int32_t with_device_io(cenote_context* ctx, std::vector<std::pair<const void*, size_t>> in,
                       std::vector<std::pair<void*, size_t>> out, F&& launch) {
    std::vector<std::unique_ptr<DeviceBuffer>> din, dout;
    std::vector<void*> pin, pout;
    for (auto& b : in) {
        din.push_back(std::make_unique<DeviceBuffer>());
        CN_CUDA(din.back()->alloc(b.second));
        CN_CUDA(cudaMemcpyAsync(din.back()->ptr, b.first, b.second, cudaMemcpyHostToDevice, ctx->stream));
        pin.push_back(din.back()->ptr);
    }
    for (auto& b : out) {
        dout.push_back(std::make_unique<DeviceBuffer>());
        CN_CUDA(dout.back()->alloc(b.second));
        CN_CUDA(cudaMemsetAsync(dout.back()->ptr, 0, b.second, ctx->stream));
        pout.push_back(dout.back()->ptr);
    }
    launch(pin, pout);
    CN_CUDA(cudaGetLastError());
    for (size_t i = 0; i < out.size(); ++i)
        CN_CUDA(cudaMemcpyAsync(out[i].first, pout[i], out[i].second, cudaMemcpyDeviceToHost, ctx->stream));
    return wait_stream(ctx->stream, ctx->sync_ev, 600000.0);
}
}  // namespace

extern "C" {

int32_t cenote_probe_sampler(cenote_context* ctx, uint32_t pixel, uint32_t dimension, uint32_t count, float* points,
                             float* values) {
    CN_CHECK(ctx && points && values, CENOTE_E_INVALID_ARGUMENT, "null argument");
    if (count == 0) return CENOTE_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    return with_device_io(ctx, {}, {{points, size_t(count) * 8}, {values, size_t(count) * 4}},
                          [&](std::vector<void*>&, std::vector<void*>& o) {
                              probe_sampler(pixel, dimension, count, static_cast<float2*>(o[0]), static_cast<float*>(o[1]),
                                            ctx->stream);
                          });
}

int32_t cenote_probe_bsdf(cenote_context* ctx, const cenote_material* m, const float* wo, const float* wi, uint32_t n,
                          uint32_t exiting, float* f, float* pdf) {
    CN_CHECK(ctx && m && wo && wi && f && pdf, CENOTE_E_INVALID_ARGUMENT, "null argument");
    if (n == 0) return CENOTE_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    return with_device_io(ctx, {{wo, size_t(n) * 12}, {wi, size_t(n) * 12}}, {{f, size_t(n) * 12}, {pdf, size_t(n) * 4}},
                          [&](std::vector<void*>& i, std::vector<void*>& o) {
                              probe_bsdf(ctx->tables.as<float>(), *m, static_cast<float3*>(i[0]),
                                         static_cast<float3*>(i[1]), n, exiting, static_cast<float3*>(o[0]),
                                         static_cast<float*>(o[1]), ctx->stream);
                          });
}

int32_t cenote_probe_bsdf_sample(cenote_context* ctx, const cenote_material* m, const float* wo, const float* u,
                                 uint32_t n, uint32_t exiting, float* wi, float* pdf, uint32_t* lobe) {
    CN_CHECK(ctx && m && wo && u && wi && pdf && lobe, CENOTE_E_INVALID_ARGUMENT, "null argument");
    if (n == 0) return CENOTE_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    return with_device_io(ctx, {{wo, size_t(n) * 12}, {u, size_t(n) * 12}},
                          {{wi, size_t(n) * 12}, {pdf, size_t(n) * 4}, {lobe, size_t(n) * 4}},
                          [&](std::vector<void*>& i, std::vector<void*>& o) {
                              probe_bsdf_sample(ctx->tables.as<float>(), *m, static_cast<float3*>(i[0]),
                                                static_cast<float3*>(i[1]), n, exiting, static_cast<float3*>(o[0]),
                                                static_cast<float*>(o[1]), static_cast<uint32_t*>(o[2]), ctx->stream);
                          });
}

static int32_t probe_closest(cenote_scene* sc, const float* origins, const float* directions, uint32_t n,
                             uint32_t* hits, float* t, bool queued) {
    CN_CHECK(sc && origins && directions && hits && t, CENOTE_E_INVALID_ARGUMENT, "null argument");
    if (n == 0) return CENOTE_OK;
    cenote_context* ctx = sc->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    uint32_t flag = 0;
    int32_t rc = with_device_io(ctx, {{origins, size_t(n) * 12}, {directions, size_t(n) * 12}},
                                {{hits, size_t(n) * 16}, {t, size_t(n) * 4}, {&flag, 4}},
                                [&](std::vector<void*>& i, std::vector<void*>& o) {
                                    auto probe = queued ? probe_intersect_queued : probe_intersect;
                                    probe(sc->ds, static_cast<float3*>(i[0]), static_cast<float3*>(i[1]), n,
                                          static_cast<uint4*>(o[0]), static_cast<float*>(o[1]),
                                          static_cast<uint32_t*>(o[2]), ctx->stream);
                                });
    if (rc == CENOTE_OK && flag) return fail(CENOTE_E_OVERFLOW, "traversal bound exceeded");
    return rc;
}

int32_t cenote_probe_intersect(cenote_scene* sc, const float* origins, const float* directions, uint32_t n,
                               uint32_t* hits, float* t) {
    return probe_closest(sc, origins, directions, n, hits, t, false);
}

int32_t cenote_probe_intersect_queued(cenote_scene* sc, const float* origins, const float* directions, uint32_t n,
                                      uint32_t* hits, float* t) {
    return probe_closest(sc, origins, directions, n, hits, t, true);
}

static int32_t probe_shadows(cenote_scene* sc, const float* origins, const float* directions, const float* tmax,
                             const uint32_t* targets, uint32_t n, float* out, bool queued) {
    CN_CHECK(sc && origins && directions && tmax && targets && out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(!queued || !sc->ds.has_nonopaque, CENOTE_E_INVALID_ARGUMENT,
             "the queued shadow walk serves scenes whose triangles are all opaque");
    if (n == 0) return CENOTE_OK;
    cenote_context* ctx = sc->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    uint32_t flag = 0;
    int32_t rc = with_device_io(
        ctx, {{origins, size_t(n) * 12}, {directions, size_t(n) * 12}, {tmax, size_t(n) * 4}, {targets, size_t(n) * 8}},
        {{out, size_t(n) * 4}, {&flag, 4}}, [&](std::vector<void*>& i, std::vector<void*>& o) {
            auto probe = queued ? probe_shadow_queued : probe_shadow;
            probe(sc->ds, static_cast<float3*>(i[0]), static_cast<float3*>(i[1]), static_cast<float*>(i[2]),
                  static_cast<uint2*>(i[3]), n, static_cast<float*>(o[0]), static_cast<uint32_t*>(o[1]), ctx->stream);
        });
    if (rc == CENOTE_OK && flag) return fail(CENOTE_E_OVERFLOW, "traversal bound exceeded");
    return rc;
}

int32_t cenote_probe_shadow(cenote_scene* sc, const float* origins, const float* directions, const float* tmax,
                            const uint32_t* targets, uint32_t n, float* out) {
    return probe_shadows(sc, origins, directions, tmax, targets, n, out, false);
}

int32_t cenote_probe_shadow_queued(cenote_scene* sc, const float* origins, const float* directions,
                                   const float* tmax, const uint32_t* targets, uint32_t n, float* out) {
    return probe_shadows(sc, origins, directions, tmax, targets, n, out, true);
}

int32_t cenote_probe_env_sample(cenote_scene* sc, const float* u, uint32_t n, float* directions, float* pdf,
                                uint32_t* row_col) {
    CN_CHECK(sc && u && directions && pdf && row_col, CENOTE_E_INVALID_ARGUMENT, "null argument");
    if (n == 0) return CENOTE_OK;
    cenote_context* ctx = sc->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    return with_device_io(ctx, {{u, size_t(n) * 8}},
                          {{directions, size_t(n) * 12}, {pdf, size_t(n) * 4}, {row_col, size_t(n) * 8}},
                          [&](std::vector<void*>& i, std::vector<void*>& o) {
                              probe_env_sample(sc->ds, static_cast<float2*>(i[0]), n, static_cast<float3*>(o[0]),
                                               static_cast<float*>(o[1]), static_cast<uint2*>(o[2]), ctx->stream);
                          });
}

int32_t cenote_probe_env_pdf(cenote_scene* sc, const float* directions, uint32_t n, float* pdf) {
    CN_CHECK(sc && directions && pdf, CENOTE_E_INVALID_ARGUMENT, "null argument");
    if (n == 0) return CENOTE_OK;
    cenote_context* ctx = sc->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    return with_device_io(ctx, {{directions, size_t(n) * 12}}, {{pdf, size_t(n) * 4}},
                          [&](std::vector<void*>& i, std::vector<void*>& o) {
                              probe_env_pdf(sc->ds, static_cast<float3*>(i[0]), n, static_cast<float*>(o[0]),
                                            ctx->stream);
                          });
}

int32_t cenote_probe_texture(cenote_scene* sc, uint32_t index, uint32_t mode, const float* uv, uint32_t n, float* rgba) {
    CN_CHECK(sc && uv && rgba, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(index < sc->ds.texture_count, CENOTE_E_INVALID_ARGUMENT, "texture index out of range");
    CN_CHECK(mode <= 3, CENOTE_E_INVALID_ARGUMENT, "unknown probe mode");
    if (n == 0) return CENOTE_OK;
    cenote_context* ctx = sc->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    return with_device_io(ctx, {{uv, size_t(n) * 8}}, {{rgba, size_t(n) * 16}},
                          [&](std::vector<void*>& i, std::vector<void*>& o) {
                              probe_texture(sc->ds, index, mode, static_cast<float2*>(i[0]), n,
                                            static_cast<float4*>(o[0]), ctx->stream);
                          });
}

// ---- texture prep ----------------------------------------------------------------------

uint64_t cenote_texture_bytes(uint32_t format, uint32_t width, uint32_t height) {
    return texture_bytes(format, width, height);
}

int32_t cenote_texture_encode(uint32_t format, const uint8_t* rgba8, uint32_t width, uint32_t height, void* out) {
    CN_CHECK(rgba8 && out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(texture_encode(format, rgba8, width, height, static_cast<uint8_t*>(out)), CENOTE_E_INVALID_ARGUMENT,
             "not a BC format, or a size it cannot take (BC extents are multiples of 4)");
    return CENOTE_OK;
}

int32_t cenote_texture_encode_float(uint32_t format, const float* rgba32f, uint32_t width, uint32_t height,
                                    void* out) {
    CN_CHECK(rgba32f && out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(texture_encode_float(format, rgba32f, width, height, static_cast<uint8_t*>(out)),
             CENOTE_E_INVALID_ARGUMENT, "not BC6H unsigned, or a size it cannot take (extents are multiples of 4)");
    return CENOTE_OK;
}

// ---- environment tables without device allocation ------------------------------------

int32_t cenote_env_tables_static(cenote_context* ctx, const float* texels, uint32_t width, uint32_t height,
                                 float* marginal, float* conditional, float* pdfs, double* power) {
    CN_CHECK(ctx && texels && marginal && conditional && pdfs, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(width > 0 && height > 0, CENOTE_E_INVALID_ARGUMENT, "zero-sized environment");
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    double* scratch = nullptr;
    size_t max_texels = 0;
    uint32_t max_rows = 0;
    cudaEvent_t done = nullptr;
    CN_CUDA(static_env_scratch(ctx->device, &scratch, &max_texels, &max_rows, &done));
    if (static_env_pending(ctx->device)) {
        // An earlier call on this device returned before its work finished:
        // that work may still write the scratch.
        int32_t rc = wait_event(done, 600000.0);
        if (rc == CENOTE_E_TIMEOUT)
            return fail(CENOTE_E_TIMEOUT, "an earlier allocation-free environment build on this device is still running");
        if (rc != CENOTE_OK) return rc;
        static_env_set_pending(ctx->device, false);
    }
    const size_t n = size_t(width) * height;
    CN_CHECK(n <= max_texels && height <= max_rows, CENOTE_E_INVALID_ARGUMENT,
             "environment " + std::to_string(width) + "x" + std::to_string(height) +
                 " exceeds the allocation-free build's limit of " + std::to_string(max_texels) + " texels and " +
                 std::to_string(max_rows) + " rows");
    // Row constants from the host's libm, as the allocating build computes them.
    std::vector<double> rows(2 * size_t(height));
    const double PI = 3.141592653589793;
    for (uint32_t r = 0; r < height; ++r) {
        rows[r] = std::sin((double(r) + 0.5) / double(height) * PI);
        double th0 = double(r) / double(height) * PI, th1 = double(r + 1) / double(height) * PI;
        rows[height + r] = 2.0 * PI / double(width) * (std::cos(th0) - std::cos(th1));
    }
    double* totals = scratch + 2 * n + 2 * size_t(height);
    double* row_consts = totals + 2;
    CN_CUDA(cudaMemcpyAsync(row_consts, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    launch_env_tables(reinterpret_cast<const float4*>(texels), row_consts, row_consts + height, width, height, scratch,
                      marginal, conditional, pdfs, totals, ctx->stream);
    CN_CUDA(cudaGetLastError());
    double host_totals[2] = {0.0, 0.0};
    CN_CUDA(cudaMemcpyAsync(host_totals, totals, sizeof host_totals, cudaMemcpyDeviceToHost, ctx->stream));
    int32_t rc = wait_stream(ctx->stream, done, 600000.0);
    if (rc == CENOTE_E_TIMEOUT) static_env_set_pending(ctx->device, true);
    if (rc != CENOTE_OK) return rc;
    if (power) *power = host_totals[1];
    return CENOTE_OK;
}

}  // extern "C"
