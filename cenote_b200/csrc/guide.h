// The learned directional guide: shapes, parameter layout, the vMF mixture
// head (shared by the training kernels and guided sampling in the shading
// kernel) and the launchers of guide.cu.
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cn {
namespace guide {

constexpr uint32_t IN = 96;       // encoded inputs (81 used, zero padded to a multiple of 16)
constexpr uint32_t HIDDEN = 64;
constexpr uint32_t LOBES = 8;
constexpr uint32_t OUT = 5 * LOBES;  // per lobe: raw direction (3), raw concentration, logit
constexpr uint32_t OUT_PAD = 48;     // the last layer's MMA width
// The mixture as shading reads it, activated once per vertex by inference:
// six groups of LOBES floats (mu.x, mu.y, mu.z, kappa, weight, and the vMF
// normalisation kappa / (2 pi (1 - e^{-2 kappa}))), 16-byte aligned groups.
constexpr uint32_t OUT_ACT = 6 * LOBES;
constexpr uint32_t TILE = 128;       // rows per CTA tile (the MMA's M)
constexpr uint32_t ACT = IN + 3 * HIDDEN;  // saved activations per row (BF16)
constexpr uint32_t FREQS = 12;       // frequency bands of the position encoding

// FP32 parameters, row-major [out][in] weights followed by their bias.
constexpr uint32_t P_W1 = 0, P_B1 = P_W1 + HIDDEN * IN;
constexpr uint32_t P_W2 = P_B1 + HIDDEN, P_B2 = P_W2 + HIDDEN * HIDDEN;
constexpr uint32_t P_W3 = P_B2 + HIDDEN, P_B3 = P_W3 + HIDDEN * HIDDEN;
constexpr uint32_t P_W4 = P_B3 + HIDDEN, P_B4 = P_W4 + OUT * HIDDEN;
constexpr uint32_t PARAMS = P_B4 + OUT;  // 17,128

struct Buffers {
    float* params;  // FP32 master weights
    float* grad;
    float* m;
    float* v;
    __nv_bfloat16 *w1, *w2, *w3, *w4;  // BF16 copies (w4 padded to OUT_PAD rows)
    float* b4;                          // last bias padded to OUT_PAD
    int* err;                           // set when a tensor-core wait ran out
};

// ---- the mixture head -----------------------------------------------------------------

struct Lobe {
    float3 mu;
    float kappa;
    float norm;  // |raw direction|, for the gradient through the normalisation
};

// Lobe i from its five raw outputs: mu = r / |r|, kappa = 0.01 + softplus(x).
__host__ __device__ inline Lobe lobe(const float* o) {
    Lobe L;
    float n = sqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] + 1e-12f);
    L.norm = n;
    L.mu = make_float3(o[0] / n, o[1] / n, o[2] / n);
    float x = fminf(fmaxf(o[3], -20.0f), 20.0f);
    L.kappa = 0.01f + log1pf(expf(x));
    return L;
}

// vMF density on the sphere: kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (cos - 1)}.
__host__ __device__ inline float vmf_pdf(float kappa, float cosw) {
    return kappa / (6.283185307f * (1.0f - expf(-2.0f * kappa))) * expf(kappa * (cosw - 1.0f));
}

struct MixtureGrad {
    float d[OUT];  // d(-weight log q(w)) / d(raw outputs)
    float log_q;
};

// ---- inputs ------------------------------------------------------------------------------

// The encoded inputs of one vertex: position p (in [0,1]^3 of the scene's
// bounds) in FREQS sine/cosine bands per axis, then n, wo and p; zero padded.
__host__ __device__ inline void encode(float3 p, float3 n, float3 wo, float* f) {
    const float c[3] = {p.x, p.y, p.z};
    uint32_t k = 0;
    for (uint32_t b = 0; b < FREQS; ++b) {
        const float s = 3.14159265f * float(1u << b);
        for (int a = 0; a < 3; ++a) {
            float sv, cv;
#ifdef __CUDA_ARCH__
            __sincosf(s * c[a], &sv, &cv);
#else
            sv = sinf(s * c[a]);
            cv = cosf(s * c[a]);
#endif
            f[k++] = sv;
            f[k++] = cv;
        }
    }
    f[k++] = n.x;
    f[k++] = n.y;
    f[k++] = n.z;
    f[k++] = wo.x;
    f[k++] = wo.y;
    f[k++] = wo.z;
    f[k++] = p.x;
    f[k++] = p.y;
    f[k++] = p.z;
    while (k < IN) f[k++] = 0.0f;
}

// One training record: a guided-mode surface vertex, 64 bytes.
//   q0 = (position, pdf of the sampled direction; the target weight once resolved)
//   q1 = (shading normal, luminance of the throughput after the scatter)
//   q2 = (outgoing direction, luminance of the path's radiance before the next vertex; < 0 until known)
//   q3 = (sampled direction, path index as bits)
struct Record {
    float4 q0, q1, q2, q3;
};

// ---- the mixture at a vertex, from its raw outputs -------------------------------------------
#ifdef __CUDACC__

// Lobe weights by softmax of the logits (o[5i + 4]).
__device__ inline void lobe_weights(const float* o, float* w) {
    float m = -1e30f;
    for (int i = 0; i < LOBES; ++i) m = fmaxf(m, o[5 * i + 4]);
    float s = 0.0f;
    for (int i = 0; i < LOBES; ++i) {
        w[i] = __expf(o[5 * i + 4] - m);
        s += w[i];
    }
    for (int i = 0; i < LOBES; ++i) w[i] /= s;
}


// The activated mixture (OUT_ACT layout) from the raw outputs: the lobes'
// means, concentrations, softmax weights and vMF normalisations, computed
// as lobe(), lobe_weights() and vmf_pdf() compute them.
__device__ inline void activate(const float* o, float* a) {
    float w[LOBES];
    lobe_weights(o, w);
    for (uint32_t i = 0; i < LOBES; ++i) {
        Lobe L = lobe(o + 5 * i);
        a[i] = L.mu.x;
        a[LOBES + i] = L.mu.y;
        a[2 * LOBES + i] = L.mu.z;
        a[3 * LOBES + i] = L.kappa;
        a[4 * LOBES + i] = w[i];
        a[5 * LOBES + i] = L.kappa / (6.283185307f * (1.0f - expf(-2.0f * L.kappa)));
    }
}

// The mixture's density at direction d: the sum over lobes of weight times
// the vMF density (vmf_pdf), read from the activated layout.
__device__ inline float mixture_pdf_act(const float* a, float3 d) {
    float q = 0.0f;
    for (uint32_t i = 0; i < LOBES; ++i) {
        const float cosw = a[i] * d.x + a[LOBES + i] * d.y + a[2 * LOBES + i] * d.z;
        const float kappa = a[3 * LOBES + i];
        q += a[4 * LOBES + i] * (a[5 * LOBES + i] * expf(kappa * (cosw - 1.0f)));
    }
    return q;
}

// A direction from the mixture: lobe by u_lobe, then the vMF around its mean
// (inverse-cdf cos theta = 1 + log(u + (1 - u) e^{-2 kappa}) / kappa).
__device__ inline float3 mixture_sample_act(const float* a, float u_lobe, float u1, float u2) {
    int pick = LOBES - 1;
    float acc = 0.0f;
    for (int i = 0; i < int(LOBES); ++i) {
        acc += a[4 * LOBES + i];
        if (u_lobe < acc) {
            pick = i;
            break;
        }
    }
    const float kappa = a[3 * LOBES + pick];
    float ct = 1.0f + logf(u1 + (1.0f - u1) * __expf(-2.0f * kappa)) / kappa;
    ct = fminf(fmaxf(ct, -1.0f), 1.0f);
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float sp, cp;
    __sincosf(6.283185307f * u2, &sp, &cp);
    // Frame around mu (Duff et al. 2017).
    float3 n = make_float3(a[pick], a[LOBES + pick], a[2 * LOBES + pick]);
    float sg = n.z >= 0.0f ? 1.0f : -1.0f;
    float aa = -1.0f / (sg + n.z);
    float b = n.x * n.y * aa;
    float3 t = make_float3(1.0f + sg * n.x * n.x * aa, sg * b, -sg * n.x);
    float3 bt = make_float3(b, sg + n.y * n.y * aa, -n.y);
    return make_float3(st * cp * t.x + st * sp * bt.x + ct * n.x, st * cp * t.y + st * sp * bt.y + ct * n.y,
                       st * cp * t.z + st * sp * bt.z + ct * n.z);
}

#endif  // __CUDACC__

// ---- launchers (guide.cu) -----------------------------------------------------------------

cudaError_t configure(int device, int* sms);
void launch_cast(const Buffers& b, cudaStream_t s);
// out[rows][OUT] from FP32 features [rows][IN]; `save` (nullable) [rows][ACT].
void launch_forward(const Buffers& b, const float* feats, uint32_t rows, float* out, __nv_bfloat16* save, int sms,
                    cudaStream_t s);
// dz4[rows][OUT_PAD] = d(mean_s -w_s log q(dir_s))/d(out), loss += the mean.
void launch_loss(const Buffers& b, const float* out, const float* dirs, const float* weights, uint32_t rows,
                 float inv_batch, __nv_bfloat16* dz4, float* loss, cudaStream_t s);
// b.grad += dL/dparams through the saved activations.
void launch_backward(const Buffers& b, const __nv_bfloat16* save, const __nv_bfloat16* dz4, uint32_t rows, int sms,
                     cudaStream_t s);
// One Adam step (beta 0.9 / 0.999), zeroing the gradient.
void launch_adam(const Buffers& b, float lr, uint32_t step, cudaStream_t s);

}  // namespace guide

struct DeviceScene;
struct PathPool;

namespace guide {

// The activated mixture (OUT_ACT floats) of every hit path of `bounce` into pool.guide_out.
void launch_infer_paths(const Buffers& b, const DeviceScene& scene, const PathPool& pool, uint32_t bounce,
                        uint32_t n0, int sms, cudaStream_t s);
// Turn the wave's records into target weights L / pdf (L from the paths'
// final radiance and the snapshot the next vertex took).
void launch_resolve_records(Record* recs, const uint32_t* count, uint32_t capacity, const float4* rad, cudaStream_t s);

// Scratch of the training steps (device).
struct TrainScratch {
    float* out;            // [rows][OUT]
    __nv_bfloat16* save;   // [rows][ACT]
    __nv_bfloat16* dz4;    // [rows][OUT_PAD]
    float* sums;           // [2]: batch weight sum, loss
    uint32_t rows;
};
// One step on `rows` records starting at `offset` (wrapping over the count).
void launch_train_records(const Buffers& b, const TrainScratch& t, const Record* recs, const uint32_t* count,
                          uint32_t capacity, uint32_t offset, float3 bbox_min, float bbox_inv, float lr,
                          uint32_t step, int sms, cudaStream_t s);

}  // namespace guide
}  // namespace cn
