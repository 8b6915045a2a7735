// The learned directional guide: shapes, parameter layout, the vMF mixture
// head (shared by the training kernels and guided sampling in the shading
// kernel) and the launchers of guide.cu.
#pragma once
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
}  // namespace cn
