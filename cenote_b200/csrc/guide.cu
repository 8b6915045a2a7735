// The learned directional guide: a small MLP (96 encoded inputs -> 3 x 64
// ReLU -> 40 outputs = 8 von Mises-Fisher lobes) evaluated and trained with
// tcgen05 tensor-core kernels, BF16 operands, FP32 accumulation in TMEM.
//
// The reference has no learned guiding; the network, its mixture head and
// the online training objective are this library's. The objective is the
// KL-divergence estimator of neural importance sampling (Müller et al.,
// "Neural Importance Sampling", ACM TOG 2019): for directions w_s drawn with
// pdf p_s and radiance estimates L_s, minimise  -mean_s (L_s / p_s) log q(w_s).
//
// Kernels (one CTA = 128 threads; thread t owns row t of a 128-row tile and
// TMEM lane t):
//  * forward: per tile, features -> shared memory (K-major canonical), then
//    four layers, each = MMAs issued by one thread into a TMEM accumulator,
//    commit to an mbarrier, TMEM -> registers (+bias, ReLU) -> BF16 rows of
//    the next layer's A operand. Optionally saves every activation.
//  * loss: per sample, the mixture, its log-density and dL/d(outputs).
//  * backward: per tile, dZ of each layer, the input gradient dA = dZ W (MMA
//    into a scratch TMEM region) and the weight gradient dW += dZ^T A
//    accumulated across the CTA's tiles in TMEM (M padded to 128 rows), then
//    added into global FP32 gradients once per CTA.
//  * adam: FP32 master weights, BF16 copies for the MMAs.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "guide.h"
#include "records.h"
#include "umma.cuh"
#include "wavefront.h"

namespace cn {
namespace guide {

using umma::kmajor_offset;

namespace {

constexpr uint32_t WAIT_LIMIT = 1u << 24;  // mbarrier polls before giving up

// ---- parameter layout (FP32 master, row-major [out][in]) -----------------------

struct Net {
    const __nv_bfloat16* w[4];  // BF16 copies, row-major [out][in]; w[3] has OUT_PAD rows (40.. zero)
    const float* b[4];          // biases (b[3] has OUT_PAD entries, 40.. zero)
};

__device__ __forceinline__ uint32_t ld_u32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// Pack 8 floats into 8 BF16 (round to nearest even).
__device__ __forceinline__ uint4 pack8(const float* v) {
    uint4 r;
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 c = __floats2bfloat162_rn(v[4], v[5]), d = __floats2bfloat162_rn(v[6], v[7]);
    r.x = *reinterpret_cast<uint32_t*>(&a);
    r.y = *reinterpret_cast<uint32_t*>(&b);
    r.z = *reinterpret_cast<uint32_t*>(&c);
    r.w = *reinterpret_cast<uint32_t*>(&d);
    return r;
}

// Row r of a K-major canonical matrix with `cols` columns from `cols` floats.
__device__ __forceinline__ void store_row(uint8_t* base, uint32_t r, uint32_t cols, const float* v) {
    for (uint32_t c = 0; c < cols; c += 8)
        *reinterpret_cast<uint4*>(base + kmajor_offset(r, c, cols)) = pack8(v + c);
}

// A global row-major BF16 [rows][cols] matrix into a canonical shared one
// (rows beyond `valid` zero), cooperatively.
__device__ void load_matrix(uint8_t* dst, const __nv_bfloat16* src, uint32_t rows, uint32_t valid, uint32_t cols) {
    for (uint32_t i = threadIdx.x; i < rows * (cols / 8); i += blockDim.x) {
        uint32_t r = i / (cols / 8), c = (i % (cols / 8)) * 8;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r < valid) v = *reinterpret_cast<const uint4*>(src + size_t(r) * cols + c);
        *reinterpret_cast<uint4*>(dst + kmajor_offset(r, c, cols)) = v;
    }
}

// The transpose of a row-major BF16 [rows][cols] matrix as a canonical
// [cols][rows] one (so W^T is K-major for the input-gradient MMAs).
__device__ void load_matrix_t(uint8_t* dst, const __nv_bfloat16* src, uint32_t rows, uint32_t cols) {
    for (uint32_t i = threadIdx.x; i < rows * cols; i += blockDim.x) {
        uint32_t r = i / cols, c = i % cols;
        *reinterpret_cast<__nv_bfloat16*>(dst + kmajor_offset(c, r, rows)) = src[size_t(r) * cols + c];
    }
}

// Issue `k / 16` MMAs D = A[128 x k] * B[n x k]^T and commit to `bar`.
__device__ __forceinline__ void issue_layer(uint32_t d_tmem, uint32_t a_base, uint32_t b_base, uint32_t k, uint32_t n,
                                            uint64_t* bar, bool accumulate_first) {
    const uint32_t idesc = umma::idesc_bf16_f32(128, n);
    for (uint32_t k0 = 0; k0 < k; k0 += 16)
        umma::mma_bf16(d_tmem, umma::kslice_desc(a_base, k0, k), umma::kslice_desc(b_base, k0, k), idesc,
                       accumulate_first || k0 > 0);
    umma::commit(bar);
}

// Everyone waits for the MMAs of phase `parity`; false (on every thread) if
// the bound ran out anywhere.
__device__ __forceinline__ bool wait_all(uint64_t* bar, uint32_t parity, int* sflag) {
    if (!umma::mbar_wait(bar, parity, WAIT_LIMIT)) atomicOr(sflag, 1);
    __syncthreads();
    umma::fence_after_sync();
    return *sflag == 0;
}

// This thread's TMEM row, `n` columns from `col`.
__device__ __forceinline__ void read_row(uint32_t tmem, uint32_t col, uint32_t n, float* v) {
    const uint32_t lane = (threadIdx.x / 32u) * 32u;
    for (uint32_t c = 0; c < n; c += 16) umma::tmem_ld16(umma::tmem_at(tmem, lane, col + c), v + c);
    umma::tmem_wait_ld();
}

// ---- shared-memory plan ------------------------------------------------------------

struct FwdSmem {  // offsets in bytes
    static constexpr uint32_t W1 = 0;                               // 64 x 96
    static constexpr uint32_t W2 = W1 + HIDDEN * IN * 2;            // 64 x 64
    static constexpr uint32_t W3 = W2 + HIDDEN * HIDDEN * 2;        // 64 x 64
    static constexpr uint32_t W4 = W3 + HIDDEN * HIDDEN * 2;        // 48 x 64
    static constexpr uint32_t A0 = W4 + OUT_PAD * HIDDEN * 2;       // 128 x 96
    static constexpr uint32_t A1 = A0 + TILE * IN * 2;              // 128 x 64
    static constexpr uint32_t A2 = A1 + TILE * HIDDEN * 2;
    static constexpr uint32_t A3 = A2 + TILE * HIDDEN * 2;
    static constexpr uint32_t BIAS = A3 + TILE * HIDDEN * 2;        // 64 * 3 + 48 floats
    static constexpr uint32_t BAR = BIAS + (3 * HIDDEN + OUT_PAD) * 4;
    static constexpr uint32_t SLOT = BAR + 8;
    static constexpr uint32_t FLAG = SLOT + 4;
    static constexpr uint32_t BYTES = FLAG + 12;
};
static_assert(FwdSmem::A0 % 16 == 0 && FwdSmem::BAR % 8 == 0, "alignment");
static_assert(FwdSmem::BYTES <= 227 * 1024, "shared memory");

__device__ void load_net(uint8_t* smem, const Net& net) {
    load_matrix(smem + FwdSmem::W1, net.w[0], HIDDEN, HIDDEN, IN);
    load_matrix(smem + FwdSmem::W2, net.w[1], HIDDEN, HIDDEN, HIDDEN);
    load_matrix(smem + FwdSmem::W3, net.w[2], HIDDEN, HIDDEN, HIDDEN);
    load_matrix(smem + FwdSmem::W4, net.w[3], OUT_PAD, OUT_PAD, HIDDEN);
    float* bias = reinterpret_cast<float*>(smem + FwdSmem::BIAS);
    for (uint32_t i = threadIdx.x; i < 3 * HIDDEN + OUT_PAD; i += blockDim.x)
        bias[i] = i < 3 * HIDDEN ? net.b[i / HIDDEN][i % HIDDEN] : net.b[3][i - 3 * HIDDEN];
}

// One tile through the network. `feat` holds this thread's row of inputs;
// `out` receives its OUT raw outputs. `save` (nullable) receives the
// activations of the row: A0 (IN), A1..A3 (HIDDEN each) as BF16.
__device__ bool forward_tile(uint8_t* smem, uint32_t tmem, uint32_t& phase, const float* feat, float* out,
                             __nv_bfloat16* save) {
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + FwdSmem::BAR);
    int* sflag = reinterpret_cast<int*>(smem + FwdSmem::FLAG);
    const float* bias = reinterpret_cast<const float*>(smem + FwdSmem::BIAS);
    const uint32_t row = threadIdx.x;
    const uint32_t base = umma::smem_u32(smem);
    store_row(smem + FwdSmem::A0, row, IN, feat);
    if (save)
        for (uint32_t c = 0; c < IN; c += 8)
            *reinterpret_cast<uint4*>(save + c) = *reinterpret_cast<uint4*>(smem + FwdSmem::A0 + kmajor_offset(row, c, IN));
    const uint32_t a_off[4] = {FwdSmem::A0, FwdSmem::A1, FwdSmem::A2, FwdSmem::A3};
    const uint32_t w_off[4] = {FwdSmem::W1, FwdSmem::W2, FwdSmem::W3, FwdSmem::W4};
    float v[HIDDEN];
    for (int l = 0; l < 4; ++l) {
        const uint32_t k = l == 0 ? IN : HIDDEN, n = l == 3 ? OUT_PAD : HIDDEN;
        umma::fence_async_smem();
        umma::fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) {
            umma::fence_after_sync();
            issue_layer(tmem, base + a_off[l], base + w_off[l], k, n, bar, false);
        }
        if (!wait_all(bar, phase, sflag)) return false;
        phase ^= 1u;
        read_row(tmem, 0, n, v);
        const float* bl = bias + l * HIDDEN;
        if (l < 3) {
            for (uint32_t c = 0; c < HIDDEN; ++c) v[c] = fmaxf(v[c] + bl[c], 0.0f);
            store_row(smem + a_off[l + 1], row, HIDDEN, v);
            if (save)
                for (uint32_t c = 0; c < HIDDEN; c += 8)
                    *reinterpret_cast<uint4*>(save + IN + l * HIDDEN + c) =
                        *reinterpret_cast<uint4*>(smem + a_off[l + 1] + kmajor_offset(row, c, HIDDEN));
        } else {
            for (uint32_t c = 0; c < OUT; ++c) out[c] = v[c] + bl[c];
        }
    }
    return true;
}

// Persistent forward over `rows` rows of global FP32 features [rows][IN].
__global__ void __launch_bounds__(TILE, 1) k_forward(Net net, const float* __restrict__ feats, uint32_t rows,
                                                     float* __restrict__ out, __nv_bfloat16* __restrict__ save,
                                                     int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + FwdSmem::SLOT);
    int* sflag = reinterpret_cast<int*>(smem + FwdSmem::FLAG);
    if (threadIdx.x == 0) {
        umma::mbar_init(reinterpret_cast<uint64_t*>(smem + FwdSmem::BAR), 1);
        *sflag = 0;
    }
    if (threadIdx.x < 32) umma::tmem_alloc(slot, 64);
    load_net(smem, net);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    float feat[IN], o[OUT];
    for (uint32_t tile = blockIdx.x; tile * TILE < rows; tile += gridDim.x) {
        const uint32_t r = tile * TILE + threadIdx.x;
        for (uint32_t c = 0; c < IN; ++c) feat[c] = r < rows ? feats[size_t(r) * IN + c] : 0.0f;
        bool ok = forward_tile(smem, tmem, phase, feat, o, save && r < rows ? save + size_t(r) * ACT : nullptr);
        if (!ok) {
            if (threadIdx.x == 0) atomicExch(err, 1);
            break;
        }
        if (r < rows)
            for (uint32_t c = 0; c < OUT; ++c) out[size_t(r) * OUT + c] = o[c];
    }
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::tmem_dealloc(tmem, 64);
        umma::tmem_relinquish();
    }
}

// ---- the mixture head ---------------------------------------------------------------

}  // namespace

__device__ __noinline__ MixtureGrad mixture_grad(const float* o, float3 w, float weight) {
    MixtureGrad g;
    float logit_max = -1e30f;
    for (int i = 0; i < LOBES; ++i) logit_max = fmaxf(logit_max, o[5 * i + 4]);
    float wsum = 0.0f, wl[LOBES], vl[LOBES], kap[LOBES], cosw[LOBES], rn[LOBES];
    float3 mu[LOBES];
    for (int i = 0; i < LOBES; ++i) {
        wl[i] = __expf(o[5 * i + 4] - logit_max);
        wsum += wl[i];
    }
    float q = 0.0f;
    for (int i = 0; i < LOBES; ++i) {
        wl[i] /= wsum;
        Lobe L = lobe(o + 5 * i);
        mu[i] = L.mu;
        kap[i] = L.kappa;
        rn[i] = L.norm;
        cosw[i] = L.mu.x * w.x + L.mu.y * w.y + L.mu.z * w.z;
        vl[i] = vmf_pdf(L.kappa, cosw[i]);
        q += wl[i] * vl[i];
    }
    q = fmaxf(q, 1e-20f);
    g.log_q = logf(q);
    const float dq = -weight / q;  // d(-weight log q)/dq
    for (int i = 0; i < LOBES; ++i) {
        const float* oi = o + 5 * i;
        float* gi = g.d + 5 * i;
        gi[4] = dq * wl[i] * (vl[i] - q);
        float e2 = __expf(-2.0f * kap[i]);
        float dlogc = 1.0f / kap[i] - 2.0f * e2 / (1.0f - e2);
        float dv_dk = vl[i] * (dlogc + (cosw[i] - 1.0f));
        float x = fminf(fmaxf(oi[3], -20.0f), 20.0f);
        float sig = 1.0f / (1.0f + __expf(-x));
        gi[3] = dq * wl[i] * dv_dk * sig;
        // dv/dr = v k (w - (mu.w) mu) / |r|
        float s = dq * wl[i] * vl[i] * kap[i] / rn[i];
        gi[0] = s * (w.x - cosw[i] * mu[i].x);
        gi[1] = s * (w.y - cosw[i] * mu[i].y);
        gi[2] = s * (w.z - cosw[i] * mu[i].z);
    }
    return g;
}

namespace {

// Per sample: the loss term -c log q(w) and dL/d(outputs) (mean over the
// batch), written as BF16 dZ4 rows of OUT_PAD (padding zero).
__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ dirs, const float* __restrict__ weights,
                       uint32_t rows, float inv_batch, __nv_bfloat16* __restrict__ dz4, float* loss) {
    float acc = 0.0f;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        float3 w = make_float3(dirs[3 * r], dirs[3 * r + 1], dirs[3 * r + 2]);
        float c = weights[r] * inv_batch;
        MixtureGrad g = mixture_grad(out + size_t(r) * OUT, w, c);
        acc += -c * g.log_q;
        for (uint32_t k = 0; k < OUT_PAD; ++k)
            dz4[size_t(r) * OUT_PAD + k] = __float2bfloat16_rn(k < OUT ? g.d[k] : 0.0f);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// ---- backward ----------------------------------------------------------------------

struct BwdSmem {
    static constexpr uint32_t W2T = 0;                         // 64 x 64 (W2^T)
    static constexpr uint32_t W3T = W2T + HIDDEN * HIDDEN * 2; // 64 x 64
    static constexpr uint32_t W4T = W3T + HIDDEN * HIDDEN * 2; // 64 x 48 (W4^T, K = 48)
    static constexpr uint32_t DZ = W4T + HIDDEN * OUT_PAD * 2; // 128 x 64 (or 48) dZ rows
    static constexpr uint32_t DZT = DZ + TILE * HIDDEN * 2;    // 128 x 128 dZ^T (rows >= n zero)
    static constexpr uint32_t AT = DZT + TILE * TILE * 2;      // 96 x 128 A^T
    static constexpr uint32_t BAR = AT + IN * TILE * 2;
    static constexpr uint32_t SLOT = BAR + 8;
    static constexpr uint32_t FLAG = SLOT + 4;
    static constexpr uint32_t BYTES = FLAG + 12;
};
static_assert(BwdSmem::BYTES <= 227 * 1024, "shared memory");

// TMEM columns of the backward kernel: the four weight-gradient accumulators
// (M = 128 rows, the first 64 or 40 valid) and the input-gradient scratch.
constexpr uint32_t T_DW1 = 0, T_DW2 = 96, T_DW3 = 160, T_DW4 = 224, T_DA = 288, T_COLS = 512;

// dW_l^T (as [n rows][k cols]) += dZ^T A over this tile, with dZ (rows of n)
// and A (rows of k) given per thread.
__device__ void stage_weight_grad(uint8_t* smem, const float* dz, uint32_t n, const __nv_bfloat16* act, uint32_t k) {
    const uint32_t b = threadIdx.x;
    for (uint32_t f = 0; f < n; ++f)
        *reinterpret_cast<__nv_bfloat16*>(smem + BwdSmem::DZT + kmajor_offset(f, b, TILE)) = __float2bfloat16_rn(dz[f]);
    for (uint32_t f = 0; f < k; ++f)
        *reinterpret_cast<__nv_bfloat16*>(smem + BwdSmem::AT + kmajor_offset(f, b, TILE)) = act[f];
}

__global__ void __launch_bounds__(TILE, 1) k_backward(Net net, const __nv_bfloat16* __restrict__ save,
                                                      const __nv_bfloat16* __restrict__ dz4, uint32_t rows,
                                                      float* __restrict__ grad, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + BwdSmem::BAR);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + BwdSmem::SLOT);
    int* sflag = reinterpret_cast<int*>(smem + BwdSmem::FLAG);
    if (threadIdx.x == 0) {
        umma::mbar_init(bar, 1);
        *sflag = 0;
    }
    if (threadIdx.x < 32) umma::tmem_alloc(slot, T_COLS);
    load_matrix_t(smem + BwdSmem::W2T, net.w[1], HIDDEN, HIDDEN);
    load_matrix_t(smem + BwdSmem::W3T, net.w[2], HIDDEN, HIDDEN);
    load_matrix_t(smem + BwdSmem::W4T, net.w[3], OUT_PAD, HIDDEN);
    // dZ^T rows past the layer's width stay zero for the whole kernel.
    for (uint32_t i = threadIdx.x; i < TILE * TILE / 8; i += blockDim.x)
        reinterpret_cast<uint4*>(smem + BwdSmem::DZT)[i] = make_uint4(0, 0, 0, 0);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t base = umma::smem_u32(smem);
    uint32_t phase = 0;
    bool first = true, ok = true;
    float dz[HIDDEN], da[HIDDEN];
    float bgrad[3 * HIDDEN + OUT];
    for (uint32_t i = 0; i < 3 * HIDDEN + OUT; ++i) bgrad[i] = 0.0f;
    const uint32_t dw_col[4] = {T_DW1, T_DW2, T_DW3, T_DW4};
    const uint32_t wt_off[4] = {0, BwdSmem::W2T, BwdSmem::W3T, BwdSmem::W4T};
    for (uint32_t tile = blockIdx.x; ok && tile * TILE < rows; tile += gridDim.x) {
        const uint32_t r = tile * TILE + threadIdx.x;
        const bool live = r < rows;
        const __nv_bfloat16* act = save + size_t(live ? r : 0) * ACT;
        // Layer 4: dZ4 from the loss.
        for (uint32_t c = 0; c < OUT_PAD; ++c) dz[c] = live ? __bfloat162float(dz4[size_t(r) * OUT_PAD + c]) : 0.0f;
        for (int l = 3; l >= 0 && ok; --l) {
            const uint32_t n = l == 3 ? OUT_PAD : HIDDEN;           // this layer's outputs
            const uint32_t k = l == 0 ? IN : HIDDEN;                 // its inputs
            const __nv_bfloat16* a_in = act + (l == 0 ? 0 : IN + (l - 1) * HIDDEN);
            for (uint32_t c = 0; c < n; ++c) bgrad[l * HIDDEN + c] += (l == 3 && c >= OUT) ? 0.0f : dz[c];
            // Stage dZ^T / A^T for dW, and dZ rows for dA.
            __syncthreads();  // previous MMAs of this CTA have read the buffers (waited below)
            stage_weight_grad(smem, dz, n, live ? a_in : act, k);
            if (!live) {
                for (uint32_t f = 0; f < k; ++f)
                    *reinterpret_cast<__nv_bfloat16*>(smem + BwdSmem::AT + kmajor_offset(f, threadIdx.x, TILE)) =
                        __float2bfloat16_rn(0.0f);
            }
            if (l > 0) store_row(smem + BwdSmem::DZ, threadIdx.x, n, dz);
            umma::fence_async_smem();
            umma::fence_before_sync();
            __syncthreads();
            if (threadIdx.x == 0) {
                umma::fence_after_sync();
                // dW_l += dZ^T (rows: n, padded to 128) x A (k columns), K = the tile's 128 rows.
                const uint32_t idw = umma::idesc_bf16_f32(128, k);
                for (uint32_t k0 = 0; k0 < TILE; k0 += 16)
                    umma::mma_bf16(tmem + dw_col[l], umma::kslice_desc(base + BwdSmem::DZT, k0, TILE),
                                   umma::kslice_desc(base + BwdSmem::AT, k0, TILE), idw, !first || k0 > 0);
                // dA = dZ (128 x n) x W_l (n x k): B = W_l^T as [k rows][n].
                if (l > 0) {
                    const uint32_t ida = umma::idesc_bf16_f32(128, k);
                    for (uint32_t k0 = 0; k0 < n; k0 += 16)
                        umma::mma_bf16(tmem + T_DA, umma::kslice_desc(base + BwdSmem::DZ, k0, n),
                                       umma::kslice_desc(base + wt_off[l], k0, n), ida, k0 > 0);
                }
                umma::commit(bar);
            }
            if (!wait_all(bar, phase, sflag)) {
                ok = false;
                break;
            }
            phase ^= 1u;
            if (l > 0) {
                read_row(tmem, T_DA, k, da);
                // ReLU: the activation fed forward was positive exactly where Z was.
                for (uint32_t c = 0; c < k; ++c) dz[c] = __bfloat162float(a_in[c]) > 0.0f ? da[c] : 0.0f;
                if (!live)
                    for (uint32_t c = 0; c < k; ++c) dz[c] = 0.0f;
            }
        }
        first = false;
    }
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    // The accumulated weight gradients (lane = output row) into global FP32.
    if (ok && !first) {
        umma::fence_after_sync();
        const uint32_t woff[4] = {P_W1, P_W2, P_W3, P_W4};
        const uint32_t nrow[4] = {HIDDEN, HIDDEN, HIDDEN, OUT};
        const uint32_t ncol[4] = {IN, HIDDEN, HIDDEN, HIDDEN};
        for (int l = 0; l < 4; ++l) {
            float v[IN];
            read_row(tmem, dw_col[l], ncol[l], v);
            if (threadIdx.x < nrow[l])
                for (uint32_t c = 0; c < ncol[l]; ++c) atomicAdd(grad + woff[l] + threadIdx.x * ncol[l] + c, v[c]);
        }
    }
    // Bias gradients: a warp reduction per entry, then one atomic per warp.
    const uint32_t boff[4] = {P_B1, P_B2, P_B3, P_B4};
    for (uint32_t i = 0; i < 3 * HIDDEN + OUT; ++i) {
        float s = bgrad[i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && s != 0.0f) atomicAdd(grad + boff[i / HIDDEN] + i % HIDDEN, s);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::tmem_dealloc(tmem, T_COLS);
        umma::tmem_relinquish();
    }
}

// ---- Adam ----------------------------------------------------------------------------

__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       uint32_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        g[i] = 0.0f;
    }
}

// BF16 copies of the weights (W4 padded to OUT_PAD rows) and the padded bias.
__global__ void k_cast(const float* __restrict__ p, __nv_bfloat16* __restrict__ w1, __nv_bfloat16* __restrict__ w2,
                       __nv_bfloat16* __restrict__ w3, __nv_bfloat16* __restrict__ w4, float* __restrict__ b4) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < HIDDEN * IN) w1[i] = __float2bfloat16_rn(p[P_W1 + i]);
    if (i < HIDDEN * HIDDEN) {
        w2[i] = __float2bfloat16_rn(p[P_W2 + i]);
        w3[i] = __float2bfloat16_rn(p[P_W3 + i]);
    }
    if (i < OUT_PAD * HIDDEN) w4[i] = __float2bfloat16_rn(i < OUT * HIDDEN ? p[P_W4 + i] : 0.0f);
    if (i < OUT_PAD) b4[i] = i < OUT ? p[P_B4 + i] : 0.0f;
}

// ---- in the wavefront ------------------------------------------------------------------------

__device__ __forceinline__ float3 ld3(const float* p, uint32_t v) {
    return make_float3(__ldg(p + 3 * v), __ldg(p + 3 * v + 1), __ldg(p + 3 * v + 2));
}

// A hit's world position and geometric normal turned against the ray: the
// guide's inputs (the shading kernel records the same quantities).
__device__ void hit_frame(const DeviceScene& s, uint4 h, float3 dir, float3& pos, float3& nrm) {
    const GeomRecord& g = s.geometry[h.x];
    const uint32_t prim = h.y;
    const float b1 = __uint_as_float(h.z), b2 = __uint_as_float(h.w);
    uint32_t i0 = __ldg(g.indices + 3 * prim), i1 = __ldg(g.indices + 3 * prim + 1), i2 = __ldg(g.indices + 3 * prim + 2);
    float3 v0 = ld3(g.positions, i0), v1 = ld3(g.positions, i1), v2 = ld3(g.positions, i2);
    float3 e1 = make_float3(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z), e2 = make_float3(v2.x - v0.x, v2.y - v0.y, v2.z - v0.z);
    float3 op = make_float3(v0.x + b1 * e1.x + b2 * e2.x, v0.y + b1 * e1.y + b2 * e2.y, v0.z + b1 * e1.z + b2 * e2.z);
    float3 on = make_float3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x);
    pos = make_float3(g.o2w[0][0] * op.x + g.o2w[0][1] * op.y + g.o2w[0][2] * op.z + g.o2w[0][3],
                      g.o2w[1][0] * op.x + g.o2w[1][1] * op.y + g.o2w[1][2] * op.z + g.o2w[1][3],
                      g.o2w[2][0] * op.x + g.o2w[2][1] * op.y + g.o2w[2][2] * op.z + g.o2w[2][3]);
    float3 wn = make_float3(g.w2o[0][0] * on.x + g.w2o[1][0] * on.y + g.w2o[2][0] * on.z,
                            g.w2o[0][1] * on.x + g.w2o[1][1] * on.y + g.w2o[2][1] * on.z,
                            g.w2o[0][2] * on.x + g.w2o[1][2] * on.y + g.w2o[2][2] * on.z);
    float inv = rsqrtf(wn.x * wn.x + wn.y * wn.y + wn.z * wn.z);
    wn = make_float3(wn.x * inv, wn.y * inv, wn.z * inv);
    if (wn.x * dir.x + wn.y * dir.y + wn.z * dir.z > 0.0f) wn = make_float3(-wn.x, -wn.y, -wn.z);
    nrm = wn;
}

__device__ __forceinline__ float3 unit_pos(const DeviceScene& s, float3 p) {
    return make_float3((p.x - s.bbox_min[0]) * s.bbox_inv, (p.y - s.bbox_min[1]) * s.bbox_inv,
                       (p.z - s.bbox_min[2]) * s.bbox_inv);
}

// ---- inference in the wavefront: warp groups sharing one copy of the network ----------
//
// A CTA of WG warp groups (128 threads each): every group runs its own 128-row
// tiles through the network with its own operand buffers, TMEM columns and
// mbarrier, while the weights are staged once per CTA. With 16 warps per SM
// the scattered loads of one group's next tile (hit records, vertices,
// transforms) overlap the other groups' tensor-core layers. Features go
// straight to the BF16 operand in 8-column chunks and outputs straight from
// TMEM to global memory, so a thread holds neither its 96 inputs nor its 40
// outputs in registers. The arithmetic (encoding, BF16 rounding, MMA order,
// bias and ReLU) is that of forward_tile: the outputs are bitwise the same.
constexpr uint32_t WG = 4;

struct InferSmem {  // offsets in bytes
    static constexpr uint32_t W1 = FwdSmem::W1, W2 = FwdSmem::W2, W3 = FwdSmem::W3, W4 = FwdSmem::W4;
    static constexpr uint32_t BIAS = W4 + OUT_PAD * HIDDEN * 2;               // 64 * 3 + 48 floats
    static constexpr uint32_t GROUPS = (BIAS + (3 * HIDDEN + OUT_PAD) * 4 + 1023u) & ~1023u;
    static constexpr uint32_t A0 = 0, H = TILE * IN * 2, GROUP = H + TILE * HIDDEN * 2;  // within a group
    static constexpr uint32_t BAR = GROUPS + WG * GROUP;
    static constexpr uint32_t SLOT = BAR + 8 * WG;
    static constexpr uint32_t FLAG = SLOT + 4;
    static constexpr uint32_t BYTES = FLAG + 4 * WG;
};
static_assert(InferSmem::GROUPS % 1024 == 0 && InferSmem::BAR % 8 == 0, "alignment");
static_assert(InferSmem::BYTES <= 227 * 1024, "shared memory");

__device__ void load_net_at(uint8_t* smem, const Net& net, uint32_t bias_off) {
    load_matrix(smem + FwdSmem::W1, net.w[0], HIDDEN, HIDDEN, IN);
    load_matrix(smem + FwdSmem::W2, net.w[1], HIDDEN, HIDDEN, HIDDEN);
    load_matrix(smem + FwdSmem::W3, net.w[2], HIDDEN, HIDDEN, HIDDEN);
    load_matrix(smem + FwdSmem::W4, net.w[3], OUT_PAD, OUT_PAD, HIDDEN);
    float* bias = reinterpret_cast<float*>(smem + bias_off);
    for (uint32_t i = threadIdx.x; i < 3 * HIDDEN + OUT_PAD; i += blockDim.x)
        bias[i] = i < 3 * HIDDEN ? net.b[i / HIDDEN][i % HIDDEN] : net.b[3][i - 3 * HIDDEN];
}

// Features 8c .. 8c + 7 of encode(p, n, wo), computed as encode computes them.
__device__ __forceinline__ void encode_chunk(uint32_t c, float3 p, float3 n, float3 wo, float* f) {
    if (c < 9) {
        const float co[3] = {p.x, p.y, p.z};
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t q = 4 * c + k, b = q / 3, a = q % 3;
            const float s = 3.14159265f * float(1u << b);
            __sincosf(s * co[a], &f[2 * k], &f[2 * k + 1]);
        }
    } else if (c == 9) {
        f[0] = n.x; f[1] = n.y; f[2] = n.z;
        f[3] = wo.x; f[4] = wo.y; f[5] = wo.z;
        f[6] = p.x; f[7] = p.y;
    } else {
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) f[k] = 0.0f;
        if (c == 10) f[0] = p.z;
    }
}

__device__ __forceinline__ void group_sync(uint32_t g) {
    asm volatile("bar.sync %0, %1;" ::"r"(1u + g), "r"(TILE) : "memory");
}

__global__ void __launch_bounds__(TILE * WG, 1) k_infer_paths(Net net, DeviceScene scene, PathPool pool,
                                                              uint32_t bounce, uint32_t n0, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + InferSmem::SLOT);
    const uint32_t g = threadIdx.x / TILE, row = threadIdx.x % TILE;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + InferSmem::BAR) + g;
    int* gflag = reinterpret_cast<int*>(smem + InferSmem::FLAG) + g;
    uint8_t* gbase = smem + InferSmem::GROUPS + g * InferSmem::GROUP;
    const float* bias = reinterpret_cast<const float*>(smem + InferSmem::BIAS);
    const uint32_t count = min(bounce == 0 ? n0 : pool.counters[CTR_RAYS + bounce], pool.capacity);
    const uint32_t* queue = pool.queue[bounce & 1u];
    if (threadIdx.x < WG) {
        umma::mbar_init(reinterpret_cast<uint64_t*>(smem + InferSmem::BAR) + threadIdx.x, 1);
        reinterpret_cast<int*>(smem + InferSmem::FLAG)[threadIdx.x] = 0;
    }
    if (threadIdx.x < 32) umma::tmem_alloc(slot, 64 * WG);
    load_net_at(smem, net, InferSmem::BIAS);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *slot + 64u * g;  // this group's 64 columns
    const uint32_t base = umma::smem_u32(smem);
    const uint32_t a_off[4] = {InferSmem::GROUPS + g * InferSmem::GROUP + InferSmem::A0,
                               InferSmem::GROUPS + g * InferSmem::GROUP + InferSmem::H,
                               InferSmem::GROUPS + g * InferSmem::GROUP + InferSmem::H,
                               InferSmem::GROUPS + g * InferSmem::GROUP + InferSmem::H};
    const uint32_t w_off[4] = {FwdSmem::W1, FwdSmem::W2, FwdSmem::W3, FwdSmem::W4};
    const uint32_t lane_base = ((threadIdx.x / 32u) % 4u) * 32u;
    uint32_t phase = 0;
    for (uint32_t tile = blockIdx.x * WG + g; tile * TILE < count; tile += gridDim.x * WG) {
        const uint32_t i = tile * TILE + row;
        uint32_t path = 0;
        bool hit = false;
        float3 p = make_float3(0.0f, 0.0f, 0.0f), nrm = p, wo = p;
        if (i < count) {
            path = bounce == 0 ? i : queue[i];
            const uint4 h = pool.hit[path];
            hit = h.x != LIGHT_NONE;
            if (hit) {
                const float4 d4 = pool.dir[path];
                const float3 dir = make_float3(d4.x, d4.y, d4.z);
                float3 wp;
                hit_frame(scene, h, dir, wp, nrm);
                p = unit_pos(scene, wp);
                wo = make_float3(-dir.x, -dir.y, -dir.z);
            }
        }
        for (uint32_t c = 0; c < IN / 8; ++c) {
            float f[8];
            if (hit) encode_chunk(c, p, nrm, wo, f);
            else
                for (uint32_t k = 0; k < 8; ++k) f[k] = 0.0f;
            *reinterpret_cast<uint4*>(gbase + InferSmem::A0 + kmajor_offset(row, 8 * c, IN)) = pack8(f);
        }
        bool ok = true;
        for (int l = 0; l < 4 && ok; ++l) {
            const uint32_t k = l == 0 ? IN : HIDDEN, n = l == 3 ? OUT_PAD : HIDDEN;
            umma::fence_async_smem();
            umma::fence_before_sync();
            group_sync(g);
            if (row == 0) {
                umma::fence_after_sync();
                issue_layer(tmem, base + a_off[l], base + w_off[l], k, n, bar, false);
            }
            if (!umma::mbar_wait(bar, phase, WAIT_LIMIT)) atomicOr(gflag, 1);
            group_sync(g);
            umma::fence_after_sync();
            ok = *gflag == 0;
            phase ^= 1u;
            if (!ok) break;
            const float* bl = bias + l * HIDDEN;
            if (l < 3) {
                for (uint32_t c0 = 0; c0 < HIDDEN; c0 += 16) {
                    float v[16];
                    umma::tmem_ld16(umma::tmem_at(tmem, lane_base, c0), v);
                    umma::tmem_wait_ld();
                    for (uint32_t c = 0; c < 16; ++c) v[c] = fmaxf(v[c] + bl[c0 + c], 0.0f);
                    *reinterpret_cast<uint4*>(gbase + InferSmem::H + kmajor_offset(row, c0, HIDDEN)) = pack8(v);
                    *reinterpret_cast<uint4*>(gbase + InferSmem::H + kmajor_offset(row, c0 + 8, HIDDEN)) = pack8(v + 8);
                }
            } else {
                // The raw outputs, then the mixture activated once for shading.
                float o[OUT_PAD];
                for (uint32_t c0 = 0; c0 < OUT_PAD; c0 += 16) {
                    umma::tmem_ld16(umma::tmem_at(tmem, lane_base, c0), o + c0);
                    umma::tmem_wait_ld();
                    for (uint32_t c = 0; c < 16; ++c) o[c0 + c] += bl[c0 + c];
                }
                if (hit) {
                    float a[OUT_ACT];
                    activate(o, a);
                    float4* dst = reinterpret_cast<float4*>(pool.guide_out + size_t(path) * OUT_ACT);
                    for (uint32_t c = 0; c < OUT_ACT; c += 4) dst[c / 4] = make_float4(a[c], a[c + 1], a[c + 2], a[c + 3]);
                }
            }
        }
        if (!ok) {
            if (row == 0) atomicExch(err, 1);
            break;
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::tmem_dealloc(*slot, 64 * WG);
        umma::tmem_relinquish();
    }
}

__device__ __forceinline__ float lum(float3 c) { return 0.2722287f * c.x + 0.6740818f * c.y + 0.0536895f * c.z; }

__global__ void k_resolve_records(Record* recs, const uint32_t* count, uint32_t capacity, const float4* rad) {
    const uint32_t n = min(*count, capacity);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Record r = recs[i];
        float c = 0.0f;
        if (r.q2.w >= 0.0f && r.q0.w > 0.0f) {
            float4 f = rad[__float_as_uint(r.q3.w)];
            float L = (lum(make_float3(f.x, f.y, f.z)) - r.q2.w) / fmaxf(r.q1.w, 1e-12f);
            c = fmaxf(L, 0.0f) / r.q0.w;
            if (!isfinite(c)) c = 0.0f;
        }
        recs[i].q0.w = c;
    }
}

// Row r of the batch starting at `offset`: a prime stride (above any record
// count, hence coprime to it) walks the wave's records as a permutation, so
// every batch spans the whole wave. Records arrive in shading order, which the
// material sort groups by material: contiguous batches would each see one or
// two materials.
__device__ __forceinline__ uint32_t batch_record(uint32_t offset, uint32_t r, uint32_t n) {
    return uint32_t((uint64_t(offset) + uint64_t(r) * 2654435761ull) % n);
}

// Training forward over records: inputs encoded from each record.
__global__ void __launch_bounds__(TILE, 1) k_forward_records(Net net, const Record* __restrict__ recs,
                                                             const uint32_t* count, uint32_t capacity, uint32_t offset,
                                                             uint32_t rows, float3 bmin, float binv,
                                                             float* __restrict__ out, __nv_bfloat16* __restrict__ save,
                                                             float* sums, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + FwdSmem::SLOT);
    int* sflag = reinterpret_cast<int*>(smem + FwdSmem::FLAG);
    const uint32_t n = min(*count, capacity);
    if (threadIdx.x == 0) {
        umma::mbar_init(reinterpret_cast<uint64_t*>(smem + FwdSmem::BAR), 1);
        *sflag = 0;
    }
    if (threadIdx.x < 32) umma::tmem_alloc(slot, 64);
    load_net(smem, net);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    float feat[IN], o[OUT];
    float wsum = 0.0f;
    for (uint32_t tile = blockIdx.x; n > 0 && tile * TILE < rows; tile += gridDim.x) {
        const uint32_t r = tile * TILE + threadIdx.x;
        if (r < rows) {
            const Record rc = recs[batch_record(offset, r, n)];
            float3 p = make_float3((rc.q0.x - bmin.x) * binv, (rc.q0.y - bmin.y) * binv, (rc.q0.z - bmin.z) * binv);
            encode(p, make_float3(rc.q1.x, rc.q1.y, rc.q1.z), make_float3(rc.q2.x, rc.q2.y, rc.q2.z), feat);
            wsum += rc.q0.w;
        } else {
            for (uint32_t c = 0; c < IN; ++c) feat[c] = 0.0f;
        }
        if (!forward_tile(smem, tmem, phase, feat, o, r < rows ? save + size_t(r) * ACT : nullptr)) {
            if (threadIdx.x == 0) atomicExch(err, 1);
            break;
        }
        if (r < rows)
            for (uint32_t c = 0; c < OUT; ++c) out[size_t(r) * OUT + c] = o[c];
    }
    for (int k = 16; k > 0; k >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, k);
    if ((threadIdx.x & 31) == 0) atomicAdd(sums, wsum);
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::tmem_dealloc(tmem, 64);
        umma::tmem_relinquish();
    }
}

// Loss over records: weights normalised by the batch mean and clamped at 20
// (one bright sample must not dominate a step), then averaged.
__global__ void k_loss_records(const float* __restrict__ out, const Record* __restrict__ recs, const uint32_t* count,
                               uint32_t capacity, uint32_t offset, uint32_t rows, const float* sums,
                               __nv_bfloat16* __restrict__ dz4, float* loss) {
    const uint32_t n = min(*count, capacity);
    const float mean = sums[0] / float(rows);
    float acc = 0.0f;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        float c = 0.0f;
        float3 w = make_float3(0.0f, 0.0f, 1.0f);
        if (n > 0 && mean > 0.0f) {
            const Record rc = recs[batch_record(offset, r, n)];
            c = fminf(rc.q0.w / mean, 20.0f) / float(rows);
            w = make_float3(rc.q3.x, rc.q3.y, rc.q3.z);
        }
        MixtureGrad g = mixture_grad(out + size_t(r) * OUT, w, c);
        acc += -c * g.log_q;
        for (uint32_t k = 0; k < OUT_PAD; ++k)
            dz4[size_t(r) * OUT_PAD + k] = __float2bfloat16_rn(k < OUT ? g.d[k] : 0.0f);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

}  // namespace

// ---- host launchers ----------------------------------------------------------------------

static Net view(const Buffers& b) {
    Net n;
    n.w[0] = b.w1;
    n.w[1] = b.w2;
    n.w[2] = b.w3;
    n.w[3] = b.w4;
    n.b[0] = b.params + P_B1;
    n.b[1] = b.params + P_B2;
    n.b[2] = b.params + P_B3;
    n.b[3] = b.b4;
    return n;
}

cudaError_t configure(int device, int* sms) {
    cudaError_t e = cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, FwdSmem::BYTES);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_infer_paths, cudaFuncAttributeMaxDynamicSharedMemorySize, InferSmem::BYTES);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_forward_records, cudaFuncAttributeMaxDynamicSharedMemorySize, FwdSmem::BYTES);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, BwdSmem::BYTES);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, device);
    return e;
}

void launch_cast(const Buffers& b, cudaStream_t s) {
    k_cast<<<(HIDDEN * IN + 255) / 256, 256, 0, s>>>(b.params, b.w1, b.w2, b.w3, b.w4, b.b4);
}

void launch_forward(const Buffers& b, const float* feats, uint32_t rows, float* out, __nv_bfloat16* save, int sms,
                    cudaStream_t s) {
    uint32_t tiles = (rows + TILE - 1) / TILE;
    int grid = int(tiles < uint32_t(sms) ? tiles : uint32_t(sms));
    if (grid < 1) return;
    k_forward<<<grid, TILE, FwdSmem::BYTES, s>>>(view(b), feats, rows, out, save, b.err);
}

void launch_loss(const Buffers& b, const float* out, const float* dirs, const float* weights, uint32_t rows,
                 float inv_batch, __nv_bfloat16* dz4, float* loss, cudaStream_t s) {
    int grid = int((rows + 255) / 256);
    if (grid > 148 * 8) grid = 148 * 8;
    if (grid < 1) return;
    k_loss<<<grid, 256, 0, s>>>(out, dirs, weights, rows, inv_batch, dz4, loss);
}

void launch_backward(const Buffers& b, const __nv_bfloat16* save, const __nv_bfloat16* dz4, uint32_t rows, int sms,
                     cudaStream_t s) {
    uint32_t tiles = (rows + TILE - 1) / TILE;
    int grid = int(tiles < uint32_t(sms) ? tiles : uint32_t(sms));
    if (grid < 1) return;
    k_backward<<<grid, TILE, BwdSmem::BYTES, s>>>(view(b), save, dz4, rows, b.grad, b.err);
}

void launch_adam(const Buffers& b, float lr, uint32_t step, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f / (1.0f - powf(b1, float(step)));
    const float c2 = 1.0f / (1.0f - powf(b2, float(step)));
    k_adam<<<(PARAMS + 255) / 256, 256, 0, s>>>(b.params, b.grad, b.m, b.v, PARAMS, lr, b1, b2, eps, c1, c2);
}

void launch_infer_paths(const Buffers& b, const DeviceScene& scene, const PathPool& pool, uint32_t bounce,
                        uint32_t n0, int sms, cudaStream_t s) {
    // One CTA of WG warp groups per SM: the groups hide each other's gathers and waits.
    k_infer_paths<<<sms, TILE * WG, InferSmem::BYTES, s>>>(view(b), scene, pool, bounce, n0, b.err);
}

void launch_resolve_records(Record* recs, const uint32_t* count, uint32_t capacity, const float4* rad, cudaStream_t s) {
    k_resolve_records<<<148 * 4, 256, 0, s>>>(recs, count, capacity, rad);
}

void launch_train_records(const Buffers& b, const TrainScratch& t, const Record* recs, const uint32_t* count,
                          uint32_t capacity, uint32_t offset, float3 bbox_min, float bbox_inv, float lr,
                          uint32_t step, int sms, cudaStream_t s) {
    cudaMemsetAsync(t.sums, 0, 8, s);
    uint32_t tiles = (t.rows + TILE - 1) / TILE;
    int grid = int(tiles < uint32_t(sms) ? tiles : uint32_t(sms));
    k_forward_records<<<grid, TILE, FwdSmem::BYTES, s>>>(view(b), recs, count, capacity, offset, t.rows, bbox_min,
                                                         bbox_inv, t.out, t.save, t.sums, b.err);
    int lgrid = int((t.rows + 255) / 256);
    if (lgrid > 148 * 8) lgrid = 148 * 8;
    k_loss_records<<<lgrid, 256, 0, s>>>(t.out, recs, count, capacity, offset, t.rows, t.sums, t.dz4, t.sums + 1);
    launch_backward(b, t.save, t.dz4, t.rows, sms, s);
    launch_adam(b, lr, step, s);
    launch_cast(b, s);
}

}  // namespace guide
}  // namespace cn
