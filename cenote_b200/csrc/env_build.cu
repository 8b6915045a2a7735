// The environment's importance-sampling tables, built on the device in FP64.
//
// Same tables and the same arithmetic as the host build of
// crates/cenote/src/environment.rs:130-218: f32 luminance, 3×3-max dilation
// (wrap in u, clamp in v) times the row's sin θ, f64 marginal and conditional
// CDFs cast to f32, the separate f32 pdf table and the f64 power integral.
// Every sum runs in the reference's sequential order — one thread per row for
// the row sums, one thread for the flat total — because a tree-ordered f64
// sum rounds differently and the CDF indices must match bit for bit. The
// per-row sin θ and solid angles are evaluated on the host with the same libm
// call the reference makes, so they are bit-identical inputs here.
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>

#include "records.h"

namespace cn {
namespace {

__device__ __forceinline__ float luminance_rn(float r, float g, float b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(r, 0.2722287f), __fmul_rn(g, 0.6740818f)), __fmul_rn(b, 0.0536895f));
}

__global__ void k_env_lum(const float4* __restrict__ tex, double* __restrict__ lum, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 t = tex[i];
        lum[i] = double(luminance_rn(t.x, t.y, t.z));
    }
}

__global__ void k_env_weight(const double* __restrict__ lum, const double* __restrict__ sin_theta,
                             double* __restrict__ weight, uint32_t w, uint32_t h) {
    uint32_t n = w * h;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t row = i / w, col = i - row * w;
        double peak = 0.0;
        for (int dr = -1; dr <= 1; ++dr) {
            int rr = int(row) + dr;
            uint32_t r = rr < 0 ? 0u : min(uint32_t(rr), h - 1);
            for (int dc = -1; dc <= 1; ++dc) {
                int cc = int(col) + dc;
                uint32_t c = cc < 0 ? uint32_t(cc + int(w)) : (uint32_t(cc) >= w ? uint32_t(cc) - w : uint32_t(cc));
                peak = fmax(peak, lum[size_t(r) * w + c]);
            }
        }
        weight[i] = __dmul_rn(peak, sin_theta[row]);
    }
}

// One thread per row: the row sum, the row's conditional CDF and the
// undilated luminance sum for the power integral, all sequential in f64.
__global__ void k_env_rows(const double* __restrict__ weight, const double* __restrict__ lum,
                           double* __restrict__ row_sum, double* __restrict__ lum_sum, float* __restrict__ conditional,
                           uint32_t w, uint32_t h) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= h) return;
    const double* wr = weight + size_t(row) * w;
    double rs = 0.0;
    for (uint32_t c = 0; c < w; ++c) rs = __dadd_rn(rs, wr[c]);
    row_sum[row] = rs;
    float* cdf = conditional + size_t(row) * (w + 1);
    cdf[0] = 0.0f;
    double run = 0.0;
    for (uint32_t c = 0; c < w; ++c) {
        run = __dadd_rn(run, wr[c]);
        cdf[c + 1] = rs > 0.0 ? __double2float_rn(__ddiv_rn(run, rs)) : 0.0f;
    }
    cdf[w] = 1.0f;
    const double* lr = lum + size_t(row) * w;
    double ls = 0.0;
    for (uint32_t c = 0; c < w; ++c) ls = __dadd_rn(ls, lr[c]);
    lum_sum[row] = ls;
}

// The flat total over every weight in row-major order, the marginal CDF and
// the power integral: sequential by definition. Two warps: the second stages
// the next 1,024 weights into shared memory with coalesced loads while lane 0
// of the first adds the current 1,024 in order (eight loads ahead of the
// dependent adds), so the sum rounds exactly like the host's left fold and
// only the chain of FP64 adds is serial.
__global__ void __launch_bounds__(64) k_env_marginal(const double* __restrict__ weight, const double* __restrict__ row_sum,
                                                     const double* __restrict__ lum_sum, const double* __restrict__ solid,
                                                     float* __restrict__ marginal, double* __restrict__ out, uint32_t w,
                                                     uint32_t h) {
    __shared__ double buf[2][1024];
    const uint32_t warp = threadIdx.x / 32u, lane = threadIdx.x % 32u;
    const size_t n = size_t(w) * h;
    const size_t chunks = (n + 1023) / 1024;
    auto stage = [&](size_t c) {
        const size_t base = c * 1024;
        const size_t m = n - base < 1024 ? n - base : 1024;
        double* dst = buf[c & 1];
#pragma unroll 8
        for (uint32_t k = 0; k < 32; ++k) {
            const size_t j = size_t(k) * 32 + lane;
            if (j < m) dst[j] = weight[base + j];
        }
    };
    double total = 0.0;
    if (warp == 1 && chunks > 0) stage(0);
    __syncthreads();
    for (size_t c = 0; c < chunks; ++c) {
        if (warp == 1) {
            if (c + 1 < chunks) stage(c + 1);
        } else if (lane == 0) {
            const size_t m = n - c * 1024 < 1024 ? n - c * 1024 : 1024;
            const double* src = buf[c & 1];
            size_t j = 0;
            for (; j + 8 <= m; j += 8) {
                double v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = src[j + k];
#pragma unroll
                for (int k = 0; k < 8; ++k) total = __dadd_rn(total, v[k]);
            }
            for (; j < m; ++j) total = __dadd_rn(total, src[j]);
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    marginal[0] = 0.0f;
    double run = 0.0;
    for (uint32_t r = 0; r < h; ++r) {
        run = __dadd_rn(run, row_sum[r]);
        marginal[r + 1] = total > 0.0 ? __double2float_rn(__ddiv_rn(run, total)) : 0.0f;
    }
    marginal[h] = 1.0f;
    double power = 0.0;
    for (uint32_t r = 0; r < h; ++r) power = __dadd_rn(power, __dmul_rn(solid[r], lum_sum[r]));
    out[0] = total;
    out[1] = power;
}

__global__ void k_env_pdfs(const double* __restrict__ weight, const double* __restrict__ totals, float* __restrict__ pdfs,
                           uint32_t w, uint32_t h) {
    const double total = totals[0];
    const double scale = total > 0.0 ? __ddiv_rn(double(size_t(w) * h), total) : 0.0;
    size_t n = size_t(w) * h;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        pdfs[i] = __double2float_rn(__dmul_rn(weight[i], scale));
}

// Cutpoint tables: for CDF r (0: the marginal over h rows; 1 + k: row k's
// conditional over w columns) and bucket b, the last index i below the CDF's
// count with cdf[i] <= b / ENV_CUTS, by the same search sample_cdf runs.
__global__ void k_env_cuts(const float* __restrict__ marginal, const float* __restrict__ conditional, uint32_t* cut,
                           uint32_t w, uint32_t h) {
    const size_t n = size_t(h + 1) * (ENV_CUTS + 1);
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const uint32_t r = uint32_t(k / (ENV_CUTS + 1)), b = uint32_t(k % (ENV_CUTS + 1));
        const float* cdf = r == 0 ? marginal : conditional + size_t(r - 1) * (w + 1);
        const uint32_t count = r == 0 ? h : w;
        const float u = float(b) / float(ENV_CUTS);
        uint32_t lo = 0, hi = count;
        while (lo + 1 < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (cdf[mid] <= u) lo = mid;
            else hi = mid;
        }
        cut[k] = lo;
    }
}

}  // namespace

void launch_env_cuts(const float* marginal, const float* conditional, uint32_t w, uint32_t h, uint32_t* cut,
                     cudaStream_t stream) {
    const size_t n = size_t(h + 1) * (ENV_CUTS + 1);
    int grid = int((n + 255) / 256);
    if (grid > 148 * 32) grid = 148 * 32;
    k_env_cuts<<<grid, 256, 0, stream>>>(marginal, conditional, cut, w, h);
}

// scratch: 3·w·h + 3·h doubles + 2 doubles; results into marginal (h+1),
// conditional (h·(w+1)), pdfs (w·h) and totals (total, power).
void launch_env_tables(const float4* texels, const double* sin_theta, const double* solid, uint32_t w, uint32_t h,
                       double* scratch, float* marginal, float* conditional, float* pdfs, double* totals,
                       cudaStream_t stream) {
    const size_t n = size_t(w) * h;
    double* lum = scratch;
    double* weight = lum + n;
    double* row_sum = weight + n;
    double* lum_sum = row_sum + h;
    int grid = int((n + 255) / 256);
    if (grid > 148 * 32) grid = 148 * 32;
    k_env_lum<<<grid, 256, 0, stream>>>(texels, lum, uint32_t(n));
    k_env_weight<<<grid, 256, 0, stream>>>(lum, sin_theta, weight, w, h);
    k_env_rows<<<(h + 63) / 64, 64, 0, stream>>>(weight, lum, row_sum, lum_sum, conditional, w, h);
    k_env_marginal<<<1, 64, 0, stream>>>(weight, row_sum, lum_sum, solid, marginal, totals, w, h);
    k_env_pdfs<<<grid, 256, 0, stream>>>(weight, totals, pdfs, w, h);
}

// ---- scratch for the allocation-free entry point --------------------------------
//
// cenote_env_tables_static builds the same tables with its FP64 scratch in
// this file-scope device array instead of cudaMalloc'd memory. Every device
// that loads the library holds it until the process exits; every call on a
// device shares it, so calls whose work overlaps on the GPU race (the
// context's lock serialises calls made through one context). Layout, in
// doubles: luminance (n) | weights (n) | row sums (h) | luminance row sums (h)
// | total and power (2) | sin θ per row (h) | solid angle per row (h). Every
// element a call reads was written earlier in the same call, so nothing needs
// clearing between calls.
constexpr size_t STATIC_ENV_MAX_TEXELS = size_t(1) << 18;  // 262,144 texels: 512x512, 1024x256, ...
constexpr uint32_t STATIC_ENV_MAX_ROWS = 1024;
constexpr size_t STATIC_ENV_SCRATCH_DOUBLES = 2 * STATIC_ENV_MAX_TEXELS + 4 * size_t(STATIC_ENV_MAX_ROWS) + 2;

static __device__ __align__(256) double g_env_scratch[STATIC_ENV_SCRATCH_DOUBLES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_env_scratch_mu;
double* g_env_scratch_ptr[kMaxDevices] = {};
cudaEvent_t g_env_scratch_done[kMaxDevices] = {};  // recorded after each call's last write
bool g_env_scratch_pending[kMaxDevices] = {};      // a call gave up waiting on that event
}  // namespace

// The device address of g_env_scratch on the current device. The host-side
// name is a stand-in, not a device address; the real one comes from
// cudaGetSymbolAddress, looked up once per device (with that device current)
// and cached. The first lookup may load this library's kernels onto the
// device, which is why a caller's first call should come before any stream
// capture.
// The same set-up creates the device's completion event (an event, not
// memory): each call records it after its last write, and a call that gave
// up waiting marks the scratch pending, so the next call on the device
// first waits for that work instead of overwriting the scratch under it.
cudaError_t static_env_scratch(int device, double** out, size_t* max_texels, uint32_t* max_rows,
                               cudaEvent_t* done) {
    *max_texels = STATIC_ENV_MAX_TEXELS;
    *max_rows = STATIC_ENV_MAX_ROWS;
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_env_scratch_mu);
    if (!g_env_scratch_ptr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_env_scratch);
        if (e != cudaSuccess) return e;
        e = cudaEventCreateWithFlags(&g_env_scratch_done[device], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
        g_env_scratch_ptr[device] = static_cast<double*>(ptr);
    }
    *out = g_env_scratch_ptr[device];
    *done = g_env_scratch_done[device];
    return cudaSuccess;
}

bool static_env_pending(int device) {
    std::lock_guard<std::mutex> lock(g_env_scratch_mu);
    return device >= 0 && device < kMaxDevices && g_env_scratch_pending[device];
}

void static_env_set_pending(int device, bool pending) {
    std::lock_guard<std::mutex> lock(g_env_scratch_mu);
    if (device >= 0 && device < kMaxDevices) g_env_scratch_pending[device] = pending;
}

}  // namespace cn
