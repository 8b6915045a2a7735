// The guide's C ABI (include/cenote_c.h, cenote_guide_*): parameters, a
// forward pass and one training step over host arrays. The tensor-core
// kernels are in guide.cu.
#include <cmath>
#include <cstring>
#include <vector>

#include "guide.h"
#include "runtime.h"

using namespace cn;

namespace {

// Initial weights: uniform in +-sqrt(6 / fan_in) (He et al. 2015, for ReLU
// layers), biases zero, from a splitmix64 stream of the seed.
void init_params(uint64_t seed, std::vector<float>& p) {
    p.assign(guide::PARAMS, 0.0f);
    uint64_t x = seed;
    auto next = [&]() {
        x += 0x9e3779b97f4a7c15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return double(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](uint32_t off, uint32_t n, uint32_t fan_in) {
        const double a = std::sqrt(6.0 / fan_in);
        for (uint32_t i = 0; i < n; ++i) p[off + i] = float((2.0 * next() - 1.0) * a);
    };
    fill(guide::P_W1, guide::HIDDEN * guide::IN, 81);  // 81 of the 96 inputs carry signal
    fill(guide::P_W2, guide::HIDDEN * guide::HIDDEN, guide::HIDDEN);
    fill(guide::P_W3, guide::HIDDEN * guide::HIDDEN, guide::HIDDEN);
    fill(guide::P_W4, guide::OUT * guide::HIDDEN, guide::HIDDEN);
}

int32_t check_err(cenote_guide* g) {
    int e = 0;
    CN_CUDA(cudaMemcpy(&e, g->err.ptr, 4, cudaMemcpyDeviceToHost));
    if (e) {
        CN_CUDA(cudaMemset(g->err.ptr, 0, 4));
        return fail(CENOTE_E_TIMEOUT, "a tensor-core wait of the guide kernels ran out");
    }
    return CENOTE_OK;
}

}  // namespace

extern "C" {

int32_t cenote_guide_create(cenote_context* ctx, uint64_t seed, cenote_guide** out) {
    CN_CHECK(ctx && out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CN_CUDA(cudaSetDevice(ctx->device));
    auto g = std::make_unique<cenote_guide>();
    g->ctx = ctx;
    CN_CUDA(guide::configure(ctx->device, &g->sms));
    const size_t P = guide::PARAMS * 4;
    CN_CUDA(g->params.alloc(P));
    CN_CUDA(g->grad.alloc(P));
    CN_CUDA(g->m.alloc(P));
    CN_CUDA(g->v.alloc(P));
    CN_CUDA(g->w1.alloc(guide::HIDDEN * guide::IN * 2));
    CN_CUDA(g->w2.alloc(guide::HIDDEN * guide::HIDDEN * 2));
    CN_CUDA(g->w3.alloc(guide::HIDDEN * guide::HIDDEN * 2));
    CN_CUDA(g->w4.alloc(guide::OUT_PAD * guide::HIDDEN * 2));
    CN_CUDA(g->b4.alloc(guide::OUT_PAD * 4));
    CN_CUDA(g->err.alloc(16));
    CN_CUDA(g->loss.alloc(16));
    std::vector<float> p;
    init_params(seed, p);
    CN_CUDA(cudaMemcpy(g->params.ptr, p.data(), P, cudaMemcpyHostToDevice));
    CN_CUDA(cudaMemset(g->grad.ptr, 0, P));
    CN_CUDA(cudaMemset(g->m.ptr, 0, P));
    CN_CUDA(cudaMemset(g->v.ptr, 0, P));
    CN_CUDA(cudaMemset(g->err.ptr, 0, 16));
    guide::launch_cast(g->view(), ctx->stream);
    CN_CUDA(cudaGetLastError());
    CN_CUDA(cudaStreamSynchronize(ctx->stream));
    retain(ctx);
    *out = g.release();
    return CENOTE_OK;
}

void cenote_guide_destroy(cenote_guide* g) {
    if (!g) return;
    cenote_context* ctx = g->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete g;
    release(ctx);
}

int32_t cenote_guide_params(cenote_guide* g, float* params) {
    CN_CHECK(g && params, CENOTE_E_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(g->ctx->mu);
    CN_CUDA(cudaSetDevice(g->ctx->device));
    CN_CUDA(cudaStreamSynchronize(g->ctx->stream));
    CN_CUDA(cudaMemcpy(params, g->params.ptr, guide::PARAMS * 4, cudaMemcpyDeviceToHost));
    return CENOTE_OK;
}

int32_t cenote_guide_set_params(cenote_guide* g, const float* params) {
    CN_CHECK(g && params, CENOTE_E_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(g->ctx->mu);
    CN_CUDA(cudaSetDevice(g->ctx->device));
    CN_CUDA(cudaMemcpy(g->params.ptr, params, guide::PARAMS * 4, cudaMemcpyHostToDevice));
    guide::launch_cast(g->view(), g->ctx->stream);
    CN_CUDA(cudaGetLastError());
    return wait_stream(g->ctx->stream, g->ctx->sync_ev, 60000.0);
}

int32_t cenote_guide_forward(cenote_guide* g, const float* feats, uint32_t n, float* out) {
    CN_CHECK(g && feats && out, CENOTE_E_INVALID_ARGUMENT, "null argument");
    if (n == 0) return CENOTE_OK;
    std::lock_guard<std::mutex> lock(g->ctx->mu);
    CN_CUDA(cudaSetDevice(g->ctx->device));
    CN_CUDA(g->ensure(n));
    cudaStream_t s = g->ctx->stream;
    CN_CUDA(cudaMemcpyAsync(g->feats.ptr, feats, size_t(n) * guide::IN * 4, cudaMemcpyHostToDevice, s));
    guide::launch_forward(g->view(), g->feats.as<float>(), n, g->out.as<float>(), nullptr, g->sms, s);
    CN_CUDA(cudaGetLastError());
    CN_CUDA(cudaMemcpyAsync(out, g->out.ptr, size_t(n) * guide::OUT * 4, cudaMemcpyDeviceToHost, s));
    int32_t rc = wait_stream(s, g->ctx->sync_ev, 60000.0);
    if (rc != CENOTE_OK) return rc;
    return check_err(g);
}

int32_t cenote_guide_train_step(cenote_guide* g, const float* feats, const float* dirs, const float* weights,
                                uint32_t n, float lr, float* loss, float* grads) {
    CN_CHECK(g && feats && dirs && weights, CENOTE_E_INVALID_ARGUMENT, "null argument");
    CN_CHECK(n > 0, CENOTE_E_INVALID_ARGUMENT, "empty batch");
    std::lock_guard<std::mutex> lock(g->ctx->mu);
    CN_CUDA(cudaSetDevice(g->ctx->device));
    CN_CUDA(g->ensure(n));
    cudaStream_t s = g->ctx->stream;
    CN_CUDA(cudaMemcpyAsync(g->feats.ptr, feats, size_t(n) * guide::IN * 4, cudaMemcpyHostToDevice, s));
    CN_CUDA(cudaMemcpyAsync(g->dirs.ptr, dirs, size_t(n) * 12, cudaMemcpyHostToDevice, s));
    CN_CUDA(cudaMemcpyAsync(g->weights.ptr, weights, size_t(n) * 4, cudaMemcpyHostToDevice, s));
    CN_CUDA(cudaMemsetAsync(g->loss.ptr, 0, 4, s));
    guide::Buffers b = g->view();
    guide::launch_forward(b, g->feats.as<float>(), n, g->out.as<float>(), g->save.as<__nv_bfloat16>(), g->sms, s);
    guide::launch_loss(b, g->out.as<float>(), g->dirs.as<float>(), g->weights.as<float>(), n, 1.0f / float(n),
                       g->dz4.as<__nv_bfloat16>(), g->loss.as<float>(), s);
    guide::launch_backward(b, g->save.as<__nv_bfloat16>(), g->dz4.as<__nv_bfloat16>(), n, g->sms, s);
    CN_CUDA(cudaGetLastError());
    if (grads) CN_CUDA(cudaMemcpyAsync(grads, g->grad.ptr, guide::PARAMS * 4, cudaMemcpyDeviceToHost, s));
    if (loss) CN_CUDA(cudaMemcpyAsync(loss, g->loss.ptr, 4, cudaMemcpyDeviceToHost, s));
    if (lr > 0.0f) {
        g->step++;
        guide::launch_adam(b, lr, g->step, s);
        guide::launch_cast(b, s);
    } else {
        CN_CUDA(cudaMemsetAsync(g->grad.ptr, 0, guide::PARAMS * 4, s));
    }
    CN_CUDA(cudaGetLastError());
    int32_t rc = wait_stream(s, g->ctx->sync_ev, 60000.0);
    if (rc != CENOTE_OK) return rc;
    return check_err(g);
}

}  // extern "C"
