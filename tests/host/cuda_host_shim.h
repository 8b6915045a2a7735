// Host definitions of the handful of CUDA device intrinsics the traversal
// header uses, so tests can compile cenote_b200/csrc/traverse.cuh with g++
// and run the exact kernel traversal code on the CPU. Compiled with
// -ffp-contract=off, the *_rn helpers round exactly like the device ones.
#pragma once
#include <cstdint>
#include <cstring>
#include <cmath>
#include <cuda_runtime.h>

#define __noinline__
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fdiv_rn(float a, float b) { return a / b; }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __ddiv_rn(double a, double b) { return a / b; }
inline float __double2float_rn(double d) { return float(d); }
inline float __uint_as_float(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t __float_as_uint(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline int __clz(uint32_t x) { return x ? __builtin_clz(x) : 32; }
inline int __popc(uint32_t x) { return __builtin_popcount(x); }
// Byte select of the pair (y:x), selector nibbles 0-7 (the sign-replicate
// bit is not used by the library).
inline uint32_t __byte_perm(uint32_t x, uint32_t y, uint32_t s) {
    uint64_t v = (uint64_t(y) << 32) | x;
    uint32_t r = 0;
    for (int k = 0; k < 4; ++k) r |= uint32_t((v >> (8 * ((s >> (4 * k)) & 7u))) & 0xffu) << (8 * k);
    return r;
}
inline int __ffs(uint32_t x) { return __builtin_ffs(int(x)); }
inline uint32_t min(uint32_t a, uint32_t b) { return a < b ? a : b; }
template <class T> inline T __ldg(const T* p) { return *p; }
inline void sincosf(float x, float* s, float* c) { *s = std::sin(x); *c = std::cos(x); }
inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
inline float saturate_host(float x) { return x < 0 ? 0 : (x > 1 ? 1 : x); }
// A pseudo-random lane count, so host runs exercise the traversal's
// postponement path (its result must not depend on those decisions).
// CN_HOST_LANES=1 reports a lone lane every time (the worst case for
// postponement, which must still terminate).
#include <cstdlib>
inline unsigned __activemask() {
    static const bool lone = std::getenv("CN_HOST_LANES") && std::atoi(std::getenv("CN_HOST_LANES")) == 1;
    if (lone) return 1u;
    static thread_local uint32_t x = 0x9e3779b9u;
    x ^= x << 13; x ^= x >> 17; x ^= x << 5;
    uint32_t lanes = x % 33u;
    return lanes == 32u ? 0xffffffffu : ((1u << lanes) - 1u);
}
