// Sobol-Burley sampling on the device: the hash-based Owen-scrambled 2D
// Sobol sequence of crates/cenote/shaders/rng.slang:68-152, with the same
// seeds, salts and dimension registry, computed without tables.
//
// Two identities keep it pure ALU:
//  * the scramble is reverse(LK(reverse(x))), and both Sobol axes are
//    themselves bit-reversals of something cheap, so the reversals cancel:
//      axis 0: reverse(index)          -> scramble = reverse(LK(index))
//      axis 1: reverse(zeta(index))    -> scramble = reverse(LK(zeta(index)))
//  * axis 1's generator is Pascal's triangle mod 2, whose column j has bit
//    (31-i) set iff C(j, i) is odd iff i's bits are a subset of j's (Lucas).
//    So reversed output bit i = XOR over supersets j of i of index bit j: the
//    GF(2) superset-sum ("zeta") transform, five shift-mask-xor steps.
#pragma once
#include <cstdint>

namespace cn {

constexpr uint32_t CAMERA_JITTER = 0, CAMERA_LENS = 1, PATH_BASE = 8;
constexpr uint32_t BSDF_LOBE = 0, BSDF_DIR = 1, NEE_LIGHT = 2, NEE_POINT = 3, RR = 4, BOUNCE_SLOTS = 8;

__device__ __forceinline__ uint32_t bounce_dim(uint32_t bounce, uint32_t slot) {
    return PATH_BASE + bounce * BOUNCE_SLOTS + slot;
}

__device__ __forceinline__ uint32_t lowbias32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x21f0aaadu;
    x ^= x >> 15;
    x *= 0xd35a2d97u;
    x ^= x >> 15;
    return x;
}

__device__ __forceinline__ uint32_t laine_karras(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}

__device__ __forceinline__ uint32_t superset_xor(uint32_t x) {
    x ^= (x >> 1) & 0x55555555u;
    x ^= (x >> 2) & 0x33333333u;
    x ^= (x >> 4) & 0x0f0f0f0fu;
    x ^= (x >> 8) & 0x00ff00ffu;
    x ^= (x >> 16) & 0x0000ffffu;
    return x;
}

__device__ __forceinline__ float unit_float(uint32_t x) { return float(x >> 8) * (1.0f / 16777216.0f); }

// nestedUniformScramble(sampleIndex, seed) = reverse(LK(reverse(i), seed)).
__device__ __forceinline__ uint32_t shuffle_index(uint32_t i, uint32_t seed) {
    return __brev(laine_karras(__brev(i), seed));
}

__device__ __forceinline__ float2 sample_2d(uint32_t pixel, uint32_t sample, uint32_t dimension) {
    uint32_t seed = lowbias32(pixel ^ lowbias32(dimension));
    uint32_t index = shuffle_index(sample, lowbias32(seed ^ 0xf8ade99au));
    float x = unit_float(__brev(laine_karras(index, lowbias32(seed ^ 0xe0aaaf76u))));
    float y = unit_float(__brev(laine_karras(superset_xor(index), lowbias32(seed ^ 0x94964d4eu))));
    return make_float2(x, y);
}

__device__ __forceinline__ float sample_1d(uint32_t pixel, uint32_t sample, uint32_t dimension) {
    uint32_t seed = lowbias32(pixel ^ lowbias32(dimension));
    uint32_t index = shuffle_index(sample, lowbias32(seed ^ 0xbff95bfeu));
    return unit_float(__brev(laine_karras(index, lowbias32(seed ^ 0x635fc02fu))));
}

// The transparency chain's plain hash stream (rng.slang:128-132).
__device__ __forceinline__ float hash_uniform(uint32_t pixel, uint32_t sample, uint32_t bounce, uint32_t crossing) {
    uint32_t h = lowbias32(pixel ^ lowbias32(sample ^ 0x9e3779b9u));
    h = lowbias32(h ^ (bounce << 8 | crossing));
    return unit_float(h);
}

}  // namespace cn
