// Test infrastructure (CPU oracle): Sobol-Burley sampling restated from
// crates/cenote/shaders/rng.slang. Integer arithmetic throughout, so the
// kernels' sampler must agree with these values bit for bit.
#pragma once
#include <cstdint>

namespace oracle {

// Dimension registry, rng.slang:29-47.
constexpr uint32_t CAMERA_JITTER = 0;
constexpr uint32_t CAMERA_LENS = 1;
constexpr uint32_t PATH_BASE = 8;
constexpr uint32_t BSDF_LOBE = 0;
constexpr uint32_t BSDF_DIR = 1;
constexpr uint32_t NEE_LIGHT = 2;
constexpr uint32_t NEE_POINT = 3;
constexpr uint32_t RR = 4;
constexpr uint32_t BOUNCE_SLOTS = 8;

inline uint32_t bounce_dimension(uint32_t bounce, uint32_t slot) {  // rng.slang:45-47
    return PATH_BASE + bounce * BOUNCE_SLOTS + slot;
}

inline uint32_t lowbias32(uint32_t x) {  // rng.slang:68-75
    x ^= x >> 16;
    x *= 0x21f0aaadu;
    x ^= x >> 15;
    x *= 0xd35a2d97u;
    x ^= x >> 15;
    return x;
}

inline uint32_t reverse_bits(uint32_t x) {
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) {
        r = (r << 1) | (x & 1u);
        x >>= 1;
    }
    return r;
}

inline uint32_t laine_karras(uint32_t x, uint32_t seed) {  // rng.slang:81-88
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}

inline uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {  // rng.slang:93-95
    return reverse_bits(laine_karras(reverse_bits(x), seed));
}

// The second Sobol axis' generator column k (rng.slang:55-64): Pascal's
// triangle mod 2, i.e. column k = column(k-1) XOR (column(k-1) >> 1).
inline uint32_t sobol_dim1_column(uint32_t k) {
    uint32_t v = 0x80000000u;
    for (uint32_t i = 0; i < k; ++i) v ^= v >> 1;
    return v;
}

inline uint32_t sobol(uint32_t index, uint32_t axis) {  // rng.slang:100-111
    if (axis == 0) return reverse_bits(index);
    uint32_t value = 0;
    for (uint32_t bit = 0; index != 0; bit++, index >>= 1) {
        if (index & 1u) value ^= sobol_dim1_column(bit);
    }
    return value;
}

inline float to_unit_float(uint32_t x) {  // rng.slang:114-116
    return float(x >> 8) * (1.0f / 16777216.0f);
}

inline float scrambled_sobol(uint32_t index, uint32_t axis, uint32_t seed) {  // rng.slang:119-121
    return to_unit_float(nested_uniform_scramble(sobol(index, axis), seed));
}

inline float hash_uniform(uint32_t pixel, uint32_t sample_index, uint32_t bounce,
                          uint32_t crossing) {  // rng.slang:128-132
    uint32_t h = lowbias32(pixel ^ lowbias32(sample_index ^ 0x9e3779b9u));
    h = lowbias32(h ^ (bounce << 8 | crossing));
    return to_unit_float(h);
}

struct F2 {
    float x, y;
};

inline F2 sample_2d(uint32_t pixel, uint32_t sample_index, uint32_t dimension) {  // rng.slang:140-145
    uint32_t seed = lowbias32(pixel ^ lowbias32(dimension));
    uint32_t index = nested_uniform_scramble(sample_index, lowbias32(seed ^ 0xf8ade99au));
    return {scrambled_sobol(index, 0, lowbias32(seed ^ 0xe0aaaf76u)),
            scrambled_sobol(index, 1, lowbias32(seed ^ 0x94964d4eu))};
}

inline float sample_1d(uint32_t pixel, uint32_t sample_index, uint32_t dimension) {  // rng.slang:148-152
    uint32_t seed = lowbias32(pixel ^ lowbias32(dimension));
    uint32_t index = nested_uniform_scramble(sample_index, lowbias32(seed ^ 0xbff95bfeu));
    return scrambled_sobol(index, 0, lowbias32(seed ^ 0x635fc02fu));
}

}  // namespace oracle
