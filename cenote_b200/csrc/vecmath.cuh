// float3 arithmetic for the kernels (CUDA's float3 carries no operators).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace cn {

__device__ __forceinline__ float3 f3(float s) { return make_float3(s, s, s); }
__device__ __forceinline__ float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4(float3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3 operator/(float s, float3 a) { return make_float3(s / a.x, s / a.y, s / a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float s) { return make_float3(a.x + s, a.y + s, a.z + s); }
__device__ __forceinline__ float3 operator+(float s, float3 a) { return make_float3(s + a.x, s + a.y, s + a.z); }
__device__ __forceinline__ float3 operator-(float3 a, float s) { return make_float3(a.x - s, a.y - s, a.z - s); }
__device__ __forceinline__ float3 operator-(float s, float3 a) { return make_float3(s - a.x, s - a.y, s - a.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normalize(float3 a) { return a / sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 fabs3(float3 a) { return make_float3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__device__ __forceinline__ float3 fmax3(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
__device__ __forceinline__ float3 fmin3(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ float3 exp3(float3 a) { return make_float3(expf(a.x), expf(a.y), expf(a.z)); }
__device__ __forceinline__ float3 log3(float3 a) { return make_float3(logf(a.x), logf(a.y), logf(a.z)); }
__device__ __forceinline__ float3 pow3(float3 a, float3 b) { return make_float3(powf(a.x, b.x), powf(a.y, b.y), powf(a.z, b.z)); }
__device__ __forceinline__ float3 fma3(float3 a, float3 b, float3 c) {
    return make_float3(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y), fmaf(a.z, b.z, c.z));
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float3 clamp3(float3 a, float lo, float hi) {
    return make_float3(clampf(a.x, lo, hi), clampf(a.y, lo, hi), clampf(a.z, lo, hi));
}
__device__ __forceinline__ float saturatef(float x) { return clampf(x, 0.0f, 1.0f); }
__device__ __forceinline__ float3 saturate3(float3 a) { return clamp3(a, 0.0f, 1.0f); }
// x·(1−t) + y·t, the FMix form the reference's lerp lowers to.
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float3 lerp3(float3 a, float3 b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float3 lerp3(float3 a, float3 b, float3 t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float avg3(float3 v) { return (v.x + v.y + v.z) / 3.0f; }
__device__ __forceinline__ bool any_pos(float3 v) { return v.x > 0.0f || v.y > 0.0f || v.z > 0.0f; }
__device__ __forceinline__ float max3(float3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
__device__ __forceinline__ float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }

}  // namespace cn
