// Test infrastructure: the CPU oracle's 3-vector, templated on the scalar so
// the same restatement runs in FP32 (mirroring the kernels' rounding) and in
// FP64 (the reference value the FP32 kernels are judged against).
//
// This file, like everything under oracle/, is the checker only: the shipped
// library never includes, links or runs it.
#pragma once
#include <cmath>
#include <cstdint>
#include <algorithm>

namespace oracle {

template <class T>
struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    explicit V3(T s) : x(s), y(s), z(s) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    template <class U>
    explicit V3(const V3<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator+(V3<T> a, T s) { return {a.x + s, a.y + s, a.z + s}; }
template <class T> inline V3<T> operator+(T s, V3<T> a) { return {s + a.x, s + a.y, s + a.z}; }
template <class T> inline V3<T> operator-(V3<T> a, T s) { return {a.x - s, a.y - s, a.z - s}; }
template <class T> inline V3<T> operator-(T s, V3<T> a) { return {s - a.x, s - a.y, s - a.z}; }
template <class T> inline V3<T> operator/(T s, V3<T> a) { return {s / a.x, s / a.y, s / a.z}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }

template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> inline V3<T> normalize(V3<T> a) { return a / std::sqrt(dot(a, a)); }
template <class T> inline V3<T> vabs(V3<T> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
template <class T> inline V3<T> vmax(V3<T> a, V3<T> b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
template <class T> inline V3<T> vmin(V3<T> a, V3<T> b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
template <class T> inline V3<T> vexp(V3<T> a) { return {std::exp(a.x), std::exp(a.y), std::exp(a.z)}; }
template <class T> inline V3<T> vlog(V3<T> a) { return {std::log(a.x), std::log(a.y), std::log(a.z)}; }
template <class T> inline V3<T> vpow(V3<T> a, V3<T> b) { return {std::pow(a.x, b.x), std::pow(a.y, b.y), std::pow(a.z, b.z)}; }
template <class T> inline V3<T> vfma(V3<T> a, V3<T> b, V3<T> c) {
    return {std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y), std::fma(a.z, b.z, c.z)};
}
template <class T> inline bool any_gt0(V3<T> a) { return a.x > 0 || a.y > 0 || a.z > 0; }
template <class T> inline T clampv(T x, T lo, T hi) { return std::min(std::max(x, lo), hi); }
template <class T> inline V3<T> vclamp(V3<T> a, T lo, T hi) { return {clampv(a.x, lo, hi), clampv(a.y, lo, hi), clampv(a.z, lo, hi)}; }
template <class T> inline T saturate(T x) { return clampv(x, T(0), T(1)); }
template <class T> inline V3<T> vsaturate(V3<T> a) { return vclamp(a, T(0), T(1)); }
// Slang's lerp lowers to SPIR-V FMix: x·(1−a) + y·a.
template <class T> inline T lerp(T a, T b, T t) { return a * (T(1) - t) + b * t; }
template <class T> inline V3<T> lerp(V3<T> a, V3<T> b, T t) { return a * (T(1) - t) + b * t; }
template <class T> inline V3<T> lerp(V3<T> a, V3<T> b, V3<T> t) { return a * (T(1) - t) + b * t; }
template <class T> inline T average(V3<T> v) { return (v.x + v.y + v.z) / T(3); }
template <class T> inline T signum(T x) { return x > 0 ? T(1) : (x < 0 ? T(-1) : T(0)); }

using V3f = V3<float>;

}  // namespace oracle
