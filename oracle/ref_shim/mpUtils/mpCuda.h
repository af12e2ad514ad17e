/*
 * TEST INFRASTRUCTURE ONLY. Host stand-in for the parts of mpUtils (>= 0.12, not vendored with
 * GraSPH2 and not installed here) that GraSPH2's physics headers use, so that those headers --
 * src/computeDerivatives.h, src/integration.h, src/sph/{kernel,eos,models}.h -- compile unchanged
 * with g++ for the CPU parity build under oracle/_ref. Written from the call sites' semantics:
 * CUDA vector structs with component-wise arithmetic, mpu::Mat<T,R,C> with [r][c] and linear (e)
 * access, and empty CUDA qualifiers so __device__/__global__ functions become host functions.
 */
#ifndef GSPH_REF_SHIM_MPCUDA_H
#define GSPH_REF_SHIM_MPCUDA_H

#include <cmath>
#include <math.h>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <tuple>
#include <type_traits>
#include <algorithm>

#define __host__
#define __device__
#define __global__
#define __shared__
#define __forceinline__ inline
#define CUDAHOSTDEV

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct double2 { double x, y; };
struct double3 { double x, y, z; };
struct double4 { double x, y, z, w; };

#define GSPH_SHIM_V3OPS(V, T)                                                                  \
    inline V operator+(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }                \
    inline V operator-(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }                \
    inline V operator-(V a) { return V{-a.x, -a.y, -a.z}; }                                    \
    inline V operator*(V a, T s) { return V{a.x * s, a.y * s, a.z * s}; }                      \
    inline V operator*(T s, V a) { return V{s * a.x, s * a.y, s * a.z}; }                      \
    inline V operator/(V a, T s) { return V{a.x / s, a.y / s, a.z / s}; }                      \
    inline V& operator+=(V& a, V b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }          \
    inline V& operator-=(V& a, V b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }          \
    inline V& operator*=(V& a, T s) { a.x *= s; a.y *= s; a.z *= s; return a; }                \
    inline V& operator+=(V& a, T s) { a.x += s; a.y += s; a.z += s; return a; }                \
    inline T dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }                       \
    inline V cross(V a, V b) { return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; } \
    inline T length(V a) { return std::sqrt(dot(a, a)); }

GSPH_SHIM_V3OPS(float3, float)
GSPH_SHIM_V3OPS(double3, double)
#undef GSPH_SHIM_V3OPS

inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
inline float max(float a, float b) { return a > b ? a : b; }
inline double max(double a, double b) { return a > b ? a : b; }
inline float min(float a, float b) { return a < b ? a : b; }
inline double min(double a, double b) { return a < b ? a : b; }

/* one host "thread": the device kernels of src/integration.h run as plain loops */
struct gsph_shim_dim3 { unsigned x, y, z; };
static const gsph_shim_dim3 threadIdx = {0, 0, 0};
static const gsph_shim_dim3 blockIdx = {0, 0, 0};
static const int warpSize = 32;
inline int atomicMin(int* a, int v) { int o = *a; if (v < o) *a = v; return o; }
inline long long atomicMin(long long* a, long long v) { long long o = *a; if (v < o) *a = v; return o; }

namespace cub {
struct Min {};
template <class T>
struct WarpReduce {
    struct TempStorage {};
    explicit WarpReduce(TempStorage&) {}
    T Reduce(T v, Min) { return v; }  /* a single lane per "warp" on the host */
};
}  // namespace cub

namespace mpu {

template <typename T, size_t R, size_t C>
struct Mat {
    T d[R * C];
    Mat() = default;
    /* scalar constructor: v on the diagonal; only ever called with 0 by the reference */
    Mat(T v) { for (size_t i = 0; i < R * C; ++i) d[i] = (i / C == i % C) ? v : T(0); }
    T* operator[](size_t r) { return d + r * C; }
    const T* operator[](size_t r) const { return d + r * C; }
    T& operator()(size_t e) { return d[e]; }
    const T& operator()(size_t e) const { return d[e]; }
    Mat& operator+=(const Mat& o) { for (size_t i = 0; i < R * C; ++i) d[i] += o.d[i]; return *this; }
    Mat& operator-=(const Mat& o) { for (size_t i = 0; i < R * C; ++i) d[i] -= o.d[i]; return *this; }
    Mat& operator*=(T s) { for (size_t i = 0; i < R * C; ++i) d[i] *= s; return *this; }
};
template <typename T, size_t R, size_t C>
Mat<T, R, C> operator+(Mat<T, R, C> a, const Mat<T, R, C>& b) { a += b; return a; }
template <typename T, size_t R, size_t C>
Mat<T, R, C> operator*(Mat<T, R, C> a, T s) { a *= s; return a; }
template <typename T, size_t R, size_t C>
Mat<T, R, C> operator*(T s, Mat<T, R, C> a) { for (size_t i = 0; i < R * C; ++i) a.d[i] = s * a.d[i]; return a; }
template <typename T, size_t R, size_t C>
Mat<T, R, C> operator/(Mat<T, R, C> a, T s) { for (size_t i = 0; i < R * C; ++i) a.d[i] /= s; return a; }
/* matrix times column vector, row-major */
inline float3 operator*(const Mat<float, 3, 3>& m, float3 v) {
    return float3{m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                  m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}
inline double3 operator*(const Mat<double, 3, 3>& m, double3 v) {
    return double3{m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                   m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}

/* integer grid-stride range: one host thread covers [0, n) */
struct gsph_range {
    size_t n;
    struct it { size_t i; size_t operator*() const { return i; } it& operator++() { ++i; return *this; }
                bool operator!=(const it& o) const { return i != o.i; } };
    it begin() const { return {0}; }
    it end() const { return {n}; }
};
template <typename T>
gsph_range gridStrideRange(T n) { return gsph_range{static_cast<size_t>(n)}; }
inline size_t numBlocks(size_t n, size_t bs) { return (n + bs - 1) / bs; }

template <template <typename...> class Tmpl, typename T>
struct is_instantiation_of : std::false_type {};
template <template <typename...> class Tmpl, typename... A>
struct is_instantiation_of<Tmpl, Tmpl<A...>> : std::true_type {};

}  // namespace mpu

#endif
