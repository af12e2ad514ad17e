/*
 * TEST INFRASTRUCTURE ONLY. CUDA stand-in for the parts of mpUtils (>= 0.12, not vendored with GraSPH2
 * and not installed here) that GraSPH2's device code uses, so that the reference's own CUDA path --
 * the tile kernels of src/particles/algorithms.h, the jobs of src/computeDerivatives.h and the
 * integrator of src/integration.h -- compiles unchanged with nvcc for sm_100a (oracle/build_ref.py,
 * into oracle/_ref/libref_cuda_<variant>.so). Written from the call sites' semantics: component-wise
 * vector arithmetic on the CUDA vector types, mpu::Mat<T,R,C> with [r][c] and linear (e) access, a
 * grid-stride index range, the launch-size helper, the template traits the launchers check, and
 * assert_cuda (which throws, as mpUtils' does).
 */
#ifndef GSPH_REF_SHIM_CUDA_MPCUDA_H
#define GSPH_REF_SHIM_CUDA_MPCUDA_H

#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <math.h>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>

#define CUDAHOSTDEV __host__ __device__

#define GSPH_SHIM_V3OPS(V, T)                                                                                  \
    __host__ __device__ inline V operator+(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }             \
    __host__ __device__ inline V operator-(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }             \
    __host__ __device__ inline V operator-(V a) { return V{-a.x, -a.y, -a.z}; }                                 \
    __host__ __device__ inline V operator*(V a, T s) { return V{a.x * s, a.y * s, a.z * s}; }                   \
    __host__ __device__ inline V operator*(T s, V a) { return V{s * a.x, s * a.y, s * a.z}; }                   \
    __host__ __device__ inline V operator/(V a, T s) { return V{a.x / s, a.y / s, a.z / s}; }                   \
    __host__ __device__ inline V& operator+=(V& a, V b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }       \
    __host__ __device__ inline V& operator-=(V& a, V b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }       \
    __host__ __device__ inline V& operator*=(V& a, T s) { a.x *= s; a.y *= s; a.z *= s; return a; }             \
    __host__ __device__ inline V& operator+=(V& a, T s) { a.x += s; a.y += s; a.z += s; return a; }             \
    __host__ __device__ inline T dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }                    \
    __host__ __device__ inline V cross(V a, V b) {                                                            \
        return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};                          \
    }                                                                                                          \
    __host__ __device__ inline T length(V a) { return sqrt(dot(a, a)); }

GSPH_SHIM_V3OPS(float3, float)
GSPH_SHIM_V3OPS(double3, double)
#undef GSPH_SHIM_V3OPS

namespace mpu {

template <typename T, size_t R, size_t C>
struct Mat {
    T d[R * C];
    Mat() = default;
    /* scalar constructor: v on the diagonal; only ever called with 0 by the reference */
    __host__ __device__ Mat(T v) {
        for (size_t i = 0; i < R * C; ++i) d[i] = (i / C == i % C) ? v : T(0);
    }
    __host__ __device__ T* operator[](size_t r) { return d + r * C; }
    __host__ __device__ const T* operator[](size_t r) const { return d + r * C; }
    __host__ __device__ T& operator()(size_t e) { return d[e]; }
    __host__ __device__ const T& operator()(size_t e) const { return d[e]; }
    __host__ __device__ Mat& operator+=(const Mat& o) {
        for (size_t i = 0; i < R * C; ++i) d[i] += o.d[i];
        return *this;
    }
    __host__ __device__ Mat& operator-=(const Mat& o) {
        for (size_t i = 0; i < R * C; ++i) d[i] -= o.d[i];
        return *this;
    }
    __host__ __device__ Mat& operator*=(T s) {
        for (size_t i = 0; i < R * C; ++i) d[i] *= s;
        return *this;
    }
};
template <typename T, size_t R, size_t C>
__host__ __device__ Mat<T, R, C> operator+(Mat<T, R, C> a, const Mat<T, R, C>& b) {
    a += b;
    return a;
}
template <typename T, size_t R, size_t C>
__host__ __device__ Mat<T, R, C> operator*(Mat<T, R, C> a, T s) {
    a *= s;
    return a;
}
template <typename T, size_t R, size_t C>
__host__ __device__ Mat<T, R, C> operator*(T s, Mat<T, R, C> a) {
    for (size_t i = 0; i < R * C; ++i) a.d[i] = s * a.d[i];
    return a;
}
template <typename T, size_t R, size_t C>
__host__ __device__ Mat<T, R, C> operator/(Mat<T, R, C> a, T s) {
    for (size_t i = 0; i < R * C; ++i) a.d[i] /= s;
    return a;
}
/* matrix times column vector, row-major */
__host__ __device__ inline float3 operator*(const Mat<float, 3, 3>& m, float3 v) {
    return float3{m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                  m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}
__host__ __device__ inline double3 operator*(const Mat<double, 3, 3>& m, double3 v) {
    return double3{m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                   m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}

/* grid-stride range over [0, n): this thread's first index, then steps of the whole grid's size */
struct gsph_grid_range {
    size_t first, n, step;
    struct it {
        size_t i, step;
        __device__ size_t operator*() const { return i; }
        __device__ it& operator++() {
            i += step;
            return *this;
        }
        __device__ bool operator!=(const it& o) const { return i < o.i; }
    };
    __device__ it begin() const { return {first, step}; }
    __device__ it end() const { return {n, step}; }
};
template <typename T>
__device__ gsph_grid_range gridStrideRange(T n) {
    return gsph_grid_range{static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x, static_cast<size_t>(n),
                           static_cast<size_t>(gridDim.x) * blockDim.x};
}
/* blocks of bs threads that cover n items (at least one) */
inline int numBlocks(size_t n, size_t bs) { return static_cast<int>(n == 0 ? 1 : (n + bs - 1) / bs); }

template <template <typename...> class Tmpl, typename T>
struct is_instantiation_of : std::false_type {};
template <template <typename...> class Tmpl, typename... A>
struct is_instantiation_of<Tmpl, Tmpl<A...>> : std::true_type {};

template <typename, template <typename> class Op, typename T>
struct gsph_detector : std::false_type {};
template <template <typename> class Op, typename T>
struct gsph_detector<std::void_t<Op<T>>, Op, T> : std::true_type {};
template <template <typename> class Op, typename T>
using is_detected = gsph_detector<void, Op, T>;

}  // namespace mpu

/* assert_cuda: a failed CUDA call throws, as mpUtils' assert_cuda does */
inline void gsph_ref_check_cuda(cudaError_t e, const char* file, int line) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(cudaGetErrorString(e)) + " at " + file + ":" + std::to_string(line));
}
#define assert_cuda(x) gsph_ref_check_cuda((x), __FILE__, __LINE__)

#endif
