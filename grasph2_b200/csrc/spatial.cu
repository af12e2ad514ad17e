// spatial.cu -- chunk bounding boxes, per-group near-chunk lists, and the Hilbert-curve reorder.
#include <cub/device/device_radix_sort.cuh>

#include "spatial.cuh"

namespace gsph {

namespace {

inline unsigned blocks_for(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

// one warp per chunk: min/max over its real particles (empty chunk: lo = +inf, hi = -inf)
__global__ void k_chunk_bounds(DevArrays a, float4* __restrict__ lo, float4* __restrict__ hi, int64_t nchunks) {
    const int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nchunks) return;
    float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY, mxz = -INFINITY;
    for (int k = lane; k < kChunk; k += 32) {
        const int64_t i = w * kChunk + k;
        if (i < a.n) {
            const float4 p = a.posm[i];
            mnx = fminf(mnx, p.x); mny = fminf(mny, p.y); mnz = fminf(mnz, p.z);
            mxx = fmaxf(mxx, p.x); mxy = fmaxf(mxy, p.y); mxz = fmaxf(mxz, p.z);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mnz = fminf(mnz, __shfl_xor_sync(0xffffffffu, mnz, o));
        mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        mxz = fmaxf(mxz, __shfl_xor_sync(0xffffffffu, mxz, o));
    }
    if (lane == 0) {
        lo[w] = make_float4(mnx, mny, mnz, 0.0f);
        hi[w] = make_float4(mxx, mxy, mxz, 0.0f);
    }
}

__device__ __forceinline__ float gap(float lo_a, float hi_a, float lo_b, float hi_b) {
    return fmaxf(0.0f, fmaxf(lo_b - hi_a, lo_a - hi_b));
}

// one block per i-group: the ordered list of chunks within h of the group's box
constexpr int kListThreads = 256;
__global__ void __launch_bounds__(kListThreads) k_chunk_lists(const float4* __restrict__ lo,
                                                              const float4* __restrict__ hi, int* __restrict__ list,
                                                              int* __restrict__ count, int64_t nchunks, float h2m) {
    constexpr int per_group = kGroup / kChunk;
    const int64_t g = blockIdx.x;
    float4 glo = lo[g * per_group], ghi = hi[g * per_group];
#pragma unroll
    for (int k = 1; k < per_group; ++k) {
        const float4 l = lo[g * per_group + k], u = hi[g * per_group + k];
        glo.x = fminf(glo.x, l.x); glo.y = fminf(glo.y, l.y); glo.z = fminf(glo.z, l.z);
        ghi.x = fmaxf(ghi.x, u.x); ghi.y = fmaxf(ghi.y, u.y); ghi.z = fmaxf(ghi.z, u.z);
    }
    __shared__ int warp_tot[kListThreads / 32];
    __shared__ int base_sh;
    if (threadIdx.x == 0) base_sh = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int* out = list + g * nchunks;
    for (int64_t r = 0; r < nchunks; r += kListThreads) {
        const int64_t c = r + threadIdx.x;
        bool near = false;
        if (c < nchunks) {
            const float4 l = lo[c], u = hi[c];
            const float dx = gap(glo.x, ghi.x, l.x, u.x), dy = gap(glo.y, ghi.y, l.y, u.y),
                        dz = gap(glo.z, ghi.z, l.z, u.z);
            near = dx * dx + dy * dy + dz * dz <= h2m;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, near);
        const int rank = __popc(ballot & ((1u << lane) - 1u));
        __syncthreads();
        if (lane == 0) warp_tot[warp] = __popc(ballot);
        __syncthreads();
        int off = base_sh;
        for (int w = 0; w < warp; ++w) off += warp_tot[w];
        if (near) out[off + rank] = static_cast<int>(c);
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < kListThreads / 32; ++w) t += warp_tot[w];
            base_sh += t;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) count[g] = base_sh;
}

// ---- space-filling-curve reorder ----------------------------------------------------------------
__device__ __forceinline__ int f2o(float f) {  // float -> int with the same order
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_bbox_init(int* bb) {
    if (threadIdx.x < 3) bb[threadIdx.x] = 0x7fffffff;
    else if (threadIdx.x < 6) bb[threadIdx.x] = static_cast<int>(0x80000000u);
}

__global__ void k_bbox(DevArrays a, int* bb) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float4 p = a.posm[i];
        const float v[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (isfinite(v[d])) {
                mn[d] = fminf(mn[d], v[d]);
                mx[d] = fmaxf(mx[d], v[d]);
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(bb + d, f2o(mn[d]));
            atomicMax(bb + 3 + d, f2o(mx[d]));
        }
    }
}

__global__ void k_curve_keys(DevArrays a, const int* bb, unsigned* keys, int* vals) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n_pad) return;
    vals[i] = static_cast<int>(i);
    if (i >= a.n) {
        keys[i] = 0xffffffffu;  // padding stays behind every real particle
        return;
    }
    const float4 p = a.posm[i];
    const float v[3] = {p.x, p.y, p.z};
    unsigned q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float lo = o2f(bb[d]), hi = o2f(bb[3 + d]);
        const float span = hi - lo;
        float t = (span > 0.0f && isfinite(v[d])) ? (v[d] - lo) / span : 0.0f;
        t = fminf(fmaxf(t, 0.0f), 1.0f);
        q[d] = static_cast<unsigned>(t * 1023.0f);
    }
    keys[i] = hilbert3(q[0], q[1], q[2]);
}

template <typename T>
__global__ void k_gather(const T* __restrict__ src, T* __restrict__ dst, const int* __restrict__ order, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[order[i]];
}

__global__ void k_iota(int* v, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) v[i] = static_cast<int>(i);
}

template <typename T>
cudaError_t permute(T* arr, T* tmp, const int* order, int64_t n, cudaStream_t st, int& launches) {
    k_gather<T><<<blocks_for(n, 256), 256, 0, st>>>(arr, tmp, order, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ++launches;
    return cudaMemcpyAsync(arr, tmp, n * sizeof(T), cudaMemcpyDeviceToDevice, st);
}

}  // namespace

size_t spatial_sort_tmp_bytes(int64_t n_pad) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<const unsigned*>(nullptr), static_cast<unsigned*>(nullptr),
                                    static_cast<const int*>(nullptr), static_cast<int*>(nullptr),
                                    static_cast<int>(n_pad));
    return bytes;
}

cudaError_t launch_chunk_bounds(const DevArrays& a, const SpatialArrays& s, cudaStream_t st) {
    const int64_t nchunks = a.n_pad / kChunk;
    k_chunk_bounds<<<blocks_for(nchunks * 32, 256), 256, 0, st>>>(a, s.box_lo, s.box_hi, nchunks);
    return cudaGetLastError();
}

cudaError_t launch_chunk_lists(const DevArrays& a, const SpatialArrays& s, float h, cudaStream_t st) {
    const int64_t nchunks = a.n_pad / kChunk;
    const float hm = h * (1.0f + kMargin);
    k_chunk_lists<<<static_cast<unsigned>(a.n_pad / kGroup), kListThreads, 0, st>>>(s.box_lo, s.box_hi, s.list,
                                                                                     s.count, nchunks, hm * hm);
    return cudaGetLastError();
}

cudaError_t launch_identity_order(const SpatialArrays& s, int64_t n_pad, cudaStream_t st) {
    k_iota<<<blocks_for(n_pad, 256), 256, 0, st>>>(s.ext_of_int, n_pad);
    return cudaGetLastError();
}

cudaError_t reorder_particles(const DevArrays& a, const SpatialArrays& s, cudaStream_t st, int& launches) {
    const int64_t np = a.n_pad;
    k_bbox_init<<<1, 32, 0, st>>>(s.bbox);
    k_bbox<<<256, 256, 0, st>>>(a, s.bbox);
    k_curve_keys<<<blocks_for(np, 256), 256, 0, st>>>(a, s.bbox, s.keys, s.order);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    launches += 3;
    size_t tb = s.sort_tmp_bytes;
    e = cub::DeviceRadixSort::SortPairs(s.sort_tmp, tb, s.keys, s.keys + np, s.order, s.order_out,
                                        static_cast<int>(np), 0, 32, st);
    if (e != cudaSuccess) return e;
    launches += 4;  // onesweep radix sort passes (approximate count for the launch counter)
    return permute_particles(a, s.order_out, s.tmp4, s.tmp8, s.ext_of_int, st, launches);
}

cudaError_t permute_particles(const DevArrays& a, const int* ord, float4* t4, double* t8, int* ext_of_int,
                              cudaStream_t st, int& launches) {
    const int64_t np = a.n_pad;
    cudaError_t e = cudaSuccess;
    float4* f4s[] = {a.posm, a.velrho, a.acc, a.xvel, a.sA, a.sB, a.dA, a.dB, a.jA, a.jB};
    for (float4* arr : f4s) {
        e = permute(arr, t4, ord, np, st, launches);
        if (e != cudaSuccess) return e;
    }
    for (int d = 0; d < 3; ++d) {
        e = permute(a.pos64 + d * np, t8, ord, np, st, launches);
        if (e != cudaSuccess) return e;
    }
    float* tf = reinterpret_cast<float*>(t4);
    e = permute(a.rhodot, tf, ord, np, st, launches);
    if (e == cudaSuccess) e = permute(a.balsara, tf, ord, np, st, launches);
    if (e == cudaSuccess) e = permute(ext_of_int, reinterpret_cast<int*>(t4), ord, np, st, launches);
    return e;
}

}  // namespace gsph
