// spatial.cuh -- particle ordering and chunk culling for the SPH passes.
//
// The reference evaluates every SPH pass over all N^2 pairs and discards those with r > h
// (src/computeDerivatives.h:72, :122, :238). Here particles are kept in Hilbert-curve order inside
// the context, every chunk of kChunk consecutive particles gets an axis-aligned bounding box each step,
// and each i-group of kGroup particles lists the chunks whose box lies within h (times 1 + kMargin) of
// its own box. The density and SPH passes visit only those chunks; gravity still covers all pairs.
// The test is conservative: a pair it skips is farther apart than h in every rounding, so the
// result is the reference's up to summation order. Ordering only affects speed, never correctness.
#pragma once

#include "common.cuh"

namespace gsph {

constexpr int kChunk = 64;     // particles per j-chunk (one bounding box)
constexpr int kGroup = 128;    // particles per i-group (threads of a culled SPH block)
constexpr float kMargin = 1e-3f;

struct SpatialArrays {
    float4* box_lo;    // [n_pad / kChunk]  chunk bounds (x, y, z, unused)
    float4* box_hi;
    int* list;         // [n_pad / kGroup][n_pad / kChunk] near chunks of each i-group
    int* count;        // [n_pad / kGroup]
    int* item_start;   // [n_pad / kGroup + 2] first work item of each group, number of items, chunks per item
    int item_target;   // items aimed at per pass (the item buffer holds item_target + groups items)
    float* item_part;  // [items][fields][kGroup] partial sums of the culled passes
    int* item_nb;      // [items][kItemNb][kGroup] neighbour indices found by the culled density pass
    int* item_nbcnt;   // [items][kGroup]
    int* item_nbover;  // [items] nonzero: some lane's list of the item overflowed
    int* ext_of_int;   // [n_pad] caller's index of the particle stored at each internal slot
    int* order;        // [n_pad] scratch: sort values / gather map
    unsigned* keys;    // [2 n_pad] sort keys (in, out)
    int* order_out;    // [n_pad]
    void* sort_tmp;    // CUB radix-sort scratch
    size_t sort_tmp_bytes;
    int* bbox;         // [6] global bounds as ordered ints
    float4* tmp4;      // [n_pad] permutation scratch
    double* tmp8;      // [3 n_pad]
};

__device__ __forceinline__ unsigned spread10(unsigned v) {  // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// 30-bit Hilbert index of a point on a 1024^3 grid: J. Skilling, "Programming the Hilbert curve",
// AIP Conf. Proc. 707 (2004): the axes are transformed in place into the transposed index
// (inverse undo + Gray encoding), whose bits interleaved from the top give the index. Consecutive
// indices are neighbouring cells, so runs of particles in this order are spatially compact.
__device__ __forceinline__ unsigned hilbert3(unsigned x0, unsigned x1, unsigned x2) {
    unsigned X[3] = {x0, x1, x2};
    constexpr unsigned M = 1u << 9;
    for (unsigned Q = M; Q > 1; Q >>= 1) {
        const unsigned P = Q - 1;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (X[i] & Q) {
                X[0] ^= P;
            } else {
                const unsigned t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    unsigned t = 0;
    for (unsigned Q = M; Q > 1; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1;
    X[0] ^= t; X[1] ^= t; X[2] ^= t;
    return (spread10(X[0]) << 2) | (spread10(X[1]) << 1) | spread10(X[2]);
}

size_t spatial_sort_tmp_bytes(int64_t n_pad);
cudaError_t launch_chunk_bounds(const DevArrays& a, const SpatialArrays& s, cudaStream_t st);
cudaError_t launch_chunk_lists(const DevArrays& a, const SpatialArrays& s, float h, cudaStream_t st);
// Sort the n real particles of `a` along the Hilbert curve and permute every per-particle array in place.
cudaError_t reorder_particles(const DevArrays& a, const SpatialArrays& s, cudaStream_t st, int& launches);
cudaError_t launch_identity_order(const SpatialArrays& s, int64_t n_pad, cudaStream_t st);
// Gather every per-particle array of `a` (all n_pad slots) and `ext_of_int` by `order` (new slot i takes
// old slot order[i]); t4 / t8 are n_pad-element scratch.
cudaError_t permute_particles(const DevArrays& a, const int* order, float4* t4, double* t8, int* ext_of_int,
                              cudaStream_t st, int& launches);

}  // namespace gsph
