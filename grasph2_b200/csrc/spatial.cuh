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

size_t spatial_sort_tmp_bytes(int64_t n_pad);
cudaError_t launch_chunk_bounds(const DevArrays& a, const SpatialArrays& s, cudaStream_t st);
cudaError_t launch_chunk_lists(const DevArrays& a, const SpatialArrays& s, float h, cudaStream_t st);
// Sort the n real particles of `a` along the Hilbert curve and permute every per-particle array in place.
cudaError_t reorder_particles(const DevArrays& a, const SpatialArrays& s, cudaStream_t st, int& launches);
cudaError_t launch_identity_order(const SpatialArrays& s, int64_t n_pad, cudaStream_t st);

}  // namespace gsph
