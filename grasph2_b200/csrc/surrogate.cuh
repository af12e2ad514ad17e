// surrogate.cuh -- launchers of the learned surrogate's per-particle kernels (surrogate.cu).
#pragma once

#include "common.cuh"
#include "spatial.cuh"

namespace gsph {

// 32 neighbour-moment features per particle in the caller's order (needs current chunk lists)
cudaError_t launch_features(const DevArrays& a, const DevParams& p, const SpatialArrays& sp, const float* mu,
                            const float* sig, float* feat, cudaStream_t s);
// K-substep proposal: constant-derivative leapfrog extrapolation + the MLP's correction
cudaError_t launch_apply(const DevArrays& a, const DevParams& p, const int* ext, const float* delta, const float* omu,
                         const float* osig, int K, cudaStream_t s);

}  // namespace gsph
