// integrate.cuh -- host launchers of the per-particle kernels (integrate.cu).
#pragma once

#include "common.cuh"

namespace gsph {

cudaError_t launch_leapfrog(const DevArrays& a, const DevParams& p, int not_first_step, cudaStream_t s);
int leapfrog_kernel_count(const DevParams& p);
size_t diag_scratch_doubles(int64_t n);
cudaError_t launch_diagnostics(const DevArrays& a, const DevParams& p, double half_kick, double* out_dev,
                               cudaStream_t s);
// the same with the pair potential summed in FP32 (compensated across tiles, FP64 across particles)
cudaError_t launch_diagnostics_fast(const DevArrays& a, const DevParams& p, double half_kick, double* out_dev,
                                    cudaStream_t s);
// O(N) comparison of the current state with two saved states (gsph_state_compare); out_dev: 4 doubles
cudaError_t launch_state_compare(const DevArrays& q, const DevArrays& p_state, const DevArrays& x0, const DevParams& p,
                                 double* scratch, double* out_dev, cudaStream_t s);
// gsph_energy_adjust: kinetic energy about the centre of mass and shear energy changed by d_kin and
// d_shear (three launches; tot_dev: kDiagFields doubles of scratch)
cudaError_t launch_energy_adjust(const DevArrays& a, const DevParams& p, double d_kin, double d_shear, double* tot_dev,
                                 cudaStream_t s);
// `ext` (nullable) maps each device slot to the caller's particle index
cudaError_t launch_pack(const DevArrays& a, int attr, const float* src_dev, const int* ext, cudaStream_t s);
cudaError_t launch_unpack(const DevArrays& a, int attr, float* dst_dev, const int* ext, cudaStream_t s);
cudaError_t launch_pack_pos64(const DevArrays& a, const double* src_dev, const int* ext, cudaStream_t s);
cudaError_t launch_unpack_pos64(const DevArrays& a, double* dst_dev, const int* ext, cudaStream_t s);
cudaError_t launch_init_padding(const DevArrays& a, cudaStream_t s);
cudaError_t launch_check_finite(const DevArrays& a, cudaStream_t s);

}  // namespace gsph
