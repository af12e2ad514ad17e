// fp64.cuh -- the double-precision build of the hot path (fp64.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/grasph2_b200.h"

namespace gsph {

struct DevParams64 {
    uint32_t flags;
    int dim;
    double H, H2, eps2, G, w_pref, dw_pref;
    double rho0, bulk, dbulk, c, shear, Y, tanfr, cohesion, alpha, beta;
    double mateps, matexp, inv_w_normalsep, xsph;
    double fixed_dt, initial_dt, min_dt, max_dt, accel_acc, vel_acc, cw_n;
    double const_acc[3], box_min[3], box_max[3], box_refl;
};

// Same roles as DevArrays, all in double4 / double; positions live in posm (x, y, z, m).
struct DevArrays64 {
    int64_t n, n_pad;
    double4 *posm, *velrho, *acc, *xvel, *sA, *sB, *dA, *dB, *jA, *jB;
    double *rhodot, *balsara;
    double* dt_state;  // [0] current, [1] next
};

DevParams64 make_dev_params64(const gsph_params& p, double w_pref, double dw_pref, double inv_w_normalsep);
cudaError_t launch64_init(const DevArrays64& a, cudaStream_t s);
cudaError_t launch64_derivatives(const DevArrays64& a, const DevParams64& p, cudaStream_t s, int& launches);
cudaError_t launch64_leapfrog(const DevArrays64& a, const DevParams64& p, int not_first_step, cudaStream_t s,
                              int& launches);
cudaError_t launch64_pack(const DevArrays64& a, int attr, const float* src, cudaStream_t s);
cudaError_t launch64_unpack(const DevArrays64& a, int attr, float* dst, cudaStream_t s);
cudaError_t launch64_unpack_d(const DevArrays64& a, int attr, double* dst, cudaStream_t s);
cudaError_t launch64_pack_pos(const DevArrays64& a, const double* src, cudaStream_t s);
cudaError_t launch64_pack_f64(const DevArrays64& a, int attr, const double* src, cudaStream_t s);
cudaError_t launch64_unpack_f64(const DevArrays64& a, int attr, double* dst, cudaStream_t s);
cudaError_t launch_narrow(const double* in, float* out, int64_t n, cudaStream_t s);
cudaError_t launch_widen(const float* in, double* out, int64_t n, cudaStream_t s);
size_t diag64_scratch_doubles(int64_t n_pad);
cudaError_t launch64_diagnostics(const DevArrays64& a, const DevParams64& p, double half_kick, double* scratch,
                                 double* out, cudaStream_t s);

}  // namespace gsph
