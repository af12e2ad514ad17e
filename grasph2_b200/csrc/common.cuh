// common.cuh -- device-side building blocks shared by the grasph2_b200 kernels (sm_100a).
//
//  * DevParams: the runtime physics parameters (gsph_params) rounded to FP32 once on the host,
//    plus the derived constants the pair loops need (H^2, 1/H, spline prefactors, eps^2).
//  * DevArrays: the device-resident particle state, structure-of-arrays in HBM.
//  * mbarrier + cp.async.bulk wrappers for the shared-memory j-tile pipeline. Waits are bounded
//    by the global timer: a wait that gives up records GSPH_DEV_ERR_TIMEOUT in the status word
//    and the kernel leaves its loop instead of spinning forever.
//  * Kahan-Babuska fold for the compensated accumulation mode.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/grasph2_b200.h"

namespace gsph {

constexpr int kPad = 1024;            // particle arrays are padded to a multiple of this
constexpr int kMaxSplit = 64;         // most j-segments per i-block
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s bound on any device-side wait

// device status word values
constexpr int GSPH_DEV_ERR_TIMEOUT = 1;

struct DevParams {
    uint32_t flags;
    int dim;
    float H, H2, inv_h, eps2, G;
    float w_pref, dw_pref;      // spline prefactors (src/sph/kernel.h:56-60, :83-87)
    float rho0, bulk, dbulk, c, c2, shear;
    float Y, tanfr, cohesion;
    float alpha, beta;          // AV strength and signal-velocity coefficient
    float mateps, matexp, inv_w_normalsep, xsph;
    float fixed_dt, initial_dt, min_dt, max_dt, accel_acc, vel_acc;
    float cw_n;
    float const_acc[3], box_min[3], box_max[3], box_refl;
    float balsara_floor;        // 1e-4 c / h of balsaraSwitch (src/sph/models.h:191)
    double eps2_d, G_d;         // FP64 copies for the diagnostics
};

__host__ __device__ inline bool has(const DevParams& p, uint32_t f) { return (p.flags & f) != 0; }

// Symmetric 3x3 tensors are stored as two float4 streams: A = (xx, yy, zz, xy), B = (xz, yz, *, *).
struct DevArrays {
    int64_t n, n_pad;
    float4* posm;     // x, y, z, m          (FP32 copy of the FP64 master, for the pair loops)
    double* pos64;    // [3][n_pad] SoA      (FP64 master positions; leapfrog drift)
    float4* velrho;   // vx, vy, vz, rho
    float4* acc;      // ax, ay, az, max_vsig
    float4* xvel;     // XSPH velocity correction
    float4* sA;       // deviatoric stress S
    float4* sB;
    float4* dA;       // dS/dt
    float4* dB;
    float* rhodot;    // drho/dt
    float* balsara;   // Balsara switch
    float4* jA;       // j-record: sigma/rho^2 (xx, yy, zz, xy)
    float4* jB;       // j-record: sigma/rho^2 (xz, yz), balsara, 0
    float4* jrec;     // nullable: [n_pad][4] = posm, velrho, jA, jB packed per particle (one 64-byte line
                      // per neighbour for the culled SPH passes' gathers), rebuilt with jA / jB
    float* part;      // j-split partial sums [segment][component][n_pad]
    float* gpart;     // gravity partial sums of the culled path [segment][component][n_pad]
    double* gfold;    // [3][n_pad]: FP64 sums of those partials (k_gravity_fold), read by the SPH finish
    float* dt_state;  // variable step: [0] current, [1] next (float bit patterns, positive)
    float4* grav;     // gravitational acceleration of the last derivative evaluation (nullable)
    double* diag;     // diagnostics scratch
    int* status;      // device status word (0 = ok)
};

// ---- mbarrier / bulk copy (PTX ISA: mbarrier, cp.async.bulk) --------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait on phase `parity`; false (and status set) when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* status) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_timer_ns() - t0 > kWaitLimitNs) {
            atomicExch(status, GSPH_DEV_ERR_TIMEOUT);
            return false;
        }
    }
    return true;
}
// 1-D bulk copy global -> shared of this CTA, completing on `bar` (no multicast).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// ---- compensated accumulation --------------------------------------------------------------
// Kahan-Babuska (Neumaier) fold of a tile partial `x` into the running pair (s, c): s + c is the
// sum; c collects the rounding error of every fold exactly (two-sum).
__device__ __forceinline__ void fold(float& s, float& c, float x) {
    const float t = s + x;
    const float e = (fabsf(s) >= fabsf(x)) ? ((s - t) + x) : ((x - t) + s);
    s = t;
    c += e;
}

// ---- warp butterflies (the ensemble's symmetric gravity stage) ----------------------------------
// NV values per lane (NV = 4 or 8) -> lane l holds the warp's sum of value (l >> (5 - log2 NV)) & (NV - 1):
// a butterfly that halves the values at each of the first log2 NV levels (fixed order, so the sums are
// the same on every run)
__device__ __forceinline__ void reduce_lanes(float (&v)[8], int lane) {
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const float send = b4 ? v[m] : v[m + 4], keep = b4 ? v[m + 4] : v[m];
        v[m] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const float send = b3 ? v[m] : v[m + 2], keep = b3 ? v[m + 2] : v[m];
        v[m] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const float send = b2 ? v[0] : v[1], keep = b2 ? v[1] : v[0];
    v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
}
__device__ __forceinline__ void reduce_lanes(float (&v)[4], int lane) {
    const bool b4 = lane & 16, b3 = lane & 8;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const float send = b4 ? v[m] : v[m + 2], keep = b4 ? v[m + 2] : v[m];
        v[m] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    const float send = b3 ? v[0] : v[1], keep = b3 ? v[1] : v[0];
    v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 4);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// ---- symmetric tensor helpers ----------------------------------------------------------------
struct Sym {
    float xx, yy, zz, xy, xz, yz;
};
__device__ __forceinline__ Sym sym_load(const float4 a, const float4 b) { return {a.x, a.y, a.z, a.w, b.x, b.y}; }

}  // namespace gsph
