// integrate.cu -- per-particle kernels: the leapfrog (src/integration.h), the variable-step
// reduction, FP64 diagnostics, and the host-layout pack/unpack used by upload/download.
//
// HBM-bound: each kernel touches each particle once with coalesced float4 / double streams.
#include "integrate.cuh"
#include "sph.cuh"

namespace gsph {

namespace {

inline unsigned blocks_for(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

__global__ void k_leapfrog_fixed(DevArrays a, DevParams p, float kick_dt) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    kick_drift(a, p, i, kick_dt, p.fixed_dt);
}

// variableTsLeapfrog_getNewTimestep (integration.h:130-169): closing half kick with the current
// step and the min of the step criteria; block min, then an integer atomicMin on the positive
// float's bit pattern
__global__ void k_dt_criteria(DevArrays a, DevParams p) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const float dt = a.dt_state[0];
    float mindt = p.max_dt;
    if (i < a.n) {
        float4 vr = a.velrho[i];
        const float4 ac = a.acc[i];
        vr.x = fmaf(ac.x, dt * 0.5f, vr.x);
        vr.y = fmaf(ac.y, dt * 0.5f, vr.y);
        vr.z = fmaf(ac.z, dt * 0.5f, vr.z);
        a.velrho[i] = vr;
        if (has(p, GSPH_ACCELERATION_CRITERION))
            mindt = fminf(mindt, sqrtf(p.accel_acc * p.H / sqrtf(ac.x * ac.x + ac.y * ac.y + ac.z * ac.z)));
        if (has(p, GSPH_VELOCITY_CRITERION)) mindt = fminf(mindt, p.vel_acc * p.H / ac.w);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mindt = fminf(mindt, __shfl_xor_sync(0xffffffffu, mindt, o));
    __shared__ float wmin[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wmin[warp] = mindt;
    __syncthreads();
    if (warp == 0) {
        mindt = (lane < static_cast<int>(blockDim.x >> 5)) ? wmin[lane] : p.max_dt;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mindt = fminf(mindt, __shfl_xor_sync(0xffffffffu, mindt, o));
        if (lane == 0) atomicMin(reinterpret_cast<int*>(a.dt_state + 1), __float_as_int(mindt));
    }
}

__global__ void k_dt_first(DevArrays a, DevParams p) {
    if (threadIdx.x == 0 && blockIdx.x == 0) a.dt_state[1] = p.initial_dt;  // integration.h:235-236
}

// variableTsLeapfrog_useNewTimestep (integration.h:171-217)
__global__ void k_leapfrog_variable(DevArrays a, DevParams p) {
    const float nxt = a.dt_state[1];
    const float dt = nxt < p.min_dt ? p.min_dt : nxt;
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    kick_drift(a, p, i, dt * 0.5f, dt);
}

// commit the step chosen above as the current one (after every block has read `next`)
__global__ void k_dt_commit(DevArrays a, DevParams p) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const float nxt = a.dt_state[1];
        a.dt_state[0] = nxt < p.min_dt ? p.min_dt : nxt;
    }
}

// ---- FP64 diagnostics ---------------------------------------------------------------------------
constexpr int kDiagFields = 12;  // e_kin, e_grav, e_int, e_shear, px, py, pz, lx, ly, lz, mass, (pad)
constexpr int kDiagThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) r += sh[w];  // fixed order
    return r;
}

// per-particle terms and, per i, its share of the pair potential against j > i; one row of
// kDiagFields block partials per CTA (deterministic second stage)
__global__ void __launch_bounds__(kDiagThreads) k_diag(DevArrays a, DevParams p, double half_kick) {
    __shared__ double tile[4][kDiagThreads];
    __shared__ double red[32];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t np = a.n_pad;
    double f[kDiagFields];
#pragma unroll
    for (int k = 0; k < kDiagFields; ++k) f[k] = 0.0;
    double xi = 0, yi = 0, zi = 0, mi = 0;
    if (i < a.n) {
        diag_terms(a, p, i, half_kick, f);
        mi = a.posm[i].w;
        xi = a.pos64[i]; yi = a.pos64[np + i]; zi = a.pos64[2 * np + i];
    }
    // pair potential: -G m_i sum_{j>i} m_j / sqrt(r^2 + eps^2), j-tiles of blockDim through shared memory
    if (has(p, GSPH_SELF_GRAVITY)) {
        const double eps2 = p.eps2_d;
        double phi = 0.0;
        const int64_t j_first = static_cast<int64_t>(blockIdx.x) * blockDim.x;  // j > i needs j >= block start
        for (int64_t t0 = j_first; t0 < a.n; t0 += blockDim.x) {
            const int64_t j = t0 + threadIdx.x;
            __syncthreads();
            if (j < a.n) {
                tile[0][threadIdx.x] = a.pos64[j];
                tile[1][threadIdx.x] = a.pos64[np + j];
                tile[2][threadIdx.x] = a.pos64[2 * np + j];
                tile[3][threadIdx.x] = a.posm[j].w;
            } else {
                tile[3][threadIdx.x] = 0.0;
                tile[0][threadIdx.x] = tile[1][threadIdx.x] = tile[2][threadIdx.x] = 0.0;
            }
            __syncthreads();
            if (i < a.n) {
                const int64_t rem = a.n - t0;
                const int cnt = rem < static_cast<int64_t>(blockDim.x) ? static_cast<int>(rem) : static_cast<int>(blockDim.x);
                for (int jj = 0; jj < cnt; ++jj) {
                    if (t0 + jj <= i) continue;
                    const double dx = tile[0][jj] - xi, dy = tile[1][jj] - yi, dz = tile[2][jj] - zi;
                    phi += tile[3][jj] / sqrt(dx * dx + dy * dy + dz * dz + eps2);
                }
            }
        }
        f[1] = -p.G_d * mi * phi;
    }
    for (int k = 0; k < kDiagFields; ++k) {
        const double s = block_sum(f[k], red);
        if (threadIdx.x == 0) a.diag[static_cast<int64_t>(blockIdx.x) * kDiagFields + k] = s;
    }
}

// The same fields with the pair potential in FP32: per i, FP32 sums over j-tiles folded with a two-sum
// (Kahan-Babuska), then FP64 across particles; the self pair is skipped by index. Relative error of
// the potential energy ~1e-7, at the cost of one FP32 N^2 sweep instead of an FP64 one.
__global__ void __launch_bounds__(kDiagThreads) k_diag_fast(DevArrays a, DevParams p, double half_kick) {
    __shared__ float4 tile[kDiagThreads];
    __shared__ double red[32];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double f[kDiagFields];
#pragma unroll
    for (int k = 0; k < kDiagFields; ++k) f[k] = 0.0;
    const bool valid = i < a.n;
    if (valid) diag_terms(a, p, i, half_kick, f);
    if (has(p, GSPH_SELF_GRAVITY)) {
        const float4 xi = a.posm[valid ? i : 0];
        float s = 0.0f, c = 0.0f;
        for (int64_t t0 = 0; t0 < a.n; t0 += blockDim.x) {
            const int64_t j = t0 + threadIdx.x;
            __syncthreads();
            tile[threadIdx.x] = j < a.n ? a.posm[j] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            __syncthreads();
            float ts = 0.0f;
            const int cnt = static_cast<int>(min(static_cast<int64_t>(blockDim.x), a.n - t0));
            for (int jj = 0; jj < cnt; ++jj) {
                const float4 q = tile[jj];
                const float dx = q.x - xi.x, dy = q.y - xi.y, dz = q.z - xi.z;
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, p.eps2)));
                const float v = q.w * rsqrtf(r2);
                ts += (t0 + jj == i) ? 0.0f : v;
            }
            fold(s, c, ts);
        }
        f[1] = -0.5 * p.G_d * static_cast<double>(xi.w) * (static_cast<double>(s) + static_cast<double>(c));
        if (!valid) f[1] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < kDiagFields; ++k) {
        const double sum = block_sum(f[k], red);
        if (threadIdx.x == 0) a.diag[static_cast<int64_t>(blockIdx.x) * kDiagFields + k] = sum;
    }
}

// Comparison of the current state Q with a saved state P (and a saved start state X0), O(N):
//   0: E_local(P) - E_local(Q) - sum_i m_i g_i . (x_P,i - x_Q,i)    (kinetic + internal + shear energy
//      exactly, the gravitational energy change to first order in the position difference, g = the
//      gravitational acceleration of Q's last derivative evaluation)
//   1: sum_i |x_P,i - x_Q,i|^2      2: sum_i |x_Q,i - x_0,i|^2      3: E_local(Q)
//   4-7: the parts of field 0: kinetic, internal, shear, first-order gravitational
__global__ void __launch_bounds__(kDiagThreads) k_state_compare(DevArrays q, DevArrays pv, DevArrays x0, DevParams p) {
    __shared__ double red[32];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double f[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < q.n) {
        double fq[kDiagFields], fp[kDiagFields];
#pragma unroll
        for (int k = 0; k < kDiagFields; ++k) fq[k] = fp[k] = 0.0;
        diag_terms(q, p, i, 0.0, fq);
        diag_terms(pv, p, i, 0.0, fp);
        const double eq = fq[0] + fq[2] + fq[3], ep = fp[0] + fp[2] + fp[3];
        const int64_t np = q.n_pad;
        double dg = 0.0, dx2 = 0.0, d02 = 0.0;
        const float4 g = q.grav ? q.grav[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float gc[3] = {g.x, g.y, g.z};
        for (int c = 0; c < 3; ++c) {
            const double xq = q.pos64[c * np + i], xp = pv.pos64[c * np + i], xs = x0.pos64[c * np + i];
            dg += static_cast<double>(gc[c]) * (xp - xq);
            dx2 += (xp - xq) * (xp - xq);
            d02 += (xq - xs) * (xq - xs);
        }
        f[0] = ep - eq - static_cast<double>(q.posm[i].w) * dg;
        f[1] = dx2;
        f[2] = d02;
        f[3] = eq;
        f[4] = fp[0] - fq[0];
        f[5] = fp[2] - fq[2];
        f[6] = fp[3] - fq[3];
        f[7] = -static_cast<double>(q.posm[i].w) * dg;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double sum = block_sum(f[k], red);
        if (threadIdx.x == 0) q.diag[static_cast<int64_t>(blockIdx.x) * kDiagFields + k] = sum;
    }
}

// Energy adjustment (gsph_energy_adjust): block partials of m, m v, 1/2 m v^2 and the shear energy ...
__global__ void __launch_bounds__(kDiagThreads) k_energy_parts(DevArrays a, DevParams p) {
    __shared__ double red[32];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double f[kDiagFields];
#pragma unroll
    for (int k = 0; k < kDiagFields; ++k) f[k] = 0.0;
    if (i < a.n) diag_terms(a, p, i, 0.0, f);
    const double g[6] = {f[10], f[4], f[5], f[6], f[0], f[3]};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double sum = block_sum(g[k], red);
        if (threadIdx.x == 0) a.diag[static_cast<int64_t>(blockIdx.x) * kDiagFields + k] = sum;
    }
}

// ... then, from the totals: peculiar velocities scaled about the centre-of-mass velocity by
// lambda_v = sqrt(1 + d_kin / E_kin,com) and the deviatoric stress by lambda_s = sqrt(1 + d_shear / E_shear)
// (each factor limited to [0.9, 1.1]; 1 when its energy is zero), then the plasticity limiter of the
// integrator. Momentum is unchanged; the kinetic energy changes by d_kin exactly, the shear energy by
// d_shear unless the limiter clips a particle.
__global__ void k_energy_adjust(DevArrays a, DevParams p, const double* __restrict__ tot, double d_kin,
                                double d_shear) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double M = tot[0];
    const double vc[3] = {M > 0 ? tot[1] / M : 0.0, M > 0 ? tot[2] / M : 0.0, M > 0 ? tot[3] / M : 0.0};
    const double ekc = tot[4] - 0.5 * M * (vc[0] * vc[0] + vc[1] * vc[1] + vc[2] * vc[2]);
    auto factor = [](double e, double d) {
        if (!(e > 0.0)) return 1.0;
        return fmin(1.1, fmax(0.9, sqrt(fmax(0.0, 1.0 + d / e))));
    };
    const double lv = factor(ekc, d_kin), ls = factor(tot[5], d_shear);
    float4 vr = a.velrho[i];
    vr.x = static_cast<float>(vc[0] + lv * (static_cast<double>(vr.x) - vc[0]));
    vr.y = static_cast<float>(vc[1] + lv * (static_cast<double>(vr.y) - vc[1]));
    vr.z = static_cast<float>(vc[2] + lv * (static_cast<double>(vr.z) - vc[2]));
    a.velrho[i] = vr;
    if (has(p, GSPH_SPH) && has(p, GSPH_SOLIDS) && ls != 1.0) {
        const float f = static_cast<float>(ls);
        float4 sa = a.sA[i], sb = a.sB[i];
        sa.x *= f; sa.y *= f; sa.z *= f; sa.w *= f;
        sb.x *= f; sb.y *= f;
        if (has(p, GSPH_PLASTICITY_MC))
            plasticity(sa, sb, p.tanfr * murnaghan(p, vr.w) + p.cohesion);
        else if (has(p, GSPH_PLASTICITY_MIESE))
            plasticity(sa, sb, p.Y);
        a.sA[i] = sa;
        a.sB[i] = sb;
    }
}

__global__ void k_diag_reduce(DevArrays a, int nblocks, double* out) {
    const int k = threadIdx.x;
    if (k >= kDiagFields) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += a.diag[static_cast<int64_t>(b) * kDiagFields + k];
    out[k] = s;
}

// ---- host layout <-> device layout ------------------------------------------------------------
// attribute ids follow the bit order of GSPH_POS ... GSPH_MAXVSIG
// `ext` maps the device slot i to the caller's particle index e (identity when null); the staging
// buffer holds the attribute in the caller's order and layout (k components per particle)
__global__ void k_pack(DevArrays a, int attr, const float* __restrict__ src, const int* __restrict__ ext) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t np = a.n_pad;
    const int64_t e = ext ? ext[i] : i;
    switch (attr) {
        case 0: {  // POS
            const float x = src[3 * e], y = src[3 * e + 1], z = src[3 * e + 2];
            a.pos64[i] = x; a.pos64[np + i] = y; a.pos64[2 * np + i] = z;
            float4 q = a.posm[i];
            q.x = x; q.y = y; q.z = z;
            a.posm[i] = q;
            break;
        }
        case 1: { float4 q = a.posm[i]; q.w = src[e]; a.posm[i] = q; break; }  // MASS
        case 2: { float4 q = a.velrho[i]; q.x = src[3 * e]; q.y = src[3 * e + 1]; q.z = src[3 * e + 2]; a.velrho[i] = q; break; }
        case 3: { float4 q = a.acc[i]; q.x = src[3 * e]; q.y = src[3 * e + 1]; q.z = src[3 * e + 2]; a.acc[i] = q; break; }
        case 4: a.balsara[i] = src[e]; break;
        case 5: a.xvel[i] = make_float4(src[3 * e], src[3 * e + 1], src[3 * e + 2], 0.0f); break;
        case 6: { float4 q = a.velrho[i]; q.w = src[e]; a.velrho[i] = q; break; }
        case 7: a.rhodot[i] = src[e]; break;
        case 8:
        case 9: {  // DSTRESS / DSTRESS_DT: 9 row-major values, symmetrised
            const float* m = src + 9 * e;
            const float4 A = make_float4(m[0], m[4], m[8], 0.5f * (m[1] + m[3]));
            const float4 B = make_float4(0.5f * (m[2] + m[6]), 0.5f * (m[5] + m[7]), 0.0f, 0.0f);
            if (attr == 8) { a.sA[i] = A; a.sB[i] = B; }
            else { a.dA[i] = A; a.dB[i] = B; }
            break;
        }
        case 10: { float4 q = a.acc[i]; q.w = src[e]; a.acc[i] = q; break; }
        default: break;
    }
}

__global__ void k_unpack(DevArrays a, int attr, float* __restrict__ dst, const int* __restrict__ ext) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t e = ext ? ext[i] : i;
    switch (attr) {
        case 0: { const float4 q = a.posm[i]; dst[3 * e] = q.x; dst[3 * e + 1] = q.y; dst[3 * e + 2] = q.z; break; }
        case 1: dst[e] = a.posm[i].w; break;
        case 2: { const float4 q = a.velrho[i]; dst[3 * e] = q.x; dst[3 * e + 1] = q.y; dst[3 * e + 2] = q.z; break; }
        case 3: { const float4 q = a.acc[i]; dst[3 * e] = q.x; dst[3 * e + 1] = q.y; dst[3 * e + 2] = q.z; break; }
        case 4: dst[e] = a.balsara[i]; break;
        case 5: { const float4 q = a.xvel[i]; dst[3 * e] = q.x; dst[3 * e + 1] = q.y; dst[3 * e + 2] = q.z; break; }
        case 6: dst[e] = a.velrho[i].w; break;
        case 7: dst[e] = a.rhodot[i]; break;
        case 8:
        case 9: {
            const float4 A = (attr == 8) ? a.sA[i] : a.dA[i];
            const float4 B = (attr == 8) ? a.sB[i] : a.dB[i];
            float* m = dst + 9 * e;
            m[0] = A.x; m[1] = A.w; m[2] = B.x;
            m[3] = A.w; m[4] = A.y; m[5] = B.y;
            m[6] = B.x; m[7] = B.y; m[8] = A.z;
            break;
        }
        case 10: dst[e] = a.acc[i].w; break;
        default: break;
    }
}

__global__ void k_pack_pos64(DevArrays a, const double* __restrict__ src, const int* __restrict__ ext) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t np = a.n_pad;
    const int64_t e = ext ? ext[i] : i;
    const double x = src[3 * e], y = src[3 * e + 1], z = src[3 * e + 2];
    a.pos64[i] = x; a.pos64[np + i] = y; a.pos64[2 * np + i] = z;
    float4 q = a.posm[i];
    q.x = static_cast<float>(x); q.y = static_cast<float>(y); q.z = static_cast<float>(z);
    a.posm[i] = q;
}

__global__ void k_unpack_pos64(DevArrays a, double* __restrict__ dst, const int* __restrict__ ext) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t np = a.n_pad;
    const int64_t e = ext ? ext[i] : i;
    dst[3 * e] = a.pos64[i]; dst[3 * e + 1] = a.pos64[np + i]; dst[3 * e + 2] = a.pos64[2 * np + i];
}

// inert padding: zero mass, far away (never a neighbour, no gravitational pull), unit density
__global__ void k_init_padding(DevArrays a) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n_pad) return;
    const float far = 1e18f;
    if (i >= a.n) {
        a.posm[i] = make_float4(far, far, far, 0.0f);
        a.velrho[i] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        a.pos64[i] = far; a.pos64[a.n_pad + i] = far; a.pos64[2 * a.n_pad + i] = far;
    } else {
        a.posm[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        a.velrho[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        a.pos64[i] = 0.0; a.pos64[a.n_pad + i] = 0.0; a.pos64[2 * a.n_pad + i] = 0.0;
    }
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    a.acc[i] = z; a.xvel[i] = z; a.sA[i] = z; a.sB[i] = z; a.dA[i] = z; a.dB[i] = z; a.jA[i] = z; a.jB[i] = z;
    a.rhodot[i] = 0.0f;
    a.balsara[i] = 0.0f;
}

// scan for NaN/Inf in the state (host-requested check); sets status bit 2
__global__ void k_check_finite(DevArrays a) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float4 q = a.posm[i], v = a.velrho[i];
    const bool bad = !(isfinite(q.x) && isfinite(q.y) && isfinite(q.z) && isfinite(q.w) && isfinite(v.x) &&
                       isfinite(v.y) && isfinite(v.z) && isfinite(v.w));
    if (bad) atomicOr(a.status, 2);
}

}  // namespace

cudaError_t launch_leapfrog(const DevArrays& a, const DevParams& p, int not_first_step, cudaStream_t s) {
    const unsigned nb = blocks_for(a.n, 256);
    if (!has(p, GSPH_VARIABLE_TIMESTEP)) {
        k_leapfrog_fixed<<<nb, 256, 0, s>>>(a, p, p.fixed_dt * (not_first_step ? 1.0f : 0.5f));
        return cudaGetLastError();
    }
    if (not_first_step) k_dt_criteria<<<nb, 256, 0, s>>>(a, p);
    else k_dt_first<<<1, 32, 0, s>>>(a, p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_leapfrog_variable<<<nb, 256, 0, s>>>(a, p);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_dt_commit<<<1, 32, 0, s>>>(a, p);
    return cudaGetLastError();
}

int leapfrog_kernel_count(const DevParams& p) { return has(p, GSPH_VARIABLE_TIMESTEP) ? 3 : 1; }

size_t diag_scratch_doubles(int64_t n) { return static_cast<size_t>(blocks_for(n, kDiagThreads)) * kDiagFields + kDiagFields; }

cudaError_t launch_diagnostics(const DevArrays& a, const DevParams& p, double half_kick, double* out_dev, cudaStream_t s) {
    const unsigned nb = blocks_for(a.n, kDiagThreads);
    k_diag<<<nb, kDiagThreads, 0, s>>>(a, p, half_kick);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_diag_reduce<<<1, 32, 0, s>>>(a, static_cast<int>(nb), out_dev);
    return cudaGetLastError();
}

cudaError_t launch_diagnostics_fast(const DevArrays& a, const DevParams& p, double half_kick, double* out_dev,
                                    cudaStream_t s) {
    const unsigned nb = blocks_for(a.n, kDiagThreads);
    k_diag_fast<<<nb, kDiagThreads, 0, s>>>(a, p, half_kick);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_diag_reduce<<<1, 32, 0, s>>>(a, static_cast<int>(nb), out_dev);
    return cudaGetLastError();
}

cudaError_t launch_state_compare(const DevArrays& q, const DevArrays& p_state, const DevArrays& x0, const DevParams& p,
                                 double* scratch, double* out_dev, cudaStream_t s) {
    const unsigned nb = blocks_for(q.n, kDiagThreads);
    DevArrays qq = q;
    qq.diag = scratch;
    k_state_compare<<<nb, kDiagThreads, 0, s>>>(qq, p_state, x0, p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_diag_reduce<<<1, 32, 0, s>>>(qq, static_cast<int>(nb), out_dev);
    return cudaGetLastError();
}

cudaError_t launch_energy_adjust(const DevArrays& a, const DevParams& p, double d_kin, double d_shear, double* tot_dev,
                                 cudaStream_t s) {
    const unsigned nb = blocks_for(a.n, kDiagThreads);
    k_energy_parts<<<nb, kDiagThreads, 0, s>>>(a, p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_diag_reduce<<<1, 32, 0, s>>>(a, static_cast<int>(nb), tot_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_energy_adjust<<<nb, kDiagThreads, 0, s>>>(a, p, tot_dev, d_kin, d_shear);
    return cudaGetLastError();
}

cudaError_t launch_pack(const DevArrays& a, int attr, const float* src_dev, const int* ext, cudaStream_t s) {
    k_pack<<<blocks_for(a.n, 256), 256, 0, s>>>(a, attr, src_dev, ext);
    return cudaGetLastError();
}
cudaError_t launch_unpack(const DevArrays& a, int attr, float* dst_dev, const int* ext, cudaStream_t s) {
    k_unpack<<<blocks_for(a.n, 256), 256, 0, s>>>(a, attr, dst_dev, ext);
    return cudaGetLastError();
}
cudaError_t launch_pack_pos64(const DevArrays& a, const double* src_dev, const int* ext, cudaStream_t s) {
    k_pack_pos64<<<blocks_for(a.n, 256), 256, 0, s>>>(a, src_dev, ext);
    return cudaGetLastError();
}
cudaError_t launch_unpack_pos64(const DevArrays& a, double* dst_dev, const int* ext, cudaStream_t s) {
    k_unpack_pos64<<<blocks_for(a.n, 256), 256, 0, s>>>(a, dst_dev, ext);
    return cudaGetLastError();
}
cudaError_t launch_init_padding(const DevArrays& a, cudaStream_t s) {
    k_init_padding<<<blocks_for(a.n_pad, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_check_finite(const DevArrays& a, cudaStream_t s) {
    k_check_finite<<<blocks_for(a.n, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace gsph
