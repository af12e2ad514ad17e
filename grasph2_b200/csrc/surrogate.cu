// surrogate.cu -- the per-particle kernels of the learned K-substep surrogate: neighbour-moment
// features of the current state (the MLP's 32 inputs) and the application of a proposal (the
// constant-derivative leapfrog extrapolation over K substeps plus the MLP's correction).
#include "surrogate.cuh"
#include "sph.cuh"

namespace gsph {

namespace {

constexpr int kF = 32;   // features per particle
constexpr int kO = 13;   // outputs per particle

// Features of particle i (one 128-thread CTA per particle group, its near chunks through shared memory):
//   0-2   v                                   3     rho / rho0 - 1
//   4-9   S (xx yy zz xy xz yz)               10    sum m_j W_ij / rho0
//   11-13 sum m_j W_ij d_ij / (h rho0)        14-16 sum m_j W_ij u_ij / rho0
//   17-22 sum m_j W_ij d_ij (x) d_ij / (h^2 rho0), symmetric (xx yy zz xy xz yz)
//   23-31 sum m_j W_ij u_ij (x) d_ij / (h rho0), row-major
// with d_ij = x_j - x_i, u_ij = v_j - v_i, over 0 < r_ij <= h; then (f - mu) / sigma when given.
__global__ void __launch_bounds__(kGroup) k_features(DevArrays a, DevParams p, const int* __restrict__ list,
                                                     const int* __restrict__ count, int64_t nchunks,
                                                     const int* __restrict__ ext, const float* __restrict__ mu,
                                                     const float* __restrict__ sig, float* __restrict__ feat) {
    __shared__ float4 P[kChunk], V[kChunk];
    const int g = blockIdx.x;
    const int64_t i = static_cast<int64_t>(g) * kGroup + threadIdx.x;
    const bool valid = i < a.n;
    const float4 xi = a.posm[valid ? i : 0];
    const float4 vi = a.velrho[valid ? i : 0];
    float s0 = 0.0f, d1[3] = {0, 0, 0}, u1[3] = {0, 0, 0}, dd[6] = {0, 0, 0, 0, 0, 0}, ud[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int nc = count[g];
    const uint32_t span = __float_as_uint(p.H2);
    for (int k = 0; k < nc; ++k) {
        const int64_t c = list[static_cast<int64_t>(g) * nchunks + k];
        __syncthreads();
        if (threadIdx.x < kChunk) {
            P[threadIdx.x] = a.posm[c * kChunk + threadIdx.x];
            V[threadIdx.x] = a.velrho[c * kChunk + threadIdx.x];
        }
        __syncthreads();
        for (int j = 0; j < kChunk; ++j) {
            const float4 q = P[j];
            const float dx = q.x - xi.x, dy = q.y - xi.y, dz = q.z - xi.z;
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if ((__float_as_uint(r2) - 1u) >= span) continue;  // 0 < r^2 <= h^2
            const float r = r2 * rsqrtf(r2);
            const float w = q.w * p.w_pref * w_poly(r * p.inv_h);
            const float ex = dx * p.inv_h, ey = dy * p.inv_h, ez = dz * p.inv_h;
            const float4 vq = V[j];
            const float ux = vq.x - vi.x, uy = vq.y - vi.y, uz = vq.z - vi.z;
            s0 += w;
            d1[0] = fmaf(w, ex, d1[0]); d1[1] = fmaf(w, ey, d1[1]); d1[2] = fmaf(w, ez, d1[2]);
            u1[0] = fmaf(w, ux, u1[0]); u1[1] = fmaf(w, uy, u1[1]); u1[2] = fmaf(w, uz, u1[2]);
            dd[0] = fmaf(w, ex * ex, dd[0]); dd[1] = fmaf(w, ey * ey, dd[1]); dd[2] = fmaf(w, ez * ez, dd[2]);
            dd[3] = fmaf(w, ex * ey, dd[3]); dd[4] = fmaf(w, ex * ez, dd[4]); dd[5] = fmaf(w, ey * ez, dd[5]);
            const float e3[3] = {ex, ey, ez}, u3[3] = {ux, uy, uz};
#pragma unroll
            for (int r0 = 0; r0 < 3; ++r0)
#pragma unroll
                for (int c0 = 0; c0 < 3; ++c0) ud[3 * r0 + c0] = fmaf(w, u3[r0] * e3[c0], ud[3 * r0 + c0]);
        }
    }
    if (!valid) return;
    const float ir = 1.0f / p.rho0;
    const float4 sa = a.sA[i], sb = a.sB[i];
    float f[kF] = {vi.x, vi.y, vi.z, vi.w * ir - 1.0f, sa.x, sa.y, sa.z, sa.w, sb.x, sb.y, s0 * ir,
                   d1[0] * ir, d1[1] * ir, d1[2] * ir, u1[0] * ir, u1[1] * ir, u1[2] * ir};
#pragma unroll
    for (int k = 0; k < 6; ++k) f[17 + k] = dd[k] * ir;
#pragma unroll
    for (int k = 0; k < 9; ++k) f[23 + k] = ud[k] * ir;
    const int64_t e = ext ? ext[i] : i;
    float* out = feat + e * kF;
#pragma unroll
    for (int k = 0; k < kF; ++k) out[k] = mu ? (f[k] - mu[k]) / sig[k] : f[k];
}

// Proposal over K substeps of the fixed-step leapfrog with the derivatives of the current state held
// constant (v is the half-step velocity; x_K = x + K dt v + K(K+1)/2 dt^2 a, v_K = v + K dt a,
// S_K = S + K dt dS/dt), plus the MLP's correction delta (caller order, output mu + sigma * delta):
// 0-2 position, 3-5 velocity, 6 density, 7-12 S (xx yy zz xy xz yz); then the plasticity limiter.
__global__ void k_apply(DevArrays a, DevParams p, const int* __restrict__ ext, const float* __restrict__ delta,
                        const float* __restrict__ omu, const float* __restrict__ osig, int K) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t e = ext ? ext[i] : i;
    float d[kO];
#pragma unroll
    for (int k = 0; k < kO; ++k) d[k] = delta ? omu[k] + osig[k] * delta[e * kO + k] : 0.0f;
    const double dt = p.fixed_dt, T = K * dt, c2 = 0.5 * K * (K + 1) * dt * dt;
    float4 vr = a.velrho[i];
    const float4 ac = a.acc[i];
    const int64_t np = a.n_pad;
    double x = a.pos64[i], y = a.pos64[np + i], z = a.pos64[2 * np + i];
    x += T * vr.x + c2 * ac.x + d[0];
    y += T * vr.y + c2 * ac.y + d[1];
    z += T * vr.z + c2 * ac.z + d[2];
    vr.x = static_cast<float>(vr.x + T * ac.x + d[3]);
    vr.y = static_cast<float>(vr.y + T * ac.y + d[4]);
    vr.z = static_cast<float>(vr.z + T * ac.z + d[5]);
    if (has(p, GSPH_SPH)) {
        vr.w = fmaxf(0.0f, static_cast<float>(vr.w + T * a.rhodot[i] + d[6]));
        if (has(p, GSPH_SOLIDS)) {
            float4 sa = a.sA[i], sb = a.sB[i];
            const float4 da = a.dA[i], db = a.dB[i];
            sa.x = static_cast<float>(sa.x + T * da.x + d[7]);
            sa.y = static_cast<float>(sa.y + T * da.y + d[8]);
            sa.z = static_cast<float>(sa.z + T * da.z + d[9]);
            sa.w = static_cast<float>(sa.w + T * da.w + d[10]);
            sb.x = static_cast<float>(sb.x + T * db.x + d[11]);
            sb.y = static_cast<float>(sb.y + T * db.y + d[12]);
            if (has(p, GSPH_PLASTICITY_MC)) plasticity(sa, sb, p.tanfr * murnaghan(p, vr.w) + p.cohesion);
            else if (has(p, GSPH_PLASTICITY_MIESE)) plasticity(sa, sb, p.Y);
            a.sA[i] = sa;
            a.sB[i] = sb;
        }
    }
    a.pos64[i] = x;
    a.pos64[np + i] = y;
    a.pos64[2 * np + i] = z;
    a.posm[i] = make_float4(static_cast<float>(x), static_cast<float>(y), static_cast<float>(z), a.posm[i].w);
    a.velrho[i] = vr;
}

inline unsigned blocks_for(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

cudaError_t launch_features(const DevArrays& a, const DevParams& p, const SpatialArrays& sp, const float* mu,
                            const float* sig, float* feat, cudaStream_t s) {
    k_features<<<static_cast<unsigned>(a.n_pad / kGroup), kGroup, 0, s>>>(a, p, sp.list, sp.count, a.n_pad / kChunk,
                                                                         sp.ext_of_int, mu, sig, feat);
    return cudaGetLastError();
}

cudaError_t launch_apply(const DevArrays& a, const DevParams& p, const int* ext, const float* delta, const float* omu,
                         const float* osig, int K, cudaStream_t s) {
    k_apply<<<blocks_for(a.n, 256), 256, 0, s>>>(a, p, ext, delta, omu, osig, K);
    return cudaGetLastError();
}

}  // namespace gsph
