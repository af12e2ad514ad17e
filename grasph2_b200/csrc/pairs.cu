// pairs.cu -- the all-pairs kernels of computeDerivatives (src/computeDerivatives.h:52-328).
//
//   k_density        calcDensity            (:52-91)    rho_i = sum_{0<r<=H} m_j W(r_ij)
//   k_pairs<VGRAD>   calcBalsaraDensityDTDStressDT (:96-162) strain/rotation rate, div v, curl
//   k_pairs<ACC>     calcAcceleration       (:167-313)  gravity + stress + AV (+XSPH, art. stress)
//   k_pairs<FUSED>   both in one pass, used whenever the acceleration does not need the Balsara
//                    values of the same step (the switch off): one N^2 sweep instead of two
//   k_gravity<I>     calcAcceleration with ENABLE_SPH off: register-blocked pure gravity
//   *_finish         sum the j-segment partials in a fixed order, then the per-particle epilogue
//                    (do_after of each job): density floor, Jaumann stress rate, drho/dt,
//                    Balsara switch, environment acceleration
//
// Arithmetic is FP32. GSPH_ACCUM_COMPENSATED accumulates each j-tile in FP32, folds the tile
// partial into a (sum, error) pair with a two-sum, and combines the j-segments in FP64.
#include <algorithm>
#include <cfloat>

#include "pairs.cuh"
#include "sph.cuh"

namespace gsph {

namespace {

// ================================================================================================
// density
// ================================================================================================
// Where the partial sums of particle i live: j-segments [seg][field][n_pad] (all-pairs kernels) or
// work items [w][field][kGroup] (culled kernels); KK = fields per slot (2K when compensated).
struct PartView {
    const float* part;
    int64_t n_pad;
    int nseg;
    const int* item_start;  // non-null: item layout
    int KK;
    bool err;               // compensation terms stored after the K sums (all-pairs segments, compensated)
    __device__ __forceinline__ void range(int64_t i, int& b, int& e) const {
        if (item_start) {
            const int64_t g = i / kGroup;
            b = item_start[g];
            e = item_start[g + 1];
        } else {
            b = 0;
            e = nseg;
        }
    }
    __device__ __forceinline__ float at(int slot, int o, int64_t i) const {
        if (item_start) return part[(static_cast<int64_t>(slot) * KK + o) * kGroup + (i % kGroup)];
        return part[(static_cast<int64_t>(slot) * KK + o) * n_pad + i];
    }
};

// one tile of the density sum: rho += m_j W~(q) over 0 < r^2 <= H^2 (self term excluded), the
// spline prefactor applied by the finish kernel
__device__ __forceinline__ float density_tile(const float4* __restrict__ J, int nj, float4 pi, uint32_t span,
                                              float inv_h) {
    float rho = 0.0f;
#pragma unroll 8
    for (int j = 0; j < nj; ++j) {
        const float4 q = J[j];
        const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        if (in_open_closed(r2, 0u, span)) {  // calcDensity: r2 <= H2 && r2 > 0 (computeDerivatives.h:72)
            const float r = r2 * rsqrtf(r2);
            rho = fmaf(q.w, w_poly(r * inv_h), rho);
        }
    }
    return rho;
}

// all-pairs density sum: blockIdx.x = i-block, blockIdx.y = j-segment
template <bool COMP>
__global__ void __launch_bounds__(256) k_density(const float4* __restrict__ posm, float* __restrict__ part,
                                                  int64_t n_pad, int jt, int nseg, DevParams p, int* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    JTilePipe<1> pipe;
    pipe.buf = reinterpret_cast<float4*>(smem_raw);
    pipe.bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * jt * sizeof(float4));
    pipe.src[0] = posm;
    pipe.jt = jt;
    pipe.status = status;
    segment_tiles(n_pad / jt, blockIdx.y, nseg, pipe.t_begin, pipe.t_end);
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const float4 pi = posm[i];
    const uint32_t span = __float_as_uint(p.H2);
    float rho_s = 0.0f, rho_c = 0.0f;
    pipe.start();
    pipe.run([&](const float4* J) {
        const float t = density_tile(J, jt, pi, span, p.inv_h);
        if (COMP) fold(rho_s, rho_c, t);
        else rho_s += t;
    });
    const int64_t seg = blockIdx.y;
    part[(seg * (COMP ? 2 : 1)) * n_pad + i] = rho_s;
    if (COMP) part[(seg * 2 + 1) * n_pad + i] = rho_c;
}

// culled density sum over the near-chunk work items (persistent grid); with LISTS every lane also
// records the indices of its neighbours in this item (for the SPH passes of the same step)
template <bool COMP, bool LISTS>
__global__ void __launch_bounds__(kGroup, 12) k_density_items(const float4* __restrict__ posm, DevParams p, CullView cv,
                                                          int* status) {
    constexpr int SJ = kStageChunks * kChunk;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ItemPipe<1> pipe;
    pipe.buf = reinterpret_cast<float4*>(smem_raw);
    pipe.bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * SJ * sizeof(float4));
    pipe.src[0] = posm;
    pipe.status = status;
    pipe.init();
    const uint32_t span = __float_as_uint(p.H2);
    const int total = cv.items();
    __shared__ float4 wbox[kGroup / 32][2];  // each warp's bounding box for the current item
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        int g, c0, c1;
        cv.item(w, g, c0, c1);
        const float4 pi = posm[static_cast<int64_t>(g) * kGroup + threadIdx.x];
        float rho_s = 0.0f, rho_c = 0.0f;
        int cnt = 0;
        // the warp's bounding box: a chunk of the group's list that lies farther than h (1 + kMargin)
        // from it (the list's own conservative bound) holds no neighbour of the warp's 32 particles, and
        // the warp skips its tests (same sums, same lists; padding lanes only widen the box)
        if (LISTS) {
            float wlo[3] = {pi.x, pi.y, pi.z}, whi[3] = {pi.x, pi.y, pi.z};
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    wlo[c] = fminf(wlo[c], __shfl_xor_sync(0xffffffffu, wlo[c], o));
                    whi[c] = fmaxf(whi[c], __shfl_xor_sync(0xffffffffu, whi[c], o));
                }
            __syncwarp();  // the previous item's reads of this warp's box are done
            if ((threadIdx.x & 31) == 0) {
                wbox[threadIdx.x >> 5][0] = make_float4(wlo[0], wlo[1], wlo[2], 0.0f);
                wbox[threadIdx.x >> 5][1] = make_float4(whi[0], whi[1], whi[2], 0.0f);
            }
            __syncwarp();
        }
        int* lst = LISTS ? cv.nb + static_cast<int64_t>(w) * kItemNb * kGroup + threadIdx.x : nullptr;
        const int* chunks = cv.list + static_cast<int64_t>(g) * cv.nchunks + c0;
        int chunk_base = 0;
        if (!pipe.run(chunks, c1 - c0, [&](const float4* J, int nj) {
                float t;
                if (LISTS) {  // the density_tile sum, recording the neighbours as well (same order)
                    t = 0.0f;
                    for (int s0 = 0; s0 < nj; s0 += kChunk) {
                        const int jc = chunks[chunk_base + s0 / kChunk], jb = jc * kChunk;
                        {
                            const float4 l = cv.box_lo[jc], u = cv.box_hi[jc];
                            const float4 wl = wbox[threadIdx.x >> 5][0], wh = wbox[threadIdx.x >> 5][1];
                            const float gx = fmaxf(0.0f, fmaxf(l.x - wh.x, wl.x - u.x)),
                                        gy = fmaxf(0.0f, fmaxf(l.y - wh.y, wl.y - u.y)),
                                        gz = fmaxf(0.0f, fmaxf(l.z - wh.z, wl.z - u.z));
                            const float hm = p.H * (1.0f + kMargin);
                            if (gx * gx + gy * gy + gz * gz > hm * hm) continue;  // warp-uniform
                        }
                        // the chunk's 64 tests into a bit mask without branches, then its set bits in
                        // ascending order (the neighbours, about 2 % of the tests)
                        unsigned m8[8];
#pragma unroll
                        for (int b = 0; b < 8; ++b) {
                            unsigned m = 0;
#pragma unroll
                            for (int u = 0; u < 8; ++u) {
                                const float4 q = J[s0 + b * 8 + u];
                                const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
                                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                                m |= static_cast<unsigned>(in_open_closed(r2, 0u, span)) << u;
                            }
                            m8[b] = m;
                        }
                        uint64_t bits = static_cast<uint64_t>(m8[0] | (m8[1] << 8) | (m8[2] << 16) | (m8[3] << 24)) |
                                        (static_cast<uint64_t>(m8[4] | (m8[5] << 8) | (m8[6] << 16) | (m8[7] << 24)) << 32);
                        while (bits) {
                            const int j = __ffsll(static_cast<long long>(bits)) - 1;
                            bits &= bits - 1;
                            const float4 q = J[s0 + j];
                            const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
                            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                            const float r = r2 * rsqrtf(r2);
                            t = fmaf(q.w, w_poly(r * p.inv_h), t);
                            if (cnt < kItemNb) lst[cnt * kGroup] = jb + j;
                            ++cnt;
                        }
                    }
                    chunk_base += nj / kChunk;
                } else {
                    t = density_tile(J, nj, pi, span, p.inv_h);
                }
                if (COMP) fold(rho_s, rho_c, t);
                else rho_s += t;
            }))
            return;
        float* out = cv.part + static_cast<int64_t>(w) * (COMP ? 2 : 1) * kGroup + threadIdx.x;
        out[0] = rho_s;
        if (COMP) out[kGroup] = rho_c;
        if (LISTS) {
            cv.nbcnt[static_cast<int64_t>(w) * kGroup + threadIdx.x] = min(cnt, kItemNb + 1);
            const int over = __syncthreads_or(cnt > kItemNb);  // the SPH passes read one flag per item
            if (threadIdx.x == 0) cv.nbover[w] = over;
        }
    }
}

// sum the slots, apply the prefactor and the optional floor (computeDerivatives.h:85-88), then
// build the j-record sigma/rho^2 of the new density
template <bool COMP>
__global__ void k_density_finish(DevArrays a, DevParams p, PartView pv) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int b, e;
    pv.range(i, b, e);
    float rho;
    if (COMP) {
        double s = 0.0;
        for (int k = b; k < e; ++k) s += static_cast<double>(pv.at(k, 0, i)) + static_cast<double>(pv.at(k, 1, i));
        rho = static_cast<float>(s * static_cast<double>(p.w_pref));
    } else {
        float s = 0.0f;
        for (int k = b; k < e; ++k) s += pv.at(k, 0, i);
        rho = s * p.w_pref;
    }
    if (has(p, GSPH_DEAL_WITH_NO_PARTNERS) && rho < 0.001f) rho = p.rho0 * 0.01f;
    float4 vr = a.velrho[i];
    vr.w = rho;
    a.velrho[i] = vr;
    float4 jA, jB;
    make_jrecord(p, rho, a.sA[i], a.sB[i], a.balsara[i], jA, jB);
    a.jA[i] = jA;
    a.jB[i] = jB;
    if (a.jrec) {
        float4* r = a.jrec + 4 * i;
        r[0] = a.posm[i]; r[1] = vr; r[2] = jA; r[3] = jB;
    }
}

// j-records from the current density (INTEGRATE_DENSITY: no density pass precedes the pairs)
__global__ void k_prepare(DevArrays a, DevParams p) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float4 vr = a.velrho[i];
    float4 jA, jB;
    make_jrecord(p, vr.w, a.sA[i], a.sB[i], a.balsara[i], jA, jB);
    a.jA[i] = jA;
    a.jB[i] = jB;
    if (a.jrec) {
        float4* r = a.jrec + 4 * i;
        r[0] = a.posm[i]; r[1] = vr; r[2] = jA; r[3] = jB;
    }
}

// ================================================================================================
// SPH pair passes
// ================================================================================================
// The all-pairs body over nj staged j-records (P: posm, V: velrho, JA/JB: sigma/rho^2): gravity when
// GRAV != 0 (computeDerivatives.h:229-235, G applied by the finish kernel), then the SPH terms of
// every neighbour. GRAV: 0 off, 1 softened (eps > 0), 2 unsoftened (eps == 0: self pair gives 0).
template <int PASS, int GRAV, bool SOLIDS>
__device__ __forceinline__ void pair_tile(PairAcc& T, float& maxv, const ISph& I, const float4* __restrict__ P,
                                          const float4* __restrict__ V, const float4* __restrict__ JA,
                                          const float4* __restrict__ JB, int nj, const DevParams& p) {
    constexpr bool DO_A = PASS != PASS_VGRAD;
    const float eps2 = I.eps2;
#pragma unroll 4
    for (int j = 0; j < nj; ++j) {
        const float4 q = P[j];
        const float dx = q.x - I.pi.x, dy = q.y - I.pi.y, dz = q.z - I.pi.z;  // d = x_j - x_i = -r_ij
        const float r2e = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
        if (GRAV != 0) {
            float inv = rsqrtf(r2e);
            if (GRAV == 2) inv = fminf(inv, 1e12f);
            const float s = q.w * inv * (inv * inv);
            T.f[F_GX] = fmaf(dx, s, T.f[F_GX]);
            T.f[F_GY] = fmaf(dy, s, T.f[F_GY]);
            T.f[F_GZ] = fmaf(dz, s, T.f[F_GZ]);
        }
        if (in_open_closed(r2e, I.lo, I.span))  // 0 < r2 <= H2
            sph_neighbour<PASS, SOLIDS>(T, maxv, I, q.w, dx, dy, dz, r2e - eps2, V[j],
                                        DO_A ? JA[j] : make_float4(0, 0, 0, 0), DO_A ? JB[j] : make_float4(0, 0, 0, 0),
                                        p);
    }
}

template <uint32_t MASK, bool COMP>
__device__ __forceinline__ void fold_tile(PairAcc& S, PairAcc& C, const PairAcc& T) {
#pragma unroll
    for (int f = 0; f < F_COUNT; ++f) {
        if (!((MASK >> f) & 1u) || f == F_MAXV) continue;
        if (COMP) fold(S.f[f], C.f[f], T.f[f]);
        else S.f[f] += T.f[f];
    }
}

// store one thread's partial sums: field o at out[o * stride] (sums) and out[(K + o) * stride]
// (compensation terms)
template <uint32_t MASK, bool COMP>
__device__ __forceinline__ void store_partials(float* out, int64_t stride, const PairAcc& S, const PairAcc& C,
                                               float maxv) {
    constexpr int K = popc_c(MASK);
#pragma unroll
    for (int f = 0; f < F_COUNT; ++f) {
        if (!((MASK >> f) & 1u)) continue;
        const int o = field_offset<MASK>(f);
        out[o * stride] = (f == F_MAXV) ? maxv : S.f[f];
        if (COMP) out[(K + o) * stride] = (f == F_MAXV) ? 0.0f : C.f[f];
    }
}

// All-pairs SPH pass: blockIdx.x = i-block, blockIdx.y = j-segment (partials [seg][field][n_pad]).
template <int PASS, int GRAV, bool SOLIDS, bool COMP>
__global__ void __launch_bounds__(256) k_pairs(DevArrays a, DevParams p, int jt, int nseg) {
    constexpr uint32_t MASK = field_mask<PASS, (GRAV != 0), SOLIDS>();
    constexpr int K = popc_c(MASK);
    constexpr int NS = (PASS == PASS_VGRAD) ? 2 : 4;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    JTilePipe<NS> pipe;
    pipe.buf = reinterpret_cast<float4*>(smem_raw);
    pipe.bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * NS * jt * sizeof(float4));
    pipe.src[0] = a.posm;
    pipe.src[1] = a.velrho;
    if constexpr (NS == 4) {
        pipe.src[2] = a.jA;
        pipe.src[3] = a.jB;
    }
    pipe.jt = jt;
    pipe.status = a.status;
    segment_tiles(a.n_pad / jt, blockIdx.y, nseg, pipe.t_begin, pipe.t_end);

    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const ISph I = load_isph<PASS, SOLIDS>(a, p, i, (GRAV == 1) ? p.eps2 : 0.0f);
    PairAcc S, C;
#pragma unroll
    for (int f = 0; f < F_COUNT; ++f) S.f[f] = C.f[f] = 0.0f;
    float maxv = 0.0f;

    pipe.start();
    pipe.run([&](const float4* stage) {
        PairAcc T;
#pragma unroll
        for (int f = 0; f < F_COUNT; ++f) T.f[f] = 0.0f;
        pair_tile<PASS, GRAV, SOLIDS>(T, maxv, I, stage, stage + jt, stage + 2 * jt, stage + 3 * jt, jt, p);
        fold_tile<MASK, COMP>(S, C, T);
    });
    store_partials<MASK, COMP>(a.part + static_cast<int64_t>(blockIdx.y) * (COMP ? 2 * K : K) * a.n_pad + i, a.n_pad,
                               S, C, maxv);
}

// Culled SPH pass (no gravity): a persistent grid walks the work items; item w covers some near
// chunks of one i-group and writes its partials to part[w][field][kGroup]. Phase 1 streams only the
// positions of those chunks through shared memory and lets every lane record the indices of its own
// neighbours (kNbCap per lane, flushed early when a lane's list is nearly full); phase 2 walks the
// per-lane lists and gathers each neighbour's records from L2, so the SPH terms run lane-dense.
constexpr int kNbCap = 64;
template <int PASS, bool SOLIDS, bool COMP>
__global__ void __launch_bounds__(kGroup, 5) k_pairs_items(DevArrays a, DevParams p, CullView cv) {
    constexpr uint32_t MASK = field_mask<PASS, false, SOLIDS>();
    constexpr int K = popc_c(MASK);
    constexpr bool DO_A = PASS != PASS_VGRAD;
    constexpr int SJ = kStageChunks * kChunk;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ItemPipe<1> pipe;
    pipe.buf = reinterpret_cast<float4*>(smem_raw);
    pipe.bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * SJ * sizeof(float4));
    pipe.src[0] = a.posm;
    pipe.status = a.status;
    const int lane = threadIdx.x & 31;
    int* nb = reinterpret_cast<int*>(smem_raw + pipe_smem_bytes(1, SJ)) + (threadIdx.x >> 5) * (kNbCap * 32);
    pipe.init();
    const int total = cv.items();
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        int g, c0, c1;
        cv.item(w, g, c0, c1);
        const int64_t i = static_cast<int64_t>(g) * kGroup + threadIdx.x;
        const ISph I = load_isph<PASS, SOLIDS>(a, p, i, 0.0f);
        PairAcc S, C, T;
#pragma unroll
        for (int f = 0; f < F_COUNT; ++f) S.f[f] = C.f[f] = T.f[f] = 0.0f;
        float maxv = 0.0f;
        // the density pass's neighbour lists of this item, when every lane's list is complete (one flag
        // per item, so no block-wide vote: the warps of a block run through list items independently)
        if (cv.nb && cv.nbover[w] == 0) {
            const int lcnt = cv.nbcnt[static_cast<int64_t>(w) * kGroup + threadIdx.x];
            const int* lst = cv.nb + static_cast<int64_t>(w) * kItemNb * kGroup + threadIdx.x;
            const float4 zero = make_float4(0, 0, 0, 0);
            const int j0 = lcnt > 0 ? lst[0] : 0;
            int jn = lcnt > 1 ? lst[kGroup] : 0;  // the index of neighbour k+1
            const float4* r0 = a.jrec + 4 * static_cast<int64_t>(j0);  // one 64-byte record per neighbour
            float4 qn = __ldg(r0), vn = __ldg(r0 + 1);
            float4 an = DO_A ? __ldg(r0 + 2) : zero, bn = DO_A ? __ldg(r0 + 3) : zero;
            // software pipeline: neighbour k+1's records and neighbour k+2's index in flight during k
            for (int k = 0; k < lcnt; ++k) {
                const float4 q = qn, vj = vn, ja = an, jb = bn;
                if (k + 1 < lcnt) {
                    const float4* r = a.jrec + 4 * static_cast<int64_t>(jn);
                    qn = __ldg(r);
                    vn = __ldg(r + 1);
                    if (DO_A) {
                        an = __ldg(r + 2);
                        bn = __ldg(r + 3);
                    }
                }
                if (k + 2 < lcnt) jn = lst[(k + 2) * kGroup];
                const float dx = q.x - I.pi.x, dy = q.y - I.pi.y, dz = q.z - I.pi.z;
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                sph_neighbour<PASS, SOLIDS>(T, maxv, I, q.w, dx, dy, dz, r2, vj, ja, jb, p);
            }
            fold_tile<MASK, COMP>(S, C, T);
            store_partials<MASK, COMP>(cv.part + static_cast<int64_t>(w) * (COMP ? 2 * K : K) * kGroup + threadIdx.x,
                                       kGroup, S, C, maxv);
            continue;
        }
        int cnt = 0;
        // phase 2 over the lane lists collected so far
        auto drain = [&]() {
            int m = cnt;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
            // software pipeline: the records of neighbour k+1 are in flight while k is computed
            const float4 zero = make_float4(0, 0, 0, 0);
            int jn = cnt > 0 ? nb[lane] : 0;
            const float4* r0 = a.jrec + 4 * static_cast<int64_t>(jn);
            float4 qn = __ldg(r0), vn = __ldg(r0 + 1);
            float4 an = DO_A ? __ldg(r0 + 2) : zero, bn = DO_A ? __ldg(r0 + 3) : zero;
            for (int k = 0; k < m; ++k) {
                const float4 q = qn, vj = vn, ja = an, jb = bn;
                if (k + 1 < cnt) {
                    jn = nb[(k + 1) * 32 + lane];
                    const float4* r = a.jrec + 4 * static_cast<int64_t>(jn);
                    qn = __ldg(r);
                    vn = __ldg(r + 1);
                    if (DO_A) {
                        an = __ldg(r + 2);
                        bn = __ldg(r + 3);
                    }
                }
                if (k < cnt) {
                    const float dx = q.x - I.pi.x, dy = q.y - I.pi.y, dz = q.z - I.pi.z;
                    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                    sph_neighbour<PASS, SOLIDS>(T, maxv, I, q.w, dx, dy, dz, r2, vj, ja, jb, p);
                }
            }
            cnt = 0;
            __syncwarp();
        };
        const int* chunks = cv.list + static_cast<int64_t>(g) * cv.nchunks + c0;
        int chunk_base = 0;  // position in `chunks` of the current stage
        if (!pipe.run(chunks, c1 - c0, [&](const float4* J, int nj) {
                for (int s0 = 0; s0 < nj; s0 += kChunk) {
                    const int jbase = chunks[chunk_base + s0 / kChunk] * kChunk;
                    // 64 independent tests into eight 8-bit masks (no serial chain), then the set bits
                    unsigned m8[8];
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        unsigned m = 0;
#pragma unroll
                        for (int t = 0; t < 8; ++t) {
                            const float4 q = J[s0 + b * 8 + t];
                            const float dx = q.x - I.pi.x, dy = q.y - I.pi.y, dz = q.z - I.pi.z;
                            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                            m |= static_cast<unsigned>(in_open_closed(r2, 0u, I.span)) << t;
                        }
                        m8[b] = m;
                    }
                    unsigned lo = m8[0] | (m8[1] << 8) | (m8[2] << 16) | (m8[3] << 24);
                    unsigned hi = m8[4] | (m8[5] << 8) | (m8[6] << 16) | (m8[7] << 24);
                    while (lo) {
                        nb[cnt * 32 + lane] = jbase + __ffs(lo) - 1;
                        ++cnt;
                        lo &= lo - 1u;
                    }
                    while (hi) {
                        nb[cnt * 32 + lane] = jbase + 32 + __ffs(hi) - 1;
                        ++cnt;
                        hi &= hi - 1u;
                    }
                    // a lane could overflow on the next chunk: process the lists now
                    if (__any_sync(0xffffffffu, cnt > kNbCap - kChunk)) drain();
                }
                chunk_base += nj / kChunk;
            }))
            return;
        drain();
        fold_tile<MASK, COMP>(S, C, T);
        store_partials<MASK, COMP>(cv.part + static_cast<int64_t>(w) * (COMP ? 2 * K : K) * kGroup + threadIdx.x,
                                   kGroup, S, C, maxv);
    }
}


// Sum the slots of one field in a fixed order: FP32 in plain mode, FP64 of (sum + error) in
// compensated mode. The max signal velocity is a max over slots.
template <uint32_t MASK, bool COMP>
__device__ __forceinline__ float seg_sum(const PartView& v, int64_t i, int f) {
    constexpr int K = popc_c(MASK);
    const int o = field_offset<MASK>(f);
    int b, e;
    v.range(i, b, e);
    if (f == F_MAXV) {
        float m = 0.0f;
        for (int k = b; k < e; ++k) m = fmaxf(m, v.at(k, o, i));
        return m;
    }
    if (COMP) {
        double s = 0.0;
        for (int k = b; k < e; ++k) {
            s += static_cast<double>(v.at(k, o, i));
            if (v.err) s += static_cast<double>(v.at(k, K + o, i));
        }
        return static_cast<float>(s);
    }
    float s = 0.0f;
    for (int k = b; k < e; ++k) s += v.at(k, o, i);
    return s;
}

// ---- the FP64 fold of the gravity partials ---------------------------------------------------------
// Both all-pairs gravity kernels leave per-particle partial sums [slot][component][n_pad]: the one-sided
// kernel's j-segments, or the symmetric kernel's G + 1 slots (its row and column sums, each written by
// one task). kFoldT threads fold one particle: thread q sums the slots [q R, (q + 1) R) in FP64 (with the
// error terms of the compensated form), then the runs are added in the order q = 0, 1, 2, 3 -- a fixed
// order, so results are deterministic. Eight particles per warp: for a slot, the eight lanes of a run
// read 32 contiguous bytes.
constexpr int kFoldT = 4;
template <bool COMP>
__device__ __forceinline__ void fold_slots(const float* __restrict__ part, int64_t n_pad, int S, int64_t i, bool valid,
                                           double (&out)[3]) {
    constexpr int K = COMP ? 6 : 3;
    const int lane = threadIdx.x & 31, q = lane >> 3;
    const int R = (S + kFoldT - 1) / kFoldT;
    const int k0 = min(S, q * R), k1 = min(S, k0 + R);
    double s[3] = {0.0, 0.0, 0.0};
    if (valid) {
#pragma unroll 4
        for (int k = k0; k < k1; ++k) {
            const float* p = part + static_cast<int64_t>(k) * K * n_pad + i;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                s[c] += static_cast<double>(__ldg(p + c * n_pad));
                if (COMP) s[c] += static_cast<double>(__ldg(p + (3 + c) * n_pad));
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {  // runs 0 + 1 + 2 + 3, in this order, on the lanes of run 0
        double t = s[c];
        t += __shfl_down_sync(0xffffffffu, s[c], 8);
        t += __shfl_down_sync(0xffffffffu, s[c], 16);
        t += __shfl_down_sync(0xffffffffu, s[c], 24);
        out[c] = t;
    }
}
__device__ __forceinline__ int64_t fold_particle() {
    return (static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u)) / kFoldT + (threadIdx.x & 7);
}

// the culled path: the fold of the gravity partials into gfold[3][n_pad], on the gravity kernel's stream
template <bool COMP>
__global__ void __launch_bounds__(256) k_gravity_fold(const float* __restrict__ part, int64_t n, int64_t n_pad, int S,
                                                      double* __restrict__ gfold) {
    const int64_t i = fold_particle();
    double t[3];
    fold_slots<COMP>(part, n_pad, S, i, i < n, t);
    if ((threadIdx.x & 31) < 8 && i < n)
        for (int c = 0; c < 3; ++c) gfold[c * n_pad + i] = t[c];
}

template <int PASS, bool GRAV, bool SOLIDS, bool COMP>
__global__ void k_pairs_finish(DevArrays a, DevParams p, PartView pv, GravSum gsum) {
    constexpr uint32_t MASK = field_mask<PASS, GRAV, SOLIDS>();
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (PASS != PASS_VGRAD && has(p, GSPH_VARIABLE_TIMESTEP) && i == 0)
        a.dt_state[1] = p.max_dt;  // nextTS reset of calcAcceleration::do_after (:306-309)
    if (i >= a.n) return;
    float g[3] = {0.0f, 0.0f, 0.0f};
    bool grav = false;
    if (PASS != PASS_VGRAD) {
        if (GRAV) {
            g[0] = seg_sum<MASK, COMP>(pv, i, F_GX);
            g[1] = seg_sum<MASK, COMP>(pv, i, F_GY);
            g[2] = seg_sum<MASK, COMP>(pv, i, F_GZ);
            grav = true;
        } else if (gsum.nseg > 0 || gsum.sym_G > 0) {  // folded on the gravity stream (k_gravity_fold)
            for (int c = 0; c < 3; ++c) g[c] = static_cast<float>(a.gfold[c * a.n_pad + i]);
            grav = true;
        }
    }
    sph_finish<PASS, SOLIDS>(a, p, i, [&](int f) { return seg_sum<MASK, COMP>(pv, i, f); }, grav, g);
}

// ================================================================================================
// pure gravity (ENABLE_SPH off): I i-particles per thread share every j read from shared memory
// ================================================================================================
// Paired FP32 (PTX ISA 8.6, sm_100+): one add/sub/mul/fma.rn.f32x2 instruction performs the same
// IEEE single-precision operation on two lanes of a 64-bit register pair, so two i-particles advance
// per issued instruction with bit-identical results to the scalar form.
__device__ __forceinline__ uint64_t u64_of(float2 v) { return *reinterpret_cast<uint64_t*>(&v); }
__device__ __forceinline__ float2 f2_of(uint64_t v) { return *reinterpret_cast<float2*>(&v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(u64_of(a)), "l"(u64_of(b)), "l"(u64_of(c)));
    return f2_of(d);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(d);
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(d);
}

// I (even) i-particles per thread in I/2 register pairs; same arithmetic order as k_gravity
template <int I, int GRAV, bool COMP>
__global__ void __launch_bounds__(128) k_gravity_x2(const float4* __restrict__ posm, float* __restrict__ part,
                                                     int64_t n_pad, int jt, int nseg, float eps2, int* status) {
    constexpr int P = I / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    JTilePipe<1> pipe;
    pipe.buf = reinterpret_cast<float4*>(smem_raw);
    pipe.bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * jt * sizeof(float4));
    pipe.src[0] = posm;
    pipe.jt = jt;
    pipe.status = status;
    segment_tiles(n_pad / jt, blockIdx.y, nseg, pipe.t_begin, pipe.t_end);

    const int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x * I + threadIdx.x;
    float2 X[P], Y[P], Z[P], AX[P], AY[P], AZ[P], CX[P], CY[P], CZ[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
        const float4 a = posm[base + static_cast<int64_t>(2 * k) * blockDim.x];
        const float4 b = posm[base + static_cast<int64_t>(2 * k + 1) * blockDim.x];
        X[k] = make_float2(a.x, b.x); Y[k] = make_float2(a.y, b.y); Z[k] = make_float2(a.z, b.z);
        AX[k] = AY[k] = AZ[k] = make_float2(0.0f, 0.0f);
        CX[k] = CY[k] = CZ[k] = make_float2(0.0f, 0.0f);
    }
    const float2 E2 = make_float2(eps2, eps2);

    pipe.start();
    pipe.run([&](const float4* J) {
        float2 TX[P], TY[P], TZ[P];
#pragma unroll
        for (int k = 0; k < P; ++k) TX[k] = TY[k] = TZ[k] = make_float2(0.0f, 0.0f);
#pragma unroll 4
        for (int j = 0; j < jt; ++j) {
            const float4 q = J[j];
            const float2 qx = make_float2(q.x, q.x), qy = make_float2(q.y, q.y), qz = make_float2(q.z, q.z),
                         qm = make_float2(q.w, q.w);
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const float2 dx = sub2(qx, X[k]), dy = sub2(qy, Y[k]), dz = sub2(qz, Z[k]);
                const float2 r2 = fma2(dz, dz, fma2(dy, dy, fma2(dx, dx, E2)));
                float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                if (GRAV == 2) inv = make_float2(fminf(inv.x, 1e12f), fminf(inv.y, 1e12f));
                const float2 s = mul2(mul2(qm, inv), mul2(inv, inv));
                if (COMP) {
                    TX[k] = fma2(dx, s, TX[k]); TY[k] = fma2(dy, s, TY[k]); TZ[k] = fma2(dz, s, TZ[k]);
                } else {
                    AX[k] = fma2(dx, s, AX[k]); AY[k] = fma2(dy, s, AY[k]); AZ[k] = fma2(dz, s, AZ[k]);
                }
            }
        }
        if (COMP) {
#pragma unroll
            for (int k = 0; k < P; ++k) {
                fold(AX[k].x, CX[k].x, TX[k].x); fold(AX[k].y, CX[k].y, TX[k].y);
                fold(AY[k].x, CY[k].x, TY[k].x); fold(AY[k].y, CY[k].y, TY[k].y);
                fold(AZ[k].x, CZ[k].x, TZ[k].x); fold(AZ[k].y, CZ[k].y, TZ[k].y);
            }
        }
    });

    const int64_t seg = blockIdx.y;
    const int K = COMP ? 6 : 3;
#pragma unroll
    for (int k = 0; k < P; ++k) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float* out = part + seg * K * n_pad + base + static_cast<int64_t>(2 * k + h) * blockDim.x;
            out[0] = h ? AX[k].y : AX[k].x;
            out[n_pad] = h ? AY[k].y : AY[k].x;
            out[2 * n_pad] = h ? AZ[k].y : AZ[k].x;
            if (COMP) {
                out[3 * n_pad] = h ? CX[k].y : CX[k].x;
                out[4 * n_pad] = h ? CY[k].y : CY[k].x;
                out[5 * n_pad] = h ? CZ[k].y : CZ[k].x;
            }
        }
    }
}
// ================================================================================================
// symmetric all-pairs gravity (Newton's third law): every unordered pair evaluated once
// ================================================================================================
// Particles form blocks of kSymB = 128 threads x 8; blocks form G groups of `gs` consecutive blocks.
// CTA t is the task (ga, gb), ga <= gb (the G(G-1)/2 pairs of distinct groups first, then the G
// diagonal ones): for every row block a of group ga it sweeps the column blocks of group gb (those
// after a when ga == gb) in j-tiles of kSymJT through shared memory. One 1/r^3 serves both particles
// of a pair: the row particle's sum stays in registers (f32x2, two row particles per instruction),
// accumulated per j-tile and then added to the running sum (plain: a sum of 256-term sums, whose
// rounding error grows with the tile count instead of the pair count; compensated: a two-sum fold whose
// error terms live in shared memory); the column particle's contribution is summed over the CTA's 1024 row particles -- in the thread, then
// across the warp by rotation (each lane takes the 32 columns of a block in turn and hands each column's
// running sum on to its neighbour), then over the four warps in shared memory -- and added to its slot
// in the partials (plain, or two-sum when compensated). The pairs inside a block (the diagonal tile) run one-sided. Each particle has G + 1
// slots, each written by one task (its row sums from tasks (g, gb), its column sums from tasks (ga, g),
// g its group); the finish kernels add a particle's slots in a fixed order, so results do not depend on
// scheduling. FMA-pipe work per pair interaction: 8 + ~0.4 operations
// against the one-sided kernel's 12.
constexpr int kSymT = 128, kSymI = 8, kSymB = kSymT * kSymI, kSymJT = 256;
static_assert(kSymB % kSymJT == 0 && kSymJT % kSymT == 0 && kSymJT % 32 == 0, "symmetric gravity tiles");
// CTAs per SM the register budget is set for. Four (128 registers, no spills with the rotating column
// sums): Plummer N = 2^20, 128 groups, 340.5 ms plain and 340.5 ms compensated, against 338.7 / 350.6 ms
// for a warp butterfly over batches of 8 columns at three CTAs per SM; five spill and run slower (359.6 ms)
constexpr int kSymCtas = 4;

__host__ __device__ __forceinline__ void sym_task(int t, int G, int& ga, int& gb) {
    const int noff = G * (G - 1) / 2;
    if (t >= noff) {
        ga = gb = t - noff;
        return;
    }
    int r = 0, rem = t;
    while (rem >= G - 1 - r) {
        rem -= G - 1 - r;
        ++r;
    }
    ga = r;
    gb = r + 1 + rem;
}

template <int GRAV, bool COMP>
__global__ void __launch_bounds__(kSymT, kSymCtas) k_gravity_sym(const float4* __restrict__ posm, float* __restrict__ part,
                                                       int64_t n_pad, int G, int gs, float eps2) {
    constexpr int P = kSymI / 2;
    constexpr int K = COMP ? 6 : 3;
    __shared__ float4 J[kSymJT];
    __shared__ float js[kSymT / 32][kSymJT][3];
    // the row particles' running sums (and, compensated, their rounding-error terms) stay in shared
    // memory, touched once per j-tile; the pair loop keeps only the tile's partials in registers
    __shared__ float2 rsh[3 * P][kSymT];
    __shared__ float2 csh[COMP ? 3 * P : 1][kSymT];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int ga, gb;
    sym_task(static_cast<int>(blockIdx.x), G, ga, gb);
    const int nb = static_cast<int>(n_pad / kSymB);
    const int ra0 = ga * gs, ra1 = min(nb, ra0 + gs);
    const int cg0 = gb * gs, cg1 = min(nb, cg0 + gs);
    const bool diag = ga == gb;
    // partials: G + 1 slots per particle, stored [slot][component][n_pad] so that a warp's 32 consecutive
    // particles write (and the fold kernel reads) 128 contiguous bytes; a particle of group g holds its row
    // sums from tasks (g, gb), gb = g .. G-1, in slots 0 .. G-1-g and its column sums from tasks (ga, g),
    // ga = 0 .. g, in slots G-g .. G, each slot written by exactly one task
    const int s_row = gb - ga, s_col = G - gb + ga;
    auto slot = [&](int64_t particle, int sl, int c) { return part + (static_cast<int64_t>(sl) * K + c) * n_pad + particle; };
    if (diag)  // the group's first block is never a column here: its column slot is zero
        for (int e = tid; e < kSymB; e += kSymT)
            for (int c = 0; c < K; ++c) *slot(static_cast<int64_t>(ra0) * kSymB + e, s_col, c) = 0.0f;
    const float2 E2 = make_float2(eps2, eps2);

    for (int a = ra0; a < ra1; ++a) {
        const int64_t base = static_cast<int64_t>(a) * kSymB + tid;
        float2 X[P], Y[P], Z[P], MI[P];
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const float4 u = posm[base + static_cast<int64_t>(2 * k) * kSymT];
            const float4 w = posm[base + static_cast<int64_t>(2 * k + 1) * kSymT];
            X[k] = make_float2(u.x, w.x); Y[k] = make_float2(u.y, w.y); Z[k] = make_float2(u.z, w.z);
            MI[k] = make_float2(-u.w, -w.w);
            rsh[k][tid] = rsh[P + k][tid] = rsh[2 * P + k][tid] = make_float2(0.0f, 0.0f);
            if (COMP) csh[k][tid] = csh[P + k][tid] = csh[2 * P + k][tid] = make_float2(0.0f, 0.0f);
        }
        // tiles: the block's own (one-sided) when diagonal, then the columns
        const int64_t d0 = static_cast<int64_t>(a) * kSymB;
        const int nd = diag ? kSymB / kSymJT : 0;
        const int64_t c0 = static_cast<int64_t>(diag ? a + 1 : cg0) * kSymB, c1 = static_cast<int64_t>(cg1) * kSymB;
        const int nc = c1 > c0 ? static_cast<int>((c1 - c0) / kSymJT) : 0;
        const int total = nd + nc;
        const bool first = a == ra0;
        auto src = [&](int k) { return k < nd ? d0 + static_cast<int64_t>(k) * kSymJT : c0 + static_cast<int64_t>(k - nd) * kSymJT; };
        constexpr int kPf = kSymJT / kSymT;  // j-records each thread stages per tile
        float4 pf[kPf];
#pragma unroll
        for (int h = 0; h < kPf; ++h) pf[h] = make_float4(0, 0, 0, 0);
        if (total > 0) {
#pragma unroll
            for (int h = 0; h < kPf; ++h) pf[h] = posm[src(0) + h * kSymT + tid];
        }
        for (int k = 0; k < total; ++k) {
            __syncthreads();  // the previous tile's reads of J and js are done
#pragma unroll
            for (int h = 0; h < kPf; ++h) J[tid + h * kSymT] = pf[h];
            __syncthreads();
            if (k + 1 < total) {
#pragma unroll
                for (int h = 0; h < kPf; ++h) pf[h] = posm[src(k + 1) + h * kSymT + tid];
            }
            float2 TX[P], TY[P], TZ[P];
#pragma unroll
            for (int q = 0; q < P; ++q) TX[q] = TY[q] = TZ[q] = make_float2(0.0f, 0.0f);
            if (k < nd) {  // one-sided, as k_gravity_x2
#pragma unroll 4
                for (int j = 0; j < kSymJT; ++j) {
                    const float4 q = J[j];
                    const float2 qx = make_float2(q.x, q.x), qy = make_float2(q.y, q.y), qz = make_float2(q.z, q.z),
                                 qm = make_float2(q.w, q.w);
#pragma unroll
                    for (int m = 0; m < P; ++m) {
                        const float2 dx = sub2(qx, X[m]), dy = sub2(qy, Y[m]), dz = sub2(qz, Z[m]);
                        const float2 r2 = fma2(dz, dz, fma2(dy, dy, fma2(dx, dx, E2)));
                        float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                        if (GRAV == 2) inv = make_float2(fminf(inv.x, 1e12f), fminf(inv.y, 1e12f));
                        const float2 sj = mul2(qm, mul2(mul2(inv, inv), inv));
                        TX[m] = fma2(dx, sj, TX[m]); TY[m] = fma2(dy, sj, TY[m]); TZ[m] = fma2(dz, sj, TZ[m]);
                    }
                }
            } else {
                // column sums by rotation: in round r of a block of 32 columns, lane l pairs its rows
                // with column (l + r) % 32, adds its share to that column's running sum and hands the sum
                // to lane l - 1, which takes the column in round r + 1; after 32 rounds lane l holds the
                // warp's sum for column l (no butterfly, no selects, 3 shuffles per column)
                const int next = (lane + 1) & 31;
#pragma unroll 1
                for (int j0 = 0; j0 < kSymJT; j0 += 32) {
                    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
#pragma unroll 2
                    for (int r = 0; r < 32; ++r) {
                        const float4 q = J[j0 + ((lane + r) & 31)];
                        const float2 qx = make_float2(q.x, q.x), qy = make_float2(q.y, q.y),
                                     qz = make_float2(q.z, q.z), qm = make_float2(q.w, q.w);
                        float2 tx = make_float2(0.0f, 0.0f), ty = tx, tz = tx;
#pragma unroll
                        for (int m = 0; m < P; ++m) {
                            const float2 dx = sub2(qx, X[m]), dy = sub2(qy, Y[m]), dz = sub2(qz, Z[m]);
                            const float2 r2 = fma2(dz, dz, fma2(dy, dy, fma2(dx, dx, E2)));
                            float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                            if (GRAV == 2) inv = make_float2(fminf(inv.x, 1e12f), fminf(inv.y, 1e12f));
                            const float2 i3 = mul2(mul2(inv, inv), inv);
                            const float2 sj = mul2(qm, i3), si = mul2(MI[m], i3);
                            TX[m] = fma2(dx, sj, TX[m]); TY[m] = fma2(dy, sj, TY[m]); TZ[m] = fma2(dz, sj, TZ[m]);
                            tx = fma2(dx, si, tx); ty = fma2(dy, si, ty); tz = fma2(dz, si, tz);
                        }
                        cx = __shfl_sync(0xffffffffu, cx + (tx.x + tx.y), next);
                        cy = __shfl_sync(0xffffffffu, cy + (ty.x + ty.y), next);
                        cz = __shfl_sync(0xffffffffu, cz + (tz.x + tz.y), next);
                    }
                    js[warp][j0 + lane][0] = cx;
                    js[warp][j0 + lane][1] = cy;
                    js[warp][j0 + lane][2] = cz;
                }
            }
            // the tile's row partials into the running sums: a two-sum fold (compensated), or one add
            // (plain: a sum of 256-term tile sums, not one running sum over the whole column group)
#pragma unroll
            for (int m = 0; m < P; ++m) {
                float2 ax = rsh[m][tid], ay = rsh[P + m][tid], az = rsh[2 * P + m][tid];
                if (COMP) {
                    float2 cx = csh[m][tid], cy = csh[P + m][tid], cz = csh[2 * P + m][tid];
                    fold(ax.x, cx.x, TX[m].x); fold(ax.y, cx.y, TX[m].y);
                    fold(ay.x, cy.x, TY[m].x); fold(ay.y, cy.y, TY[m].y);
                    fold(az.x, cz.x, TZ[m].x); fold(az.y, cz.y, TZ[m].y);
                    csh[m][tid] = cx; csh[P + m][tid] = cy; csh[2 * P + m][tid] = cz;
                } else {
                    ax = add2(ax, TX[m]); ay = add2(ay, TY[m]); az = add2(az, TZ[m]);
                }
                rsh[m][tid] = ax; rsh[P + m][tid] = ay; rsh[2 * P + m][tid] = az;
            }
            if (k >= nd) {  // this tile's column sums over the CTA's row block, into the column slot
                __syncthreads();
                const int64_t jb = c0 + static_cast<int64_t>(k - nd) * kSymJT;
#pragma unroll
                for (int h = 0; h < kSymJT / kSymT; ++h) {
                    const int j = tid + h * kSymT;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const float v = (js[0][j][c] + js[1][j][c]) + (js[2][j][c] + js[3][j][c]);
                        float* dst = slot(jb + j, s_col, c);
                        if (COMP) {
                            float* cdst = slot(jb + j, s_col, 3 + c);
                            if (first) {
                                *dst = v;
                                *cdst = 0.0f;
                            } else {
                                float sv = *dst, cv = *cdst;
                                fold(sv, cv, v);
                                *dst = sv;
                                *cdst = cv;
                            }
                        } else {
                            *dst = first ? v : *dst + v;
                        }
                    }
                }
            }
        }
        // the row sums of block a into its row slot
#pragma unroll
        for (int m = 0; m < P; ++m) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int64_t pr = base + static_cast<int64_t>(2 * m + h) * kSymT;
                *slot(pr, s_row, 0) = h ? rsh[m][tid].y : rsh[m][tid].x;
                *slot(pr, s_row, 1) = h ? rsh[P + m][tid].y : rsh[P + m][tid].x;
                *slot(pr, s_row, 2) = h ? rsh[2 * P + m][tid].y : rsh[2 * P + m][tid].x;
                if (COMP) {
                    *slot(pr, s_row, 3) = h ? csh[m][tid].y : csh[m][tid].x;
                    *slot(pr, s_row, 4) = h ? csh[P + m][tid].y : csh[P + m][tid].x;
                    *slot(pr, s_row, 5) = h ? csh[2 * P + m][tid].y : csh[2 * P + m][tid].x;
                }
            }
        }
    }
}

template <int I, int GRAV, bool COMP>
__global__ void __launch_bounds__(128) k_gravity(const float4* __restrict__ posm, float* __restrict__ part,
                                                  int64_t n_pad, int jt, int nseg, float eps2, int* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    JTilePipe<1> pipe;
    pipe.buf = reinterpret_cast<float4*>(smem_raw);
    pipe.bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * jt * sizeof(float4));
    pipe.src[0] = posm;
    pipe.jt = jt;
    pipe.status = status;
    segment_tiles(n_pad / jt, blockIdx.y, nseg, pipe.t_begin, pipe.t_end);

    const int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x * I + threadIdx.x;
    float xi[I], yi[I], zi[I], ax[I], ay[I], az[I], cx[I], cy[I], cz[I];
#pragma unroll
    for (int k = 0; k < I; ++k) {
        const float4 q = posm[base + static_cast<int64_t>(k) * blockDim.x];
        xi[k] = q.x; yi[k] = q.y; zi[k] = q.z;
        ax[k] = ay[k] = az[k] = 0.0f;
        cx[k] = cy[k] = cz[k] = 0.0f;
    }

    pipe.start();
    pipe.run([&](const float4* J) {
        float tx[I], ty[I], tz[I];
#pragma unroll
        for (int k = 0; k < I; ++k) tx[k] = ty[k] = tz[k] = 0.0f;
#pragma unroll 4
        for (int j = 0; j < jt; ++j) {
            const float4 q = J[j];
#pragma unroll
            for (int k = 0; k < I; ++k) {
                const float dx = q.x - xi[k], dy = q.y - yi[k], dz = q.z - zi[k];
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
                float inv = rsqrtf(r2);
                if (GRAV == 2) inv = fminf(inv, 1e12f);
                const float s = q.w * inv * (inv * inv);
                if (COMP) {
                    tx[k] = fmaf(dx, s, tx[k]);
                    ty[k] = fmaf(dy, s, ty[k]);
                    tz[k] = fmaf(dz, s, tz[k]);
                } else {
                    ax[k] = fmaf(dx, s, ax[k]);
                    ay[k] = fmaf(dy, s, ay[k]);
                    az[k] = fmaf(dz, s, az[k]);
                }
            }
        }
        if (COMP) {
#pragma unroll
            for (int k = 0; k < I; ++k) {
                fold(ax[k], cx[k], tx[k]);
                fold(ay[k], cy[k], ty[k]);
                fold(az[k], cz[k], tz[k]);
            }
        }
    });

    const int64_t seg = blockIdx.y;
    const int K = COMP ? 6 : 3;
#pragma unroll
    for (int k = 0; k < I; ++k) {
        float* out = part + seg * K * n_pad + base + static_cast<int64_t>(k) * blockDim.x;
        out[0] = ax[k];
        out[n_pad] = ay[k];
        out[2 * n_pad] = az[k];
        if (COMP) {
            out[3 * n_pad] = cx[k];
            out[4 * n_pad] = cy[k];
            out[5 * n_pad] = cz[k];
        }
    }
}

template <bool COMP>
__global__ void __launch_bounds__(256) k_gravity_finish(DevArrays a, DevParams p, GravSum gsum) {
    const int64_t i = fold_particle();
    if (has(p, GSPH_VARIABLE_TIMESTEP) && blockIdx.x == 0 && threadIdx.x == 0) a.dt_state[1] = p.max_dt;
    double t[3];
    fold_slots<COMP>(a.part, a.n_pad, gsum.sym_G > 0 ? gsum.sym_G + 1 : gsum.nseg, i, i < a.n, t);
    if ((threadIdx.x & 31) >= 8 || i >= a.n) return;
    float acc[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        acc[c] = COMP ? static_cast<float>(t[c] * static_cast<double>(p.G)) : p.G * static_cast<float>(t[c]);
    if (a.grav) a.grav[i] = make_float4(acc[0], acc[1], acc[2], 0.0f);
    environment(p, a.posm[i], a.velrho[i], acc[0], acc[1], acc[2]);
    a.acc[i] = make_float4(acc[0], acc[1], acc[2], 0.0f);
    a.xvel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

inline unsigned blocks_for(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

// ---- host launchers ----------------------------------------------------------------------------
// Event record that also works while `s` is being captured into a graph (as an event-record node).
cudaError_t timer_record(cudaEvent_t ev, cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &st);
    if (e != cudaSuccess) return e;
    if (st == cudaStreamCaptureStatusActive) return cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal);
    return cudaEventRecord(ev, s);
}

#define GSPH_TIMER_MARK(t, which)                          \
    do {                                                   \
        if (t) {                                           \
            cudaError_t te_ = timer_record((t)->which, s); \
            if (te_ != cudaSuccess) return te_;            \
        }                                                  \
    } while (0)

namespace {
CullView cull_view(const DevArrays& a, const SpatialArrays& sp) {
    CullView cv;
    cv.list = sp.list;
    cv.count = sp.count;
    cv.item_start = sp.item_start;
    cv.ngroups = static_cast<int>(a.n_pad / kGroup);
    cv.nchunks = a.n_pad / kChunk;
    cv.part = sp.item_part;
    cv.nb = nullptr;
    cv.nbcnt = nullptr;
    cv.nbover = nullptr;
    cv.box_lo = sp.box_lo;
    cv.box_hi = sp.box_hi;
    return cv;
}
PartView seg_view(const DevArrays& a, int nseg, int KK, bool err) {
    return PartView{a.part, a.n_pad, nseg, nullptr, KK, err};
}
PartView item_view(const DevArrays& a, const SpatialArrays& sp, int KK, bool err) {
    return PartView{sp.item_part, a.n_pad, 0, sp.item_start, KK, err};
}

// One block: chunks per item ic = ceil(total near chunks / target) so that items carry equal work,
// then the exclusive scan of the per-group item counts ceil(count / ic) in a fixed order.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) k_work_items(const int* __restrict__ count, int* __restrict__ start,
                                                             int ngroups, int target) {
    __shared__ int warp_sums[kScanThreads / 32];
    __shared__ int carry;
    __shared__ int ic_sh;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int part = 0;  // total near chunks
    for (int g = threadIdx.x; g < ngroups; g += kScanThreads) part += count[g];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) warp_sums[warp] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long total = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) total += warp_sums[w];
        const long long ic = (total + target - 1) / target;
        ic_sh = static_cast<int>(ic < 1 ? 1 : ic);
        carry = 0;
    }
    __syncthreads();
    const int ic = ic_sh;
    for (int base = 0; base < ngroups; base += kScanThreads) {
        const int g = base + threadIdx.x;
        const int v = (g < ngroups) ? (count[g] + ic - 1) / ic : 0;
        int x = v;  // inclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        __syncthreads();
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const int before = carry + (warp ? warp_sums[warp - 1] : 0) + x - v;
        if (g < ngroups) start[g] = before;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        start[ngroups] = carry;
        start[ngroups + 1] = ic;
    }
}
}  // namespace

cudaError_t launch_work_items(const DevArrays& a, const SpatialArrays& sp, int target, cudaStream_t s) {
    k_work_items<<<1, kScanThreads, 0, s>>>(sp.count, sp.item_start, static_cast<int>(a.n_pad / kGroup), target);
    return cudaGetLastError();
}

cudaError_t launch_density(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s, const KTimer* t,
                           const SpatialArrays* sp) {
    const bool comp = L.accum == GSPH_ACCUM_COMPENSATED;
    GSPH_TIMER_MARK(t, start);
    if (sp) {
        const size_t smem = pipe_smem_bytes(1, kStageChunks * kChunk);
        const CullView cv = cull_view(a, *sp);
        CullView cvl = cv;
        cvl.nb = sp->item_nb;
        cvl.nbcnt = sp->item_nbcnt;
        cvl.nbover = sp->item_nbover;
        if (comp) k_density_items<true, true><<<L.density_grid, kGroup, smem, s>>>(a.posm, p, cvl, a.status);
        else k_density_items<false, true><<<L.density_grid, kGroup, smem, s>>>(a.posm, p, cvl, a.status);
    } else {
        const int T = 256;
        const dim3 grid(static_cast<unsigned>(a.n_pad / T), static_cast<unsigned>(L.nseg));
        const size_t smem = pipe_smem_bytes(1, L.jt);
        if (comp) k_density<true><<<grid, T, smem, s>>>(a.posm, a.part, a.n_pad, L.jt, L.nseg, p, a.status);
        else k_density<false><<<grid, T, smem, s>>>(a.posm, a.part, a.n_pad, L.jt, L.nseg, p, a.status);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    GSPH_TIMER_MARK(t, stop);
    const int KK = comp ? 2 : 1;
    const PartView pv = sp ? item_view(a, *sp, KK, comp) : seg_view(a, L.nseg, KK, comp);
    if (comp) k_density_finish<true><<<blocks_for(a.n, 256), 256, 0, s>>>(a, p, pv);
    else k_density_finish<false><<<blocks_for(a.n, 256), 256, 0, s>>>(a, p, pv);
    return cudaGetLastError();
}

cudaError_t launch_prepare(const DevArrays& a, const DevParams& p, cudaStream_t s) {
    k_prepare<<<blocks_for(a.n, 256), 256, 0, s>>>(a, p);
    return cudaGetLastError();
}

namespace {
template <int PASS, int GRAV, bool SOLIDS, bool COMP>
cudaError_t pairs_t(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s, const KTimer* t,
                    const SpatialArrays* sp, int gnseg, cudaEvent_t join, bool lists) {
    constexpr int NS = (PASS == PASS_VGRAD) ? 2 : 4;
    if (sp) {  // SPH terms over the near-chunk work items; gravity partials come from elsewhere
        constexpr uint32_t MASK = field_mask<PASS, false, SOLIDS>();
        constexpr int K = popc_c(MASK);
        // position stages, then per warp the [kNbCap][32] neighbour-index lists
        const size_t smem = pipe_smem_bytes(1, kStageChunks * kChunk) + (kGroup / 32) * kNbCap * 32 * sizeof(int);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_pairs_items<PASS, SOLIDS, false>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            if (e != cudaSuccess) return e;
        }
        GSPH_TIMER_MARK(t, start);
        CullView cv = cull_view(a, *sp);
        if (lists) {
            cv.nb = sp->item_nb;
            cv.nbcnt = sp->item_nbcnt;
            cv.nbover = sp->item_nbover;
        }
        // one work item is one tile of its particles' neighbour sums (a few to tens of terms): its
        // partials carry no compensation term, and the compensated form folds the items in FP64 in the
        // finish, so both forms run the plain kernel
        k_pairs_items<PASS, SOLIDS, false><<<L.item_grid, kGroup, smem, s>>>(a, p, cv);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        GSPH_TIMER_MARK(t, stop);
        if (join) {
            e = cudaStreamWaitEvent(s, join, 0);
            if (e != cudaSuccess) return e;
        }
        k_pairs_finish<PASS, false, SOLIDS, COMP><<<blocks_for(a.n, 256), 256, 0, s>>>(
            a, p, item_view(a, *sp, K, false), grav_sum(L, PASS == PASS_VGRAD ? 0 : gnseg));
        return cudaGetLastError();
    }
    constexpr uint32_t MASK = field_mask<PASS, (GRAV != 0), SOLIDS>();
    constexpr int K = popc_c(MASK);
    const size_t smem = pipe_smem_bytes(NS, L.jt);
    auto kern = k_pairs<PASS, GRAV, SOLIDS, COMP>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    const dim3 grid(static_cast<unsigned>(a.n_pad / L.threads), static_cast<unsigned>(L.nseg));
    GSPH_TIMER_MARK(t, start);
    kern<<<grid, L.threads, smem, s>>>(a, p, L.jt, L.nseg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    GSPH_TIMER_MARK(t, stop);
    k_pairs_finish<PASS, (GRAV != 0), SOLIDS, COMP><<<blocks_for(a.n, 256), 256, 0, s>>>(
        a, p, seg_view(a, L.nseg, COMP ? 2 * K : K, COMP), GravSum{});
    return cudaGetLastError();
}

template <int PASS, int GRAV>
cudaError_t pairs_g(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s, const KTimer* t,
                    const SpatialArrays* sp, int gnseg, cudaEvent_t join, bool lists = false) {
    const bool solids = has(p, GSPH_SOLIDS);
    const bool comp = L.accum == GSPH_ACCUM_COMPENSATED;
    if (solids)
        return comp ? pairs_t<PASS, GRAV, true, true>(a, p, L, s, t, sp, gnseg, join, lists)
                    : pairs_t<PASS, GRAV, true, false>(a, p, L, s, t, sp, gnseg, join, lists);
    return comp ? pairs_t<PASS, GRAV, false, true>(a, p, L, s, t, sp, gnseg, join, lists)
                : pairs_t<PASS, GRAV, false, false>(a, p, L, s, t, sp, gnseg, join, lists);
}
}  // namespace

cudaError_t launch_pairs(int pass, const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s,
                         const KTimer* t, const SpatialArrays* sp, int gnseg, cudaEvent_t join, bool lists) {
    if (sp) {  // the culled kernels carry no gravity
        switch (pass) {
            case PASS_VGRAD: return pairs_g<PASS_VGRAD, 0>(a, p, L, s, t, sp, 0, join, lists);
            case PASS_ACC: return pairs_g<PASS_ACC, 0>(a, p, L, s, t, sp, gnseg, join, lists);
            default: return pairs_g<PASS_FUSED, 0>(a, p, L, s, t, sp, gnseg, join, lists);
        }
    }
    const int grav = !has(p, GSPH_SELF_GRAVITY) ? 0 : (p.eps2 > 0.0f ? 1 : 2);
    switch (pass) {
        case PASS_VGRAD: return pairs_g<PASS_VGRAD, 0>(a, p, L, s, t, nullptr, 0, nullptr);
        case PASS_ACC:
            return grav == 0 ? pairs_g<PASS_ACC, 0>(a, p, L, s, t, nullptr, 0, nullptr)
                             : (grav == 1 ? pairs_g<PASS_ACC, 1>(a, p, L, s, t, nullptr, 0, nullptr)
                                          : pairs_g<PASS_ACC, 2>(a, p, L, s, t, nullptr, 0, nullptr));
        default:
            return grav == 0 ? pairs_g<PASS_FUSED, 0>(a, p, L, s, t, nullptr, 0, nullptr)
                             : (grav == 1 ? pairs_g<PASS_FUSED, 1>(a, p, L, s, t, nullptr, 0, nullptr)
                                          : pairs_g<PASS_FUSED, 2>(a, p, L, s, t, nullptr, 0, nullptr));
    }
}

namespace {
template <int I, int GRAV, bool COMP>
cudaError_t gravity_t(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s, const KTimer* t,
                      bool finish) {
    const int T = L.grav_threads;
    const dim3 grid(static_cast<unsigned>(a.n_pad / (static_cast<int64_t>(T) * I)), static_cast<unsigned>(L.grav_nseg));
    const size_t smem = pipe_smem_bytes(1, L.grav_jt);
    GSPH_TIMER_MARK(t, start);
    if (L.grav_sym_G > 0) {
        const int G = L.grav_sym_G;
        k_gravity_sym<GRAV, COMP><<<static_cast<unsigned>(G * (G + 1) / 2), kSymT, 0, s>>>(
            a.posm, finish ? a.part : a.gpart, a.n_pad, G, L.grav_sym_gs, p.eps2);
    } else if constexpr (I >= 2) {
        if (L.grav_x2)
            k_gravity_x2<I, GRAV, COMP><<<grid, T, smem, s>>>(a.posm, finish ? a.part : a.gpart, a.n_pad, L.grav_jt,
                                                               L.grav_nseg, p.eps2, a.status);
        else
            k_gravity<I, GRAV, COMP><<<grid, T, smem, s>>>(a.posm, finish ? a.part : a.gpart, a.n_pad, L.grav_jt,
                                                            L.grav_nseg, p.eps2, a.status);
    } else {
        k_gravity<I, GRAV, COMP><<<grid, T, smem, s>>>(a.posm, finish ? a.part : a.gpart, a.n_pad, L.grav_jt,
                                                        L.grav_nseg, p.eps2, a.status);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    GSPH_TIMER_MARK(t, stop);
    const int S = L.grav_sym_G > 0 ? L.grav_sym_G + 1 : L.grav_nseg;
    const unsigned fold_blocks = blocks_for(a.n * kFoldT, 256);  // kFoldT threads per particle
    if (!finish) {  // the culled path: fold on this (the gravity) stream, the SPH finish reads a.gfold
        k_gravity_fold<COMP><<<fold_blocks, 256, 0, s>>>(a.gpart, a.n, a.n_pad, S, a.gfold);
        return cudaGetLastError();
    }
    k_gravity_finish<COMP><<<fold_blocks, 256, 0, s>>>(a, p, grav_sum(L, L.grav_nseg));
    return cudaGetLastError();
}
template <int GRAV, bool COMP>
cudaError_t gravity_i(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s, const KTimer* t,
                      bool finish) {
    switch (L.grav_ipt) {
        case 1: return gravity_t<1, GRAV, COMP>(a, p, L, s, t, finish);
        case 2: return gravity_t<2, GRAV, COMP>(a, p, L, s, t, finish);
        case 8: return gravity_t<8, GRAV, COMP>(a, p, L, s, t, finish);
        default: return gravity_t<4, GRAV, COMP>(a, p, L, s, t, finish);
    }
}
cudaError_t gravity_any(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s, const KTimer* t,
                        bool finish) {
    const bool comp = L.accum == GSPH_ACCUM_COMPENSATED;
    if (p.eps2 > 0.0f) return comp ? gravity_i<1, true>(a, p, L, s, t, finish) : gravity_i<1, false>(a, p, L, s, t, finish);
    return comp ? gravity_i<2, true>(a, p, L, s, t, finish) : gravity_i<2, false>(a, p, L, s, t, finish);
}
}  // namespace

cudaError_t launch_gravity(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s, const KTimer* t) {
    const bool comp = L.accum == GSPH_ACCUM_COMPENSATED;
    if (!has(p, GSPH_SELF_GRAVITY)) {  // neither gravity nor SPH: environment terms only
        if (comp) k_gravity_finish<true><<<blocks_for(a.n, 256), 256, 0, s>>>(a, p, GravSum{});
        else k_gravity_finish<false><<<blocks_for(a.n, 256), 256, 0, s>>>(a, p, GravSum{});
        return cudaGetLastError();
    }
    return gravity_any(a, p, L, s, t, true);
}

cudaError_t launch_gravity_partials(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s,
                                    const KTimer* t) {
    return gravity_any(a, p, L, s, t, false);
}

// Gravity partials of caller-provided, already padded j-records into caller-provided partials
// (the allocation-free entry point, noalloc.cu): the plain-FP32 paired kernel.
cudaError_t launch_gravity_raw(const float4* posm_padded, float* part, int64_t n_pad, int ipt, int jt, int nseg,
                               float eps2, int* status, cudaStream_t s) {
    const int T = 128;
    const dim3 grid(static_cast<unsigned>(n_pad / (static_cast<int64_t>(T) * ipt)), static_cast<unsigned>(nseg));
    const size_t smem = pipe_smem_bytes(1, jt);
    const bool soft = eps2 > 0.0f;
    if (ipt == 4) {
        if (soft) k_gravity_x2<4, 1, false><<<grid, T, smem, s>>>(posm_padded, part, n_pad, jt, nseg, eps2, status);
        else k_gravity_x2<4, 2, false><<<grid, T, smem, s>>>(posm_padded, part, n_pad, jt, nseg, eps2, status);
    } else {
        if (soft) k_gravity_x2<2, 1, false><<<grid, T, smem, s>>>(posm_padded, part, n_pad, jt, nseg, eps2, status);
        else k_gravity_x2<2, 2, false><<<grid, T, smem, s>>>(posm_padded, part, n_pad, jt, nseg, eps2, status);
    }
    return cudaGetLastError();
}

// ---- FP32 FFMA throughput probe (roofline denominator) -------------------------------------------
namespace {
constexpr int kPeakThreads = 256;
constexpr int kPeakBlocksPerSM = 4;
constexpr int kPeakChains = 16;
constexpr int kPeakUnroll = 16;
__global__ void __launch_bounds__(kPeakThreads) k_fp32_peak(float* sink, int iters) {
    float x[kPeakChains];
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) x[c] = static_cast<float>(threadIdx.x + c) * 1e-3f;
    const float a = 0.999999f, b = 1e-7f;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int u = 0; u < kPeakUnroll; ++u)
#pragma unroll
            for (int c = 0; c < kPeakChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) s += x[c];
    if (s == -1.0f) sink[blockIdx.x] = s;  // never true; keeps the chains live
}
}  // namespace

cudaError_t launch_fp32_peak(int sm_count, int iters, float* sink, cudaStream_t s) {
    k_fp32_peak<<<sm_count * kPeakBlocksPerSM, kPeakThreads, 0, s>>>(sink, iters);
    return cudaGetLastError();
}

int64_t fp32_peak_flops(int sm_count, int iters) {
    return static_cast<int64_t>(sm_count) * kPeakBlocksPerSM * kPeakThreads * static_cast<int64_t>(iters) *
           kPeakUnroll * kPeakChains * 2;
}

size_t partial_floats(const DevParams& p, const Launch& L, int64_t n_pad) {
    const int mult = (L.accum == GSPH_ACCUM_COMPENSATED) ? 2 : 1;
    size_t k = 0;
    if (has(p, GSPH_SPH)) {
        const size_t kd = 1;
        const size_t kp = static_cast<size_t>(popc_c(field_mask<PASS_FUSED, true, true>()));
        k = std::max(kd, kp);
        k = std::max<size_t>(k, static_cast<size_t>(popc_c(field_mask<PASS_FUSED, true, false>())));
        k *= static_cast<size_t>(std::max(L.nseg, 1));
    } else {
        k = 3 * static_cast<size_t>(L.grav_sym_G > 0 ? L.grav_sym_G + 1 : std::max(L.grav_nseg, 1));
    }
    return k * mult * static_cast<size_t>(n_pad);
}

int gravity_blocks_per_sm(int ipt, int threads, int jt, bool comp) {
    const size_t smem = pipe_smem_bytes(1, jt);
    int nb = 0;
    cudaError_t e = cudaSuccess;
#define GSPH_OCC(I)                                                                                      \
    e = comp ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gravity<I, 1, true>, threads, smem)  \
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gravity<I, 1, false>, threads, smem)
    switch (ipt) {
        case 1: GSPH_OCC(1); break;
        case 2: GSPH_OCC(2); break;
        case 8: GSPH_OCC(8); break;
        default: GSPH_OCC(4); break;
    }
#undef GSPH_OCC
    return (e == cudaSuccess && nb > 0) ? nb : 4;
}

size_t gravity_partial_floats(const Launch& L, int64_t n_pad) {
    const int mult = (L.accum == GSPH_ACCUM_COMPENSATED) ? 2 : 1;
    const int slots = L.grav_sym_G > 0 ? L.grav_sym_G + 1 : std::max(L.grav_nseg, 1);
    return static_cast<size_t>(3) * mult * static_cast<size_t>(slots) * static_cast<size_t>(n_pad);
}

}  // namespace gsph
