// ensemble.cu -- a batch of independent simulations of uneven particle counts, advanced together.
//
// The reference runs one simulation per process (src/main.cu:228-273). Here S simulations share one
// set of device arrays, packed back to back in the order of an offset table, with one parameter set.
// A substep is ONE persistent launch over a work queue of particle groups (kEnsGroup particles of one
// simulation each), in three stages:
//
//   DENS  gravity of the group against every particle of its own simulation, the SPH density sum and
//         the neighbour list of each particle (0 < r <= H), all from one sweep over the simulation's
//         positions staged in shared memory by bulk copies; then the j-records sigma/rho^2
//   SPH   the SPH terms over each particle's neighbour list (gathers from L2) and the per-particle
//         epilogue (stress rate, drho/dt, acceleration = G * gravity + SPH + environment)
//   KICK  the leapfrog kick-drift of the group (FP64 master positions), plasticity
//
// Queue order is stage-major, and within a stage simulations go largest first, so the long items
// start early and the short ones fill the tail. An SPH item of simulation k waits (bounded) until every
// DENS item of k is done, a KICK item until every SPH item of k is done; both wait only on items taken
// from the queue before them, which running CTAs hold and finish without waiting, so the waits end.
// Counters are released with a device-scope fence + atomic and acquired with ld.acquire + fence.
//
// Neighbour lists hold kEnsCap slots per particle (slot-major, so a warp reads them coalesced). A particle
// with more neighbours is marked and its SPH item sweeps the whole simulation instead: same result,
// slower. Sums run in a fixed order (j ascending), so results are deterministic.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "integrate.cuh"
#include "spatial.cuh"
#include "sph.cuh"

void set_global_error(const std::string& msg);                 // capi.cu
gsph::DevParams gsph_dev_params(const gsph_params& p);         // capi.cu

using namespace gsph;

namespace {

constexpr int kEnsThreads = 128;
constexpr int kEnsIpt = 4;                    // particles per thread (two f32x2 pairs in the sweep)
constexpr int kEnsGroup = kEnsThreads * kEnsIpt;    // particles per work item
constexpr int kEnsTile = 512;                 // default j-particles per shared-memory stage (autotuned)
constexpr int kEnsCap = 256;                  // neighbour-list slots per particle
constexpr int kEnsDiagF = 12;                 // diagnostic fields (as gsph_diagnostics)

enum Stage : int { ST_DENS = 0, ST_SPH = 1, ST_KICK = 2 };

struct EnsView {
    const int4* groups;  // [G] (simulation, first particle, particle count, 0); queue order
    const int4* sims;    // [S] (first particle, particle count, first group, group count)
    int ngroups, nsims;
    int stages[3];       // the stages of this launch, in order
    int nstages;
    int kick_dep;        // which done[] row a KICK item waits on (-1: none in this launch)
    int* head;           // work-queue head
    int* done;           // [2][S]: finished DENS / SPH items of each simulation
    int* nb;             // [kEnsCap][n] neighbour lists, slot-major
    int* nbcnt;          // [n] neighbour counts (kEnsCap + 1: the list overflowed)
    int64_t n;
    float kick_dt;
    int tile;            // j-particles per shared-memory stage of the DENS sweep
    int stall_sim;       // failure-path test: this simulation's SPH items wait for one DENS item more than
                         // exist, so their waits run out (-1: none)
    // symmetric gravity (GSYM stage, first in the queue when ntasks > 0): tasks (sim, row group, column
    // group, 0) of each simulation's group pairs, and the per-simulation partial slots they fill
    const int4* tasks;
    int ntasks;
    int sym;             // gravity comes from the GSYM slots (the DENS stage then skips gravity)
    float* gslot;        // all simulations' slots; simulation k's start at slot_base[k]
    const long long* slot_base;
};

// ---- paired FP32 (PTX ISA 8.6, sm_100+): two lanes per instruction, IEEE single precision ---------
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
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(u64_of(a)), "l"(u64_of(b)));
    return f2_of(d);
}

// ---- cross-CTA counters --------------------------------------------------------------------------
__device__ __forceinline__ int64_t lmin(int64_t x, int64_t y) { return x < y ? x : y; }

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// every thread's writes of the finished item, then one device-scope increment
__device__ __forceinline__ void signal_done(int* ctr) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1);
    }
}
// wait until *ctr >= target; false, with the status word set, if it gave up. The bound is status[1]
// microseconds when set (gsph_options.wait_limit_us), else kWaitLimitNs.
__device__ __forceinline__ bool wait_count(const int* ctr, int target, int* status, int* s_flag) {
    if (threadIdx.x == 0) {
        int ok = 1;
        if (ld_acquire(ctr) < target) {
            const int lim_us = status[1];
            const uint64_t limit = lim_us > 0 ? static_cast<uint64_t>(lim_us) * 1000ull : kWaitLimitNs;
            const uint64_t t0 = global_timer_ns();
            while (ld_acquire(ctr) < target) {
                if (global_timer_ns() - t0 > limit) {
                    atomicOr(status, GSPH_DEV_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(256);
            }
        }
        *s_flag = ok;
    }
    __syncthreads();
    const bool ok = *s_flag != 0;
    __threadfence();  // acquire side for every thread's own loads
    return ok;
}

// Two-stage bulk-copy pipeline over a contiguous j-range [j0, j1) of one float4 stream, `tile` records
// per stage (the last one ragged). The stage counter runs on across items so the mbarrier phases stay
// in step.
struct RangePipe {
    float4* buf;    // shared [2][tile]
    uint64_t* bar;  // shared [2]
    const float4* src;
    int* status;
    int tile;       // j-particles per stage
    uint32_t kst = 0;

    __device__ __forceinline__ void init() {
        if (threadIdx.x == 0) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            fence_barrier_init();
        }
        __syncthreads();
    }
    __device__ __forceinline__ void issue(int b, int64_t j, int nj) {
        mbar_expect_tx(&bar[b], static_cast<uint32_t>(nj * sizeof(float4)));
        bulk_g2s(buf + static_cast<int64_t>(b) * tile, src + j, static_cast<uint32_t>(nj * sizeof(float4)), &bar[b]);
    }
    // body(stage, nj, first j of the stage); false if a wait gave up
    template <typename Body>
    __device__ __forceinline__ bool run(int64_t j0, int64_t j1, Body&& body) {
        const int64_t len = j1 - j0;
        const int nst = static_cast<int>((len + tile - 1) / tile);
        auto cnt = [&](int st) { return static_cast<int>(lmin(tile, len - static_cast<int64_t>(st) * tile)); };
        if (threadIdx.x == 0)
            for (int st = 0; st < 2 && st < nst; ++st) issue((kst + st) & 1, j0 + static_cast<int64_t>(st) * tile, cnt(st));
        for (int st = 0; st < nst; ++st) {
            const int b = kst & 1;
            const bool ok = mbar_wait_bounded(&bar[b], (kst >> 1) & 1, status);
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0 && st + 1 < nst)
                    mbar_wait_bounded(&bar[(kst + 1) & 1], ((kst + 1) >> 1) & 1, status);
                __syncthreads();
                return false;
            }
            body(buf + static_cast<int64_t>(b) * tile, cnt(st), j0 + static_cast<int64_t>(st) * tile);
            __syncthreads();
            if (threadIdx.x == 0 && st + 2 < nst) issue(b, j0 + static_cast<int64_t>(st + 2) * tile, cnt(st + 2));
            ++kst;
        }
        return true;
    }
};

// Bounding box of the block's points (each thread passes its own min and max): box[0..2] = lo,
// box[3..5] = hi, in shared memory and visible to every thread on return. scratch: 6 x warps floats.
__device__ __forceinline__ void block_box(float lx, float ly, float lz, float hx, float hy, float hz, float* scratch,
                                          float* box) {
    float v[6] = {lx, ly, lz, -hx, -hy, -hz};  // all minima
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 6; ++d) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[d] = fminf(v[d], __shfl_xor_sync(0xffffffffu, v[d], o));
        if (lane == 0) scratch[warp * 6 + d] = v[d];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        float m = INFINITY;
        for (int w = 0; w < kEnsThreads / 32; ++w) m = fminf(m, scratch[w * 6 + threadIdx.x]);
        box[threadIdx.x] = threadIdx.x < 3 ? m : -m;
    }
    __syncthreads();
}

// ---- DENS: gravity + density + neighbour lists over the group's simulation -------------------------
// GRAV: 0 off, 1 softened, 2 unsoftened (the self pair gives 0 through the clamp of 1/r).
template <int GRAV, bool SPH, bool COMP>
__device__ __forceinline__ bool dens_item(const DevArrays& a, const DevParams& p, const EnsView& v, RangePipe& pipe,
                                          int4 grp, int4 sm, float* sbox) {
    constexpr int P = kEnsIpt / 2;
    const int64_t g0 = grp.y;
    int64_t idx[kEnsIpt];
    bool valid[kEnsIpt];
    float2 X[P], Y[P], Z[P], AX[P], AY[P], AZ[P], CX[P], CY[P], CZ[P];
    float rho[kEnsIpt], rhoc[kEnsIpt];
    int cnt[kEnsIpt];
#pragma unroll
    for (int k = 0; k < kEnsIpt; ++k) {
        const int o = threadIdx.x + k * kEnsThreads;
        valid[k] = o < grp.z;
        idx[k] = g0 + (valid[k] ? o : 0);
        rho[k] = rhoc[k] = 0.0f;
        cnt[k] = 0;
    }
#pragma unroll
    for (int k = 0; k < P; ++k) {
        const float4 q0 = a.posm[idx[2 * k]], q1 = a.posm[idx[2 * k + 1]];
        X[k] = make_float2(q0.x, q1.x); Y[k] = make_float2(q0.y, q1.y); Z[k] = make_float2(q0.z, q1.z);
        AX[k] = AY[k] = AZ[k] = CX[k] = CY[k] = CZ[k] = make_float2(0.0f, 0.0f);
    }
    const float2 E2 = make_float2(p.eps2, p.eps2);
    const uint32_t span = __float_as_uint(p.H2);
    const float H2 = p.H2;
    const float inv_h = p.inv_h;
    float* scratch = sbox;
    float* gbox = sbox + 6 * (kEnsThreads / 32);
    float* tbox = gbox + 6;
    const float H2m = H2 * (1.0f + 1e-3f);  // conservative: a tile farther than this has no neighbour in any rounding
    if (SPH) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
        for (int k = 0; k < P; ++k) {
            lo[0] = fminf(lo[0], fminf(X[k].x, X[k].y)); hi[0] = fmaxf(hi[0], fmaxf(X[k].x, X[k].y));
            lo[1] = fminf(lo[1], fminf(Y[k].x, Y[k].y)); hi[1] = fmaxf(hi[1], fmaxf(Y[k].x, Y[k].y));
            lo[2] = fminf(lo[2], fminf(Z[k].x, Z[k].y)); hi[2] = fmaxf(hi[2], fmaxf(Z[k].x, Z[k].y));
        }
        block_box(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], scratch, gbox);
    }

    const bool ok = pipe.run(sm.x, static_cast<int64_t>(sm.x) + sm.y, [&](const float4* J, int nj, int64_t jb) {
        // is any j of this tile within h of the group's box? (else the neighbour tests are skipped)
        bool near_tile = false;
        if (SPH) {
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int t = threadIdx.x; t < nj; t += kEnsThreads) {
                const float4 q = J[t];
                lo[0] = fminf(lo[0], q.x); hi[0] = fmaxf(hi[0], q.x);
                lo[1] = fminf(lo[1], q.y); hi[1] = fmaxf(hi[1], q.y);
                lo[2] = fminf(lo[2], q.z); hi[2] = fmaxf(hi[2], q.z);
            }
            block_box(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], scratch, tbox);
            float d2 = 0.0f;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float d = fmaxf(0.0f, fmaxf(gbox[c] - tbox[3 + c], tbox[c] - gbox[3 + c]));
                d2 = fmaf(d, d, d2);
            }
            near_tile = d2 <= H2m;
        }
        if (GRAV == 0 && !near_tile) return;  // no gravity to sum and no neighbour in this tile
        float2 TX[P], TY[P], TZ[P];
        float tr[kEnsIpt];
#pragma unroll
        for (int k = 0; k < P; ++k) TX[k] = TY[k] = TZ[k] = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < kEnsIpt; ++k) tr[k] = 0.0f;
#pragma unroll 2
        for (int j = 0; j < nj; ++j) {
            const float4 q = J[j];
            const float2 qx = make_float2(q.x, q.x), qy = make_float2(q.y, q.y), qz = make_float2(q.z, q.z),
                         qm = make_float2(q.w, q.w);
            float2 R2[P];
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const float2 dx = sub2(qx, X[k]), dy = sub2(qy, Y[k]), dz = sub2(qz, Z[k]);
                const float2 r2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
                R2[k] = r2;
                if (GRAV != 0) {
                    const float2 r2e = add2(r2, E2);
                    float2 inv = make_float2(rsqrtf(r2e.x), rsqrtf(r2e.y));
                    if (GRAV == 2) inv = make_float2(fminf(inv.x, 1e12f), fminf(inv.y, 1e12f));
                    const float2 s = mul2(mul2(qm, inv), mul2(inv, inv));
                    if (COMP) {
                        TX[k] = fma2(dx, s, TX[k]); TY[k] = fma2(dy, s, TY[k]); TZ[k] = fma2(dz, s, TZ[k]);
                    } else {
                        AX[k] = fma2(dx, s, AX[k]); AY[k] = fma2(dy, s, AY[k]); AZ[k] = fma2(dz, s, AZ[k]);
                    }
                }
            }
            if (SPH && near_tile) {
                // one warp vote per j: particles of a group are close along the curve, so for most j no
                // lane has a neighbour and the per-particle window tests are skipped
                bool near = false;
#pragma unroll
                for (int k = 0; k < P; ++k) near |= (R2[k].x <= H2) | (R2[k].y <= H2);
                if (__any_sync(0xffffffffu, near)) {
#pragma unroll
                    for (int k = 0; k < P; ++k) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            // calcDensity's window 0 < r^2 <= H^2 (computeDerivatives.h:72), also the neighbour test
                            const float rr = h ? R2[k].y : R2[k].x;
                            if (in_open_closed(rr, 0u, span)) {
                                const int kk = 2 * k + h;
                                const float r = rr * rsqrtf(rr);
                                const float w = q.w * w_poly(r * inv_h);
                                if (COMP) tr[kk] += w;
                                else rho[kk] += w;
                                if (valid[kk]) {
                                    if (cnt[kk] < kEnsCap)
                                        v.nb[static_cast<int64_t>(cnt[kk]) * v.n + idx[kk]] = static_cast<int>(jb + j);
                                    cnt[kk] = min(cnt[kk] + 1, kEnsCap + 1);
                                }
                            }
                        }
                    }
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
#pragma unroll
            for (int k = 0; k < kEnsIpt; ++k) fold(rho[k], rhoc[k], tr[k]);
        }
    });
    if (!ok) return false;

#pragma unroll
    for (int k = 0; k < kEnsIpt; ++k) {
        if (!valid[k]) continue;
        const int64_t i = idx[k];
        const int pk = k / 2, h = k % 2;
        float g[3];
        const float sx = h ? AX[pk].y : AX[pk].x, sy = h ? AY[pk].y : AY[pk].x, sz = h ? AZ[pk].y : AZ[pk].x;
        const float cx = h ? CX[pk].y : CX[pk].x, cy = h ? CY[pk].y : CY[pk].x, cz = h ? CZ[pk].y : CZ[pk].x;
        if (SPH) {  // raw gravity sums for the SPH stage, which applies G
            if (COMP) {
                g[0] = static_cast<float>(static_cast<double>(sx) + static_cast<double>(cx));
                g[1] = static_cast<float>(static_cast<double>(sy) + static_cast<double>(cy));
                g[2] = static_cast<float>(static_cast<double>(sz) + static_cast<double>(cz));
            } else {
                g[0] = sx; g[1] = sy; g[2] = sz;
            }
            a.acc[i] = make_float4(g[0], g[1], g[2], 0.0f);
            float4 vr = a.velrho[i];
            if (!has(p, GSPH_INTEGRATE_DENSITY)) {  // calcDensity::do_after (:80-90)
                float r;
                if (COMP) r = static_cast<float>((static_cast<double>(rho[k]) + static_cast<double>(rhoc[k])) *
                                                 static_cast<double>(p.w_pref));
                else r = rho[k] * p.w_pref;
                if (has(p, GSPH_DEAL_WITH_NO_PARTNERS) && r < 0.001f) r = p.rho0 * 0.01f;
                vr.w = r;
                a.velrho[i] = vr;
            }
            float4 jA, jB;
            make_jrecord(p, vr.w, a.sA[i], a.sB[i], a.balsara[i], jA, jB);
            a.jA[i] = jA;
            a.jB[i] = jB;
            v.nbcnt[i] = cnt[k];
        } else {  // gravity only: the final acceleration (as k_gravity_finish)
            if (COMP) {
                g[0] = static_cast<float>((static_cast<double>(sx) + static_cast<double>(cx)) * static_cast<double>(p.G));
                g[1] = static_cast<float>((static_cast<double>(sy) + static_cast<double>(cy)) * static_cast<double>(p.G));
                g[2] = static_cast<float>((static_cast<double>(sz) + static_cast<double>(cz)) * static_cast<double>(p.G));
            } else {
                g[0] = p.G * sx; g[1] = p.G * sy; g[2] = p.G * sz;
            }
            environment(p, a.posm[i], a.velrho[i], g[0], g[1], g[2]);
            a.acc[i] = make_float4(g[0], g[1], g[2], 0.0f);
            a.xvel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    return true;
}

// ---- GSYM: symmetric gravity over pairs of groups of one simulation --------------------------------
// Task (sim, ga, gb), ga <= gb: every pair of a particle of group ga (the rows, four per thread in two
// f32x2 pairs) and one of group gb (the columns, streamed by the pipe) is evaluated once and its 1/r^3
// serves both: the rows' sums stay in registers, the columns' are summed over the task's rows (in the
// thread, by a butterfly over the warp, then over the four warps in shared memory). The diagonal task
// (ga == gb) runs one-sided over the group's own pairs. Every particle of a simulation with G groups has
// G + 1 slots, [slot][component][particle of the simulation]: its row sums from tasks (g, gb) in slots
// 0 .. G-1-g, its column sums from tasks (ga, g) in slots G-g .. G, each written by exactly one task (the
// diagonal task zeroes slot G); the SPH stage folds them in FP64 in slot order, so results are
// deterministic. Rows past the group's end are inert (zero mass, far away); columns past the simulation's
// end are never read.
constexpr int kEnsJC = 128;  // columns per shared-memory reduction round
constexpr int kEnsJB = 8;    // columns per warp butterfly

__device__ __forceinline__ float* sim_slots(const EnsView& v, int sim) { return v.gslot + v.slot_base[sim]; }

template <int GRAV, bool COMP>
__device__ __forceinline__ bool gsym_item(const DevArrays& a, const DevParams& p, const EnsView& v, RangePipe& pipe,
                                          int4 task, int4 sm, float (*js)[kEnsJC][3]) {
    constexpr int P = kEnsIpt / 2;
    constexpr int K = COMP ? 6 : 3;
    const int G = sm.w, ga = task.y, gb = task.z;
    const bool diag = ga == gb;
    const int64_t r0 = static_cast<int64_t>(sm.x) + static_cast<int64_t>(ga) * kEnsGroup;
    const int64_t c0 = static_cast<int64_t>(sm.x) + static_cast<int64_t>(gb) * kEnsGroup;
    const int rn = min(kEnsGroup, sm.y - ga * kEnsGroup), cn = min(kEnsGroup, sm.y - gb * kEnsGroup);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t N = sm.y;
    float* part = sim_slots(v, task.x);
    auto slot = [&](int local, int sl, int c) { return part + (static_cast<int64_t>(sl) * K + c) * N + local; };
    const int s_row = gb - ga, s_col = G - gb + ga;
    const float4 inert = make_float4(1e18f, 1e18f, 1e18f, 0.0f);
    float2 X[P], Y[P], Z[P], MI[P], AX[P], AY[P], AZ[P], CX[P], CY[P], CZ[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
        const int o0 = threadIdx.x + 2 * k * kEnsThreads, o1 = o0 + kEnsThreads;
        const float4 q0 = o0 < rn ? a.posm[r0 + o0] : inert, q1 = o1 < rn ? a.posm[r0 + o1] : inert;
        X[k] = make_float2(q0.x, q1.x); Y[k] = make_float2(q0.y, q1.y); Z[k] = make_float2(q0.z, q1.z);
        MI[k] = make_float2(-q0.w, -q1.w);  // the columns receive the opposite of the rows' force
        AX[k] = AY[k] = AZ[k] = CX[k] = CY[k] = CZ[k] = make_float2(0.0f, 0.0f);
    }
    if (diag)  // the group never is a column of its own diagonal task: that slot is zero
        for (int e = threadIdx.x; e < cn; e += kEnsThreads)
            for (int c = 0; c < K; ++c) *slot(gb * kEnsGroup + e, s_col, c) = 0.0f;
    const float2 E2 = make_float2(p.eps2, p.eps2);
    const bool ok = pipe.run(c0, c0 + cn, [&](const float4* J, int nj, int64_t jb) {
        float2 TX[P], TY[P], TZ[P];
#pragma unroll
        for (int k = 0; k < P; ++k) TX[k] = TY[k] = TZ[k] = make_float2(0.0f, 0.0f);
        for (int j0 = 0; j0 < nj; j0 += kEnsJC) {
            const int jn = min(kEnsJC, nj - j0);
#pragma unroll 1
            for (int u0 = 0; u0 < jn; u0 += kEnsJB) {
                float vx[kEnsJB], vy[kEnsJB], vz[kEnsJB];
#pragma unroll
                for (int u = 0; u < kEnsJB; ++u) {
                    const float4 q = (u0 + u < jn) ? J[j0 + u0 + u] : inert;
                    const float2 qx = make_float2(q.x, q.x), qy = make_float2(q.y, q.y), qz = make_float2(q.z, q.z),
                                 qm = make_float2(q.w, q.w);
                    float2 tx = make_float2(0.0f, 0.0f), ty = tx, tz = tx;
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const float2 dx = sub2(qx, X[k]), dy = sub2(qy, Y[k]), dz = sub2(qz, Z[k]);
                        const float2 r2 = fma2(dz, dz, fma2(dy, dy, fma2(dx, dx, E2)));
                        float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                        if (GRAV == 2) inv = make_float2(fminf(inv.x, 1e12f), fminf(inv.y, 1e12f));
                        const float2 i3 = mul2(mul2(inv, inv), inv);
                        const float2 sj = mul2(qm, i3);
                        TX[k] = fma2(dx, sj, TX[k]); TY[k] = fma2(dy, sj, TY[k]); TZ[k] = fma2(dz, sj, TZ[k]);
                        if (!diag) {
                            const float2 si = mul2(MI[k], i3);
                            tx = fma2(dx, si, tx); ty = fma2(dy, si, ty); tz = fma2(dz, si, tz);
                        }
                    }
                    vx[u] = tx.x + tx.y;
                    vy[u] = ty.x + ty.y;
                    vz[u] = tz.x + tz.y;
                }
                if (!diag) {
                    reduce_lanes(vx, lane);
                    reduce_lanes(vy, lane);
                    reduce_lanes(vz, lane);
                    if ((lane & 3) == 0) {
                        const int u = u0 + ((lane >> 2) & (kEnsJB - 1));
                        js[warp][u][0] = vx[0];
                        js[warp][u][1] = vy[0];
                        js[warp][u][2] = vz[0];
                    }
                }
            }
            if (!diag) {  // this round's column sums over the task's rows, into the column slots
                __syncthreads();
                const int lc0 = static_cast<int>(jb - c0) + j0;
                for (int e = threadIdx.x; e < jn; e += kEnsThreads)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        *slot(gb * kEnsGroup + lc0 + e, s_col, c) = (js[0][e][c] + js[1][e][c]) + (js[2][e][c] + js[3][e][c]);
                        if (COMP) *slot(gb * kEnsGroup + lc0 + e, s_col, 3 + c) = 0.0f;
                    }
                __syncthreads();
            }
        }
#pragma unroll
        for (int k = 0; k < P; ++k) {  // the stage's row partials into the running sums
            if (COMP) {
                fold(AX[k].x, CX[k].x, TX[k].x); fold(AX[k].y, CX[k].y, TX[k].y);
                fold(AY[k].x, CY[k].x, TY[k].x); fold(AY[k].y, CY[k].y, TY[k].y);
                fold(AZ[k].x, CZ[k].x, TZ[k].x); fold(AZ[k].y, CZ[k].y, TZ[k].y);
            } else {
                AX[k] = add2(AX[k], TX[k]); AY[k] = add2(AY[k], TY[k]); AZ[k] = add2(AZ[k], TZ[k]);
            }
        }
    });
    if (!ok) return false;
#pragma unroll
    for (int k = 0; k < P; ++k)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int o = threadIdx.x + (2 * k + h) * kEnsThreads;
            if (o >= rn) continue;
            const int l = ga * kEnsGroup + o;
            *slot(l, s_row, 0) = h ? AX[k].y : AX[k].x;
            *slot(l, s_row, 1) = h ? AY[k].y : AY[k].x;
            *slot(l, s_row, 2) = h ? AZ[k].y : AZ[k].x;
            if (COMP) {
                *slot(l, s_row, 3) = h ? CX[k].y : CX[k].x;
                *slot(l, s_row, 4) = h ? CY[k].y : CY[k].x;
                *slot(l, s_row, 5) = h ? CZ[k].y : CZ[k].x;
            }
        }
    return true;
}

// the raw gravity sum of particle i (local index l of simulation `sim`): its G + 1 slots in FP64, in order
template <bool COMP>
__device__ __forceinline__ void gsym_fold(const EnsView& v, int sim, int4 sm, int64_t i, float (&g)[3]) {
    constexpr int K = COMP ? 6 : 3;
    const float* part = sim_slots(v, sim);
    const int64_t N = sm.y, l = i - sm.x;
    double t[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s <= sm.w; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            t[c] += static_cast<double>(__ldcg(part + (static_cast<int64_t>(s) * K + c) * N + l));
            if (COMP) t[c] += static_cast<double>(__ldcg(part + (static_cast<int64_t>(s) * K + 3 + c) * N + l));
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c] = static_cast<float>(t[c]);
}

// ---- SPH: the neighbour lists, then the per-particle epilogue --------------------------------------
template <int GRAV, int PASS, bool SOLIDS, bool COMP, bool SYM>
__device__ __forceinline__ void sph_item(const DevArrays& a, const DevParams& p, const EnsView& v, int4 grp, int4 sm) {
    constexpr bool DO_A = PASS != PASS_VGRAD;
    const float4 zero = make_float4(0, 0, 0, 0);
    const uint32_t span = __float_as_uint(p.H2);
    for (int k = 0; k < kEnsIpt; ++k) {
        const int o = threadIdx.x + k * kEnsThreads;
        if (o >= grp.z) break;
        const int64_t i = static_cast<int64_t>(grp.y) + o;
        const ISph I = load_isph<PASS, SOLIDS>(a, p, i, 0.0f);
        PairAcc T;
#pragma unroll
        for (int f = 0; f < F_COUNT; ++f) T.f[f] = 0.0f;
        float maxv = 0.0f;
        // the neighbour list, or every particle of the simulation when the list overflowed (same j order)
        const int cnt = v.nbcnt[i];
        const bool over = cnt > kEnsCap;
        const int64_t len = over ? static_cast<int64_t>(sm.y) : cnt;
        for (int64_t m = 0; m < len; ++m) {
            const int64_t j = over ? static_cast<int64_t>(sm.x) + m : v.nb[m * v.n + i];
            const float4 q = __ldcg(a.posm + j);
            const float dx = q.x - I.pi.x, dy = q.y - I.pi.y, dz = q.z - I.pi.z;
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if (!in_open_closed(r2, 0u, span)) continue;
            const float4 vj = __ldcg(a.velrho + j);
            const float4 ja = DO_A ? __ldcg(a.jA + j) : zero, jb = DO_A ? __ldcg(a.jB + j) : zero;
            sph_neighbour<PASS, SOLIDS>(T, maxv, I, q.w, dx, dy, dz, r2, vj, ja, jb, p);
        }
        float g[3];
        if (SYM) {
            gsym_fold<COMP>(v, grp.x, sm, i, g);
        } else {
            const float4 gr = a.acc[i];
            g[0] = gr.x; g[1] = gr.y; g[2] = gr.z;
        }
        sph_finish<PASS, SOLIDS>(a, p, i, [&](int f) { return f == F_MAXV ? maxv : T.f[f]; }, GRAV != 0, g);
    }
}

template <int GRAV, bool SPH, int PASS, bool SOLIDS, bool COMP, bool SYM>
__global__ void __launch_bounds__(kEnsThreads) k_ensemble(DevArrays a, DevParams p, EnsView v) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item, s_flag;
    __shared__ float s_box[6 * (kEnsThreads / 32) + 12];  // reduction scratch, group box, tile box
    __shared__ float s_js[SYM ? kEnsThreads / 32 : 1][kEnsJC][3];  // GSYM: per-warp column sums of a round
    RangePipe pipe;
    pipe.buf = reinterpret_cast<float4*>(smem_raw);
    pipe.tile = v.tile;
    pipe.bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * static_cast<size_t>(v.tile) * sizeof(float4));
    pipe.src = a.posm;
    pipe.status = a.status;
    pipe.init();
    const int total = v.ntasks + v.ngroups * v.nstages;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(v.head, 1);
        __syncthreads();
        const int q0 = s_item;
        __syncthreads();
        if (q0 >= total) break;
        if (q0 < v.ntasks) {  // GSYM: a pair of groups of one simulation
            if (SYM && GRAV != 0 && SPH) {
                const int4 task = v.tasks[q0];
                if (!gsym_item<GRAV, COMP>(a, p, v, pipe, task, v.sims[task.x], s_js)) return;
                signal_done(v.done + 2 * v.nsims + task.x);
            }
            continue;
        }
        const int q = q0 - v.ntasks;
        const int si = q / v.ngroups;  // (branches, not an index: keeps the parameter block out of local memory)
        const int stage = si == 0 ? v.stages[0] : (si == 1 ? v.stages[1] : v.stages[2]);
        const int4 grp = v.groups[q % v.ngroups];
        const int sim = grp.x;
        const int4 sm = v.sims[sim];
        if (stage == ST_DENS) {
            const bool ok = SYM ? dens_item<0, SPH, COMP>(a, p, v, pipe, grp, sm, s_box)
                                : dens_item<GRAV, SPH, COMP>(a, p, v, pipe, grp, sm, s_box);
            if (!ok) return;
            signal_done(v.done + sim);
        } else if (stage == ST_SPH) {
            if (!wait_count(v.done + sim, sm.w + (sim == v.stall_sim ? 1 : 0), a.status, &s_flag)) return;
            if (SYM && !wait_count(v.done + 2 * v.nsims + sim, sm.w * (sm.w + 1) / 2, a.status, &s_flag)) return;
            sph_item<GRAV, PASS, SOLIDS, COMP, SYM>(a, p, v, grp, sm);
            signal_done(v.done + v.nsims + sim);
        } else {
            if (v.kick_dep >= 0 && !wait_count(v.done + v.kick_dep * v.nsims + sim, sm.w, a.status, &s_flag)) return;
            for (int k = 0; k < kEnsIpt; ++k) {
                const int o = threadIdx.x + k * kEnsThreads;
                if (o < grp.z) kick_drift(a, p, static_cast<int64_t>(grp.y) + o, v.kick_dt, p.fixed_dt);
            }
        }
    }
}

// ---- per-simulation FP64 diagnostics ---------------------------------------------------------------
__device__ __forceinline__ double block_sum(double x, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = x;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) r += sh[w];
    return r;
}

// one block per group: its particles' terms and their share of the pair potential against later
// particles of the same simulation
__global__ void __launch_bounds__(kEnsThreads) k_ens_diag(DevArrays a, DevParams p, EnsView v, double half_kick,
                                                       double* part) {
    __shared__ double tile[4][kEnsThreads];
    __shared__ double red[32];
    const int4 grp = v.groups[blockIdx.x];
    const int4 sm = v.sims[grp.x];
    const int64_t s1 = static_cast<int64_t>(sm.x) + sm.y;
    const int64_t np = a.n_pad;
    double f[kEnsDiagF];
#pragma unroll
    for (int k = 0; k < kEnsDiagF; ++k) f[k] = 0.0;
    double xi[kEnsIpt], yi[kEnsIpt], zi[kEnsIpt], mi[kEnsIpt], phi[kEnsIpt];
    int64_t ii[kEnsIpt];
#pragma unroll
    for (int k = 0; k < kEnsIpt; ++k) {
        const int o = threadIdx.x + k * kEnsThreads;
        ii[k] = o < grp.z ? static_cast<int64_t>(grp.y) + o : -1;
        xi[k] = yi[k] = zi[k] = mi[k] = phi[k] = 0.0;
        if (ii[k] >= 0) {
            double t[kEnsDiagF];
#pragma unroll
            for (int c = 0; c < kEnsDiagF; ++c) t[c] = 0.0;
            diag_terms(a, p, ii[k], half_kick, t);
#pragma unroll
            for (int c = 0; c < kEnsDiagF; ++c) f[c] += t[c];
            xi[k] = a.pos64[ii[k]]; yi[k] = a.pos64[np + ii[k]]; zi[k] = a.pos64[2 * np + ii[k]];
            mi[k] = a.posm[ii[k]].w;
        }
    }
    if (has(p, GSPH_SELF_GRAVITY)) {
        const double eps2 = p.eps2_d;
        for (int64_t t0 = grp.y; t0 < s1; t0 += kEnsThreads) {
            const int64_t j = t0 + threadIdx.x;
            __syncthreads();
            if (j < s1) {
                tile[0][threadIdx.x] = a.pos64[j];
                tile[1][threadIdx.x] = a.pos64[np + j];
                tile[2][threadIdx.x] = a.pos64[2 * np + j];
                tile[3][threadIdx.x] = a.posm[j].w;
            }
            __syncthreads();
            const int cnt = static_cast<int>(lmin(kEnsThreads, s1 - t0));
#pragma unroll
            for (int k = 0; k < kEnsIpt; ++k) {
                if (ii[k] < 0) continue;
                for (int jj = 0; jj < cnt; ++jj) {
                    if (t0 + jj <= ii[k]) continue;
                    const double dx = tile[0][jj] - xi[k], dy = tile[1][jj] - yi[k], dz = tile[2][jj] - zi[k];
                    phi[k] += tile[3][jj] / sqrt(dx * dx + dy * dy + dz * dz + eps2);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kEnsIpt; ++k) f[1] -= p.G_d * mi[k] * phi[k];
    }
#pragma unroll
    for (int k = 0; k < kEnsDiagF; ++k) {
        const double s = block_sum(f[k], red);
        if (threadIdx.x == 0) part[static_cast<int64_t>(blockIdx.x) * kEnsDiagF + k] = s;
    }
}

// per simulation, its groups' partials in queue order
__global__ void k_ens_diag_reduce(EnsView v, const double* part, double* out) {
    const int k = threadIdx.x;
    if (k >= kEnsDiagF) return;
    const int4 sm = v.sims[blockIdx.x];
    double s = 0.0;
    for (int g = sm.z; g < sm.z + sm.w; ++g) s += part[static_cast<int64_t>(g) * kEnsDiagF + k];
    out[static_cast<int64_t>(blockIdx.x) * kEnsDiagF + k] = s;
}

// ---- per-simulation curve order -------------------------------------------------------------------
// bounds of each simulation's positions (one block per simulation): bbox[s] = lo xyz, hi xyz
__global__ void k_ens_bbox(DevArrays a, EnsView v, float* bbox) {
    __shared__ float red[6][32];
    const int4 sm = v.sims[blockIdx.x];
    float r[6] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};  // min x y z, -max x y z
    for (int64_t i = static_cast<int64_t>(sm.x) + threadIdx.x; i < static_cast<int64_t>(sm.x) + sm.y; i += blockDim.x) {
        const float4 p = a.posm[i];
        const float c[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (isfinite(c[d])) {
                r[d] = fminf(r[d], c[d]);
                r[3 + d] = fminf(r[3 + d], -c[d]);
            }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 6; ++d) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r[d] = fminf(r[d], __shfl_xor_sync(0xffffffffu, r[d], o));
        if (lane == 0) red[d][warp] = r[d];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        float m = INFINITY;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fminf(m, red[threadIdx.x][w]);
        bbox[blockIdx.x * 8 + threadIdx.x] = threadIdx.x < 3 ? m : -m;
    }
}

// sort key of every slot: simulation index above the 30-bit Hilbert index of the position inside
// that simulation's bounds; padding sorts last
__global__ void k_ens_keys(DevArrays a, EnsView v, const float* bbox, unsigned long long* keys, int* vals) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n_pad) return;
    vals[i] = static_cast<int>(i);
    if (i >= a.n) {
        keys[i] = ~0ull;
        return;
    }
    int lo = 0, hi = v.nsims;  // sims[lo].x <= i < sims[hi].x (simulations are packed in index order)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (v.sims[mid].x <= i) lo = mid;
        else hi = mid;
    }
    const float4 p = a.posm[i];
    const float c[3] = {p.x, p.y, p.z};
    unsigned q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float l = bbox[lo * 8 + d], span = bbox[lo * 8 + 3 + d] - l;
        float t = (span > 0.0f && isfinite(c[d])) ? (c[d] - l) / span : 0.0f;
        t = fminf(fmaxf(t, 0.0f), 1.0f);
        q[d] = static_cast<unsigned>(t * 1023.0f);
    }
    keys[i] = (static_cast<unsigned long long>(lo) << 32) | hilbert3(q[0], q[1], q[2]);
}

__global__ void k_ens_iota(int* v, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) v[i] = static_cast<int>(i);
}

size_t ens_smem(int tile) { return pipe_smem_bytes(1, tile); }

template <int GRAV, bool SPH, int PASS, bool SOLIDS, bool COMP>
cudaError_t launch_t(const DevArrays& a, const DevParams& p, const EnsView& v, int sm_count, int per_sm_cap,
                     cudaStream_t s) {
    // the symmetric-gravity form is its own instantiation (gravity + SPH only), so the one-sided
    // kernels keep their register budget
    auto kern = (SPH && GRAV != 0 && v.sym) ? k_ensemble<GRAV, SPH, PASS, SOLIDS, COMP, true>
                                            : k_ensemble<GRAV, SPH, PASS, SOLIDS, COMP, false>;
    const size_t smem = ens_smem(v.tile);
    cudaError_t e = cudaSuccess;
    if (smem > 48 * 1024) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kEnsThreads, smem);
    if (e != cudaSuccess) return e;
    per_sm = std::max(per_sm, 1);
    if (per_sm_cap > 0) per_sm = std::min(per_sm, per_sm_cap);
    const int total = v.ntasks + v.ngroups * v.nstages;
    const int grid = std::max(1, std::min(total, sm_count * per_sm));
    kern<<<grid, kEnsThreads, smem, s>>>(a, p, v);
    return cudaGetLastError();
}

template <int GRAV, bool SPH>
cudaError_t launch_g(const DevArrays& a, const DevParams& p, const EnsView& v, bool comp, int sm_count, int cap,
                     cudaStream_t s) {
    if (!SPH) {
        return comp ? launch_t<GRAV, false, PASS_ACC, false, true>(a, p, v, sm_count, cap, s)
                    : launch_t<GRAV, false, PASS_ACC, false, false>(a, p, v, sm_count, cap, s);
    }
    const bool solids = has(p, GSPH_SOLIDS);
    const bool vgrad = solids || has(p, GSPH_INTEGRATE_DENSITY);
    if (solids)
        return comp ? launch_t<GRAV, true, PASS_FUSED, true, true>(a, p, v, sm_count, cap, s)
                    : launch_t<GRAV, true, PASS_FUSED, true, false>(a, p, v, sm_count, cap, s);
    if (vgrad)
        return comp ? launch_t<GRAV, true, PASS_FUSED, false, true>(a, p, v, sm_count, cap, s)
                    : launch_t<GRAV, true, PASS_FUSED, false, false>(a, p, v, sm_count, cap, s);
    return comp ? launch_t<GRAV, true, PASS_ACC, false, true>(a, p, v, sm_count, cap, s)
                : launch_t<GRAV, true, PASS_ACC, false, false>(a, p, v, sm_count, cap, s);
}

cudaError_t launch_ensemble(const DevArrays& a, const DevParams& p, const EnsView& v, bool comp, int sm_count,
                            int cap, cudaStream_t s) {
    const bool sph = has(p, GSPH_SPH);
    if (!has(p, GSPH_SELF_GRAVITY))
        return sph ? launch_g<0, true>(a, p, v, comp, sm_count, cap, s) : launch_g<0, false>(a, p, v, comp, sm_count, cap, s);
    if (p.eps2 > 0.0f)
        return sph ? launch_g<1, true>(a, p, v, comp, sm_count, cap, s) : launch_g<1, false>(a, p, v, comp, sm_count, cap, s);
    return sph ? launch_g<2, true>(a, p, v, comp, sm_count, cap, s) : launch_g<2, false>(a, p, v, comp, sm_count, cap, s);
}

}  // namespace

// ================================================================================================
// C-ABI
// ================================================================================================
struct gsph_ensemble {
    gsph_params params{};
    gsph_options opt{};
    DevParams dp{};
    DevArrays a{};
    int device = 0, sm_count = 0;
    int nsims = 0, ngroups = 0;
    std::vector<int64_t> offsets;   // host: nsims + 1
    int4* groups = nullptr;         // device tables
    int4* sims = nullptr;
    int* counters = nullptr;        // [1 + 3 S]: queue head; finished DENS, SPH and GSYM items per simulation
    bool sym = false;               // symmetric gravity stage (GSYM) instead of gravity in the DENS sweep
    int ntasks = 0;
    int4* tasks = nullptr;          // GSYM tasks (sim, row group, column group, 0)
    long long* slot_base = nullptr; // [S] first float of each simulation's slots in gslot
    float* gslot = nullptr;
    int inject_stall = -1;          // failure-path test: stall this simulation's SPH items once
    int* nb = nullptr;
    int* nbcnt = nullptr;
    double* diag_part = nullptr;    // [G][kEnsDiagF]
    double* diag_out = nullptr;     // [S][kEnsDiagF]
    float* staging = nullptr;       // 9 n floats
    double* staging64 = nullptr;    // 3 n doubles
    // per-simulation curve order: device slot i holds the caller's row ext[i]
    int* ext = nullptr;
    int* order = nullptr;
    int* order_out = nullptr;
    unsigned long long* keys = nullptr;  // [2 n_pad]
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    float4* tmp4 = nullptr;
    double* tmp8 = nullptr;
    float* bbox = nullptr;               // [S][8]
    int steps_since_sort = 0;
    int tile = kEnsTile;   // DENS j-tile (autotuned)
    int per_sm_cap = 0;    // CTAs per SM of the persistent grid (0: as many as fit; autotuned)
    std::vector<void*> allocations;
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int64_t launches = 0;
    std::string err;
};

namespace {

int efail(gsph_ensemble* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    else set_global_error(msg);
    return code;
}
int ecuda(gsph_ensemble* e, cudaError_t c, const char* what) {
    return efail(e, GSPH_E_CUDA, std::string(what) + ": " + cudaGetErrorString(c));
}
#define ENS_CK(ens, call, what)                          \
    do {                                                 \
        cudaError_t c_ = (call);                         \
        if (c_ != cudaSuccess) return ecuda(ens, c_, what); \
    } while (0)

void* ens_alloc(gsph_ensemble* e, size_t bytes, cudaError_t& err) {
    if (err != cudaSuccess) return nullptr;
    void* p = nullptr;
    err = cudaMalloc(&p, std::max<size_t>(bytes, 16));
    if (err == cudaSuccess) {
        e->allocations.push_back(p);
        err = cudaMemset(p, 0, std::max<size_t>(bytes, 16));
    }
    return p;
}

void ens_release(gsph_ensemble* e) {
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
    if (e->capture_stream) cudaStreamDestroy(e->capture_stream);
    e->capture_stream = nullptr;
    for (void* p : e->allocations) cudaFree(p);
    e->allocations.clear();
}

EnsView view_of(const gsph_ensemble* e, const int* stages, int nstages) {
    EnsView v{};
    v.groups = e->groups;
    v.sims = e->sims;
    v.ngroups = e->ngroups;
    v.nsims = e->nsims;
    v.nstages = nstages;
    v.kick_dep = -1;
    for (int k = 0; k < nstages; ++k) {
        v.stages[k] = stages[k];
        if (stages[k] == ST_KICK && k > 0) v.kick_dep = stages[k - 1] == ST_SPH ? 1 : 0;
    }
    v.head = e->counters;
    v.done = e->counters + 1;
    v.nb = e->nb;
    v.nbcnt = e->nbcnt;
    v.n = e->a.n;
    v.kick_dt = e->dp.fixed_dt;
    v.tile = e->tile;
    v.stall_sim = -1;
    v.sym = e->sym ? 1 : 0;
    v.tasks = e->tasks;
    v.ntasks = 0;
    for (int k = 0; k < nstages; ++k)  // the GSYM tasks run with the DENS stage
        if (stages[k] == ST_DENS && e->sym) v.ntasks = e->ntasks;
    v.gslot = e->gslot;
    v.slot_base = e->slot_base;
    return v;
}

// one launch of the given stages (queue counters cleared first)
int run_stages(gsph_ensemble* e, const int* stages, int nstages, float kick_dt, cudaStream_t s) {
    EnsView v = view_of(e, stages, nstages);
    v.kick_dt = kick_dt;
    v.stall_sim = e->inject_stall;  // one-shot failure-path test hook
    e->inject_stall = -1;
    ENS_CK(e, cudaMemsetAsync(e->counters, 0, (1 + 3 * static_cast<size_t>(e->nsims)) * sizeof(int), s), "counter reset");
    ENS_CK(e, launch_ensemble(e->a, e->dp, v, e->opt.accum == GSPH_ACCUM_COMPENSATED, e->sm_count, e->per_sm_cap, s),
           "ensemble launch");
    e->launches += 1;
    return GSPH_OK;
}

int derivative_stages(const gsph_ensemble* e, int* st) {
    int n = 0;
    st[n++] = ST_DENS;
    if (e->params.flags & GSPH_SPH) st[n++] = ST_SPH;
    return n;
}

int ens_status(gsph_ensemble* e, cudaStream_t s) {
    int st = 0;
    ENS_CK(e, cudaMemcpyAsync(&st, e->a.status, sizeof(int), cudaMemcpyDeviceToHost, s), "status read");
    ENS_CK(e, cudaStreamSynchronize(s), "stream synchronize");
    if (st & GSPH_DEV_ERR_TIMEOUT) {  // report once: the state is incomplete, the context stays usable
        const int cleared = st & ~GSPH_DEV_ERR_TIMEOUT;
        ENS_CK(e, cudaMemcpyAsync(e->a.status, &cleared, sizeof(int), cudaMemcpyHostToDevice, s), "status clear");
        ENS_CK(e, cudaStreamSynchronize(s), "stream synchronize");
        return efail(e, GSPH_E_TIMEOUT, "a device-side wait gave up (ensemble queue); the results of this call are "
                                        "incomplete");
    }
    return GSPH_OK;
}

// sort every simulation's particles along its own Hilbert curve (positions as they are now)
int ens_reorder(gsph_ensemble* e, cudaStream_t s) {
    const int st[1] = {ST_DENS};
    const EnsView v = view_of(e, st, 1);
    const int64_t np = e->a.n_pad;
    k_ens_bbox<<<e->nsims, 256, 0, s>>>(e->a, v, e->bbox);
    k_ens_keys<<<static_cast<unsigned>((np + 255) / 256), 256, 0, s>>>(e->a, v, e->bbox, e->keys, e->order);
    ENS_CK(e, cudaGetLastError(), "sort keys");
    e->launches += 2;
    int end_bit = 33;
    while ((int64_t(1) << (end_bit - 32)) < e->nsims) ++end_bit;
    size_t tb = e->sort_bytes;
    ENS_CK(e, cub::DeviceRadixSort::SortPairs(e->sort_tmp, tb, e->keys, e->keys + np, e->order, e->order_out,
                                              static_cast<int>(np), 0, end_bit, s), "radix sort");
    e->launches += 4;
    int launches = 0;
    ENS_CK(e, permute_particles(e->a, e->order_out, e->tmp4, e->tmp8, e->ext, s, launches), "permute");
    e->launches += launches;
    e->steps_since_sort = 0;
    return GSPH_OK;
}

}  // namespace

extern "C" {

int gsph_ensemble_create(const gsph_params* p, const gsph_options* opt, int32_t nsims, const int64_t* counts,
                         gsph_ensemble** out) {
    if (!out) return efail(nullptr, GSPH_E_INVALID, "out is NULL");
    *out = nullptr;
    char why[160];
    const int vr = gsph_params_validate(p, why, sizeof why);
    if (vr != GSPH_OK) return efail(nullptr, vr, why);
    if (nsims < 1 || !counts) return efail(nullptr, GSPH_E_INVALID, "nsims must be >= 1 and counts non-NULL");
    if (p->flags & GSPH_VARIABLE_TIMESTEP)
        return efail(nullptr, GSPH_E_UNSUPPORTED, "ensembles use the fixed time step (VARIABLE_TIMESTEP is off)");
    if (p->flags & GSPH_BALSARA_SWITCH)
        return efail(nullptr, GSPH_E_UNSUPPORTED, "ensembles do not support BALSARA_SWITCH");
    gsph_options o;
    if (opt) o = *opt;
    else gsph_options_defaults(&o);
    if (o.accum != GSPH_ACCUM_PLAIN && o.accum != GSPH_ACCUM_COMPENSATED)
        return efail(nullptr, GSPH_E_INVALID, "options.accum must be GSPH_ACCUM_PLAIN or GSPH_ACCUM_COMPENSATED");
    if (o.precision != GSPH_PRECISION_SINGLE)
        return efail(nullptr, GSPH_E_UNSUPPORTED, "ensembles run in single precision");
    int64_t total = 0;
    for (int s = 0; s < nsims; ++s) {
        if (counts[s] < 1) return efail(nullptr, GSPH_E_INVALID, "every simulation needs at least one particle");
        total += counts[s];
        if (total >= (int64_t(1) << 31) / kEnsCap)
            return efail(nullptr, GSPH_E_INVALID, "ensemble too large (total particles x 256 list slots >= 2^31)");
    }

    gsph_ensemble* e = new (std::nothrow) gsph_ensemble();
    if (!e) return efail(nullptr, GSPH_E_NOMEM, "host allocation failed");
    e->params = *p;
    e->opt = o;
    e->dp = gsph_dev_params(*p);
    e->nsims = nsims;
    cudaError_t ce = cudaGetDevice(&e->device);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, e->device);
    if (ce != cudaSuccess) {
        delete e;
        return efail(nullptr, GSPH_E_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(ce));
    }
    // host tables: packed offsets; groups of kEnsGroup particles, simulations largest first
    e->offsets.assign(nsims + 1, 0);
    for (int s = 0; s < nsims; ++s) e->offsets[s + 1] = e->offsets[s] + counts[s];
    std::vector<int> order(nsims);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return counts[x] > counts[y]; });
    std::vector<int4> groups, sims(nsims);
    for (int s : order) {
        const int first = static_cast<int>(groups.size());
        for (int64_t g = 0; g < counts[s]; g += kEnsGroup)
            groups.push_back(make_int4(s, static_cast<int>(e->offsets[s] + g),
                                       static_cast<int>(std::min<int64_t>(kEnsGroup, counts[s] - g)), 0));
        sims[s] = make_int4(static_cast<int>(e->offsets[s]), static_cast<int>(counts[s]), first,
                            static_cast<int>(groups.size()) - first);
    }
    e->ngroups = static_cast<int>(groups.size());
    // symmetric gravity (GSYM) for gravity + SPH ensembles when asked for (the default is the one-sided
    // sweep fused with the density pass, faster on ensembles of 1k..32k-particle simulations: 45.2 vs 51.6 ms
    // per step on 512 of them, 4.63M particles): tasks (ga <= gb) of each simulation, simulations largest
    // first and in each the off-diagonal pairs before the (half-sized) diagonal ones; G + 1 slots of K
    // floats per particle
    e->sym = (p->flags & GSPH_SELF_GRAVITY) && (p->flags & GSPH_SPH) && o.gravity_form == GSPH_GRAVITY_SYMMETRIC;
    std::vector<int4> tasks;
    std::vector<long long> slot_base(nsims, 0);
    long long slot_floats = 0;
    if (e->sym) {
        const int K = o.accum == GSPH_ACCUM_COMPENSATED ? 6 : 3;
        for (int s : order) {
            const int G = sims[s].w;
            for (int ga = 0; ga < G; ++ga)
                for (int gb = ga + 1; gb < G; ++gb) tasks.push_back(make_int4(s, ga, gb, 0));
            for (int g = 0; g < G; ++g) tasks.push_back(make_int4(s, g, g, 0));
        }
        for (int s = 0; s < nsims; ++s) {
            slot_base[s] = slot_floats;
            slot_floats += static_cast<long long>(sims[s].w + 1) * K * counts[s];
        }
        e->ntasks = static_cast<int>(tasks.size());
    }

    const int64_t n = total, n_pad = (n + kPad - 1) / kPad * kPad;
    DevArrays& a = e->a;
    a.n = n;
    a.n_pad = n_pad;
    cudaError_t ae = cudaSuccess;
    auto F4 = [&]() { return static_cast<float4*>(ens_alloc(e, n_pad * sizeof(float4), ae)); };
    a.posm = F4(); a.velrho = F4(); a.acc = F4(); a.xvel = F4(); a.sA = F4(); a.sB = F4();
    a.dA = F4(); a.dB = F4(); a.jA = F4(); a.jB = F4();
    a.pos64 = static_cast<double*>(ens_alloc(e, 3 * n_pad * sizeof(double), ae));
    a.rhodot = static_cast<float*>(ens_alloc(e, n_pad * sizeof(float), ae));
    a.balsara = static_cast<float*>(ens_alloc(e, n_pad * sizeof(float), ae));
    a.dt_state = static_cast<float*>(ens_alloc(e, 4 * sizeof(float), ae));
    a.status = static_cast<int*>(ens_alloc(e, 4 * sizeof(int), ae));
    e->groups = static_cast<int4*>(ens_alloc(e, groups.size() * sizeof(int4), ae));
    e->sims = static_cast<int4*>(ens_alloc(e, sims.size() * sizeof(int4), ae));
    e->counters = static_cast<int*>(ens_alloc(e, (1 + 3 * static_cast<size_t>(nsims)) * sizeof(int), ae));
    if (e->sym) {
        e->tasks = static_cast<int4*>(ens_alloc(e, tasks.size() * sizeof(int4), ae));
        e->slot_base = static_cast<long long*>(ens_alloc(e, slot_base.size() * sizeof(long long), ae));
        e->gslot = static_cast<float*>(ens_alloc(e, static_cast<size_t>(slot_floats) * sizeof(float), ae));
    }
    if (p->flags & GSPH_SPH) {
        e->nb = static_cast<int*>(ens_alloc(e, static_cast<size_t>(kEnsCap) * n * sizeof(int), ae));
        e->nbcnt = static_cast<int*>(ens_alloc(e, n * sizeof(int), ae));
    }
    e->diag_part = static_cast<double*>(ens_alloc(e, groups.size() * kEnsDiagF * sizeof(double), ae));
    e->diag_out = static_cast<double*>(ens_alloc(e, static_cast<size_t>(nsims) * kEnsDiagF * sizeof(double), ae));
    e->staging = static_cast<float*>(ens_alloc(e, 9 * n * sizeof(float), ae));
    e->staging64 = static_cast<double*>(ens_alloc(e, 3 * n * sizeof(double), ae));
    e->ext = static_cast<int*>(ens_alloc(e, n_pad * sizeof(int), ae));
    e->order = static_cast<int*>(ens_alloc(e, n_pad * sizeof(int), ae));
    e->order_out = static_cast<int*>(ens_alloc(e, n_pad * sizeof(int), ae));
    e->keys = static_cast<unsigned long long*>(ens_alloc(e, 2 * n_pad * sizeof(unsigned long long), ae));
    cub::DeviceRadixSort::SortPairs(nullptr, e->sort_bytes, static_cast<const unsigned long long*>(nullptr),
                                    static_cast<unsigned long long*>(nullptr), static_cast<const int*>(nullptr),
                                    static_cast<int*>(nullptr), static_cast<int>(n_pad));
    e->sort_tmp = ens_alloc(e, e->sort_bytes, ae);
    e->tmp4 = static_cast<float4*>(ens_alloc(e, n_pad * sizeof(float4), ae));
    e->tmp8 = static_cast<double*>(ens_alloc(e, n_pad * sizeof(double), ae));
    e->bbox = static_cast<float*>(ens_alloc(e, static_cast<size_t>(nsims) * 8 * sizeof(float), ae));
    if (ae == cudaSuccess) ae = cudaMemcpy(e->groups, groups.data(), groups.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (ae == cudaSuccess) ae = cudaMemcpy(e->sims, sims.data(), sims.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (ae == cudaSuccess && e->sym)
        ae = cudaMemcpy(e->tasks, tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (ae == cudaSuccess && e->sym)
        ae = cudaMemcpy(e->slot_base, slot_base.data(), slot_base.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (ae == cudaSuccess) {  // status[1]: the dependency-wait bound in microseconds (0: the default)
        const int lim = std::max(0, o.wait_limit_us);
        ae = cudaMemcpy(a.status + 1, &lim, sizeof(int), cudaMemcpyHostToDevice);
    }
    if (ae == cudaSuccess) ae = launch_init_padding(a, 0);
    if (ae == cudaSuccess) {
        k_ens_iota<<<static_cast<unsigned>((n_pad + 255) / 256), 256>>>(e->ext, n_pad);
        ae = cudaGetLastError();
    }
    if (ae == cudaSuccess) ae = cudaDeviceSynchronize();
    if (ae != cudaSuccess) {
        const std::string msg = std::string("ensemble allocation failed: ") + cudaGetErrorString(ae);
        ens_release(e);
        delete e;
        return efail(nullptr, GSPH_E_NOMEM, msg);
    }
    *out = e;
    return GSPH_OK;
}

int gsph_ensemble_destroy(gsph_ensemble* e) {
    if (!e) return GSPH_E_INVALID;
    cudaDeviceSynchronize();
    ens_release(e);
    delete e;
    return GSPH_OK;
}

int gsph_ensemble_offsets(const gsph_ensemble* e, int64_t* offsets) {
    if (!e || !offsets) return efail(const_cast<gsph_ensemble*>(e), GSPH_E_INVALID, "NULL argument");
    std::memcpy(offsets, e->offsets.data(), e->offsets.size() * sizeof(int64_t));
    return GSPH_OK;
}

int gsph_ensemble_upload(gsph_ensemble* e, uint32_t mask, const gsph_host_particles* src, void* stream) {
    if (!e) return GSPH_E_INVALID;
    if (!src) return efail(e, GSPH_E_INVALID, "src is NULL");
    if (mask & ~GSPH_ALL_ATTRIBS) return efail(e, GSPH_E_INVALID, "unknown attribute bits in mask");
    const float* ptrs[11] = {src->pos, src->mass, src->vel, src->acc, src->balsara, src->xvel,
                             src->density, src->density_dt, src->dstress, src->dstress_dt, src->maxvsig};
    static const int comps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};
    for (int k = 0; k < 11; ++k)
        if ((mask >> k & 1u) && !ptrs[k]) return efail(e, GSPH_E_INVALID, "attribute pointer is NULL for a set mask bit");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (int k = 0; k < 11; ++k) {
        if (!(mask >> k & 1u)) continue;
        ENS_CK(e, cudaMemcpyAsync(e->staging, ptrs[k], comps[k] * e->a.n * sizeof(float), cudaMemcpyHostToDevice, s),
               "upload copy");
        ENS_CK(e, launch_pack(e->a, k, e->staging, e->ext, s), "upload pack");
        e->launches += 1;
    }
    if (mask & GSPH_POS) return ens_reorder(e, s);
    return GSPH_OK;
}

int gsph_ensemble_download(gsph_ensemble* e, uint32_t mask, gsph_host_particles* dst, void* stream) {
    if (!e) return GSPH_E_INVALID;
    if (!dst) return efail(e, GSPH_E_INVALID, "dst is NULL");
    if (mask & ~GSPH_ALL_ATTRIBS) return efail(e, GSPH_E_INVALID, "unknown attribute bits in mask");
    float* ptrs[11] = {dst->pos, dst->mass, dst->vel, dst->acc, dst->balsara, dst->xvel,
                       dst->density, dst->density_dt, dst->dstress, dst->dstress_dt, dst->maxvsig};
    static const int comps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};
    for (int k = 0; k < 11; ++k)
        if ((mask >> k & 1u) && !ptrs[k]) return efail(e, GSPH_E_INVALID, "attribute pointer is NULL for a set mask bit");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (int k = 0; k < 11; ++k) {
        if (!(mask >> k & 1u)) continue;
        ENS_CK(e, launch_unpack(e->a, k, e->staging, e->ext, s), "download unpack");
        e->launches += 1;
        ENS_CK(e, cudaMemcpyAsync(ptrs[k], e->staging, comps[k] * e->a.n * sizeof(float), cudaMemcpyDeviceToHost, s),
               "download copy");
    }
    return ens_status(e, s);
}

int gsph_ensemble_upload_pos64(gsph_ensemble* e, const double* pos, void* stream) {
    if (!e) return GSPH_E_INVALID;
    if (!pos) return efail(e, GSPH_E_INVALID, "pos is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    ENS_CK(e, cudaMemcpyAsync(e->staging64, pos, 3 * e->a.n * sizeof(double), cudaMemcpyHostToDevice, s), "upload copy");
    ENS_CK(e, launch_pack_pos64(e->a, e->staging64, e->ext, s), "upload pack");
    e->launches += 1;
    return GSPH_OK;
}

int gsph_ensemble_download_pos64(gsph_ensemble* e, double* pos, void* stream) {
    if (!e) return GSPH_E_INVALID;
    if (!pos) return efail(e, GSPH_E_INVALID, "pos is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    ENS_CK(e, launch_unpack_pos64(e->a, e->staging64, e->ext, s), "download unpack");
    e->launches += 1;
    ENS_CK(e, cudaMemcpyAsync(pos, e->staging64, 3 * e->a.n * sizeof(double), cudaMemcpyDeviceToHost, s), "download copy");
    return ens_status(e, s);
}

int gsph_ensemble_compute_derivatives(gsph_ensemble* e, void* stream) {
    if (!e) return GSPH_E_INVALID;
    int st[3];
    const int ns = derivative_stages(e, st);
    return run_stages(e, st, ns, e->dp.fixed_dt, reinterpret_cast<cudaStream_t>(stream));
}

int gsph_ensemble_integrate(gsph_ensemble* e, int32_t not_first_step, void* stream) {
    if (!e) return GSPH_E_INVALID;
    const int st[1] = {ST_KICK};
    const float kick = not_first_step ? e->dp.fixed_dt : 0.5f * e->dp.fixed_dt;  // fixedTsLeapfrog (integration.h:90-93)
    return run_stages(e, st, 1, kick, reinterpret_cast<cudaStream_t>(stream));
}

int gsph_ensemble_step(gsph_ensemble* e, int32_t nsteps, void* stream) {
    if (!e) return GSPH_E_INVALID;
    if (nsteps < 0) return efail(e, GSPH_E_INVALID, "nsteps < 0");
    if (nsteps == 0) return GSPH_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!e->graph_exec) {  // one launch per substep: counter reset + all three stages, captured once
        if (!e->capture_stream)
            ENS_CK(e, cudaStreamCreateWithFlags(&e->capture_stream, cudaStreamNonBlocking), "stream");
        int st[3];
        int ns = derivative_stages(e, st);
        st[ns++] = ST_KICK;
        const int64_t before = e->launches;
        ENS_CK(e, cudaStreamBeginCapture(e->capture_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        const int rc = run_stages(e, st, ns, e->dp.fixed_dt, e->capture_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(e->capture_stream, &g);
        e->launches = before;
        if (rc != GSPH_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ee != cudaSuccess) return ecuda(e, ee, "end capture");
        cudaGraphExec_t ex = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
        if (ie != cudaSuccess) {
            cudaGraphDestroy(g);
            return ecuda(e, ie, "graph instantiate");
        }
        e->graph = g;
        e->graph_exec = ex;
    }
    for (int32_t k = 0; k < nsteps; ++k) {
        if (e->opt.resort_interval > 0 && e->steps_since_sort >= e->opt.resort_interval) {
            const int rc = ens_reorder(e, s);  // permutes in place: the graph's pointers stay valid
            if (rc != GSPH_OK) return rc;
        }
        ENS_CK(e, cudaGraphLaunch(e->graph_exec, s), "graph launch");
        e->launches += 1;
        e->steps_since_sort += 1;
    }
    return GSPH_OK;
}

int gsph_ensemble_diagnostics(gsph_ensemble* e, double half_kick, gsph_diag* out, void* stream) {
    if (!e) return GSPH_E_INVALID;
    if (!out) return efail(e, GSPH_E_INVALID, "out is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int st[1] = {ST_DENS};
    const EnsView v = view_of(e, st, 1);
    k_ens_diag<<<e->ngroups, kEnsThreads, 0, s>>>(e->a, e->dp, v, half_kick, e->diag_part);
    ENS_CK(e, cudaGetLastError(), "diagnostics");
    k_ens_diag_reduce<<<e->nsims, 32, 0, s>>>(v, e->diag_part, e->diag_out);
    ENS_CK(e, cudaGetLastError(), "diagnostics reduce");
    e->launches += 2;
    std::vector<double> h(static_cast<size_t>(e->nsims) * kEnsDiagF);
    ENS_CK(e, cudaMemcpyAsync(h.data(), e->diag_out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s),
           "diagnostics read");
    const int rc = ens_status(e, s);
    if (rc != GSPH_OK) return rc;
    for (int k = 0; k < e->nsims; ++k) {
        const double* d = h.data() + static_cast<size_t>(k) * kEnsDiagF;
        gsph_diag& o = out[k];
        o.e_kin = d[0];
        o.e_grav = d[1];
        o.e_int = d[2];
        o.e_shear = d[3];
        for (int c = 0; c < 3; ++c) {
            o.momentum[c] = d[4 + c];
            o.ang_mom[c] = d[7 + c];
        }
        o.mass = d[10];
    }
    return GSPH_OK;
}

int gsph_ensemble_autotune(gsph_ensemble* e, int32_t reps, int32_t* tile, int32_t* per_sm, void* stream) {
    if (!e) return GSPH_E_INVALID;
    if (reps < 1) reps = 2;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int st[3];
    const int ns = derivative_stages(e, st);  // derivatives only: the state is left as it was
    cudaEvent_t e0, e1;
    ENS_CK(e, cudaEventCreate(&e0), "event");
    ENS_CK(e, cudaEventCreate(&e1), "event");
    float best = 1e30f;
    int bt = e->tile, bp = e->per_sm_cap;
    int rc = GSPH_OK;
    for (int t : {256, 512, 1024}) {
        for (int cap : {0, 2, 3, 4}) {
            e->tile = t;
            e->per_sm_cap = cap;
            std::vector<float> ms;
            for (int r = 0; r <= reps && rc == GSPH_OK; ++r) {
                cudaEventRecord(e0, s);
                rc = run_stages(e, st, ns, e->dp.fixed_dt, s);
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                float x = 0.0f;
                cudaEventElapsedTime(&x, e0, e1);
                if (r > 0) ms.push_back(x);
            }
            if (rc != GSPH_OK) break;
            std::sort(ms.begin(), ms.end());
            if (ms[ms.size() / 2] < best) {
                best = ms[ms.size() / 2];
                bt = t;
                bp = cap;
            }
        }
        if (rc != GSPH_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    e->tile = bt;
    e->per_sm_cap = bp;
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
    if (rc != GSPH_OK) return rc;
    if (tile) *tile = bt;
    if (per_sm) *per_sm = bp;
    return ens_status(e, s);
}

int gsph_ensemble_launch_count(const gsph_ensemble* e, int64_t* count) {
    if (!e || !count) return GSPH_E_INVALID;
    *count = e->launches;
    return GSPH_OK;
}

int gsph_ensemble_inject_stall(gsph_ensemble* e, int32_t sim) {
    if (!e) return GSPH_E_INVALID;
    if (sim < 0 || sim >= e->nsims) return efail(e, GSPH_E_INVALID, "sim out of range");
    e->inject_stall = sim;
    return GSPH_OK;
}

const char* gsph_ensemble_last_error(const gsph_ensemble* e) {
    if (e) return e->err.c_str();
    return gsph_last_error(nullptr);
}

}  // extern "C"
