// pairs.cuh -- the all-pairs j-tile engine shared by the density, velocity-gradient, acceleration
// and gravity kernels.
//
// Replaces the reference's tile loop detail::do_for_each_pair_fast_impl
// (src/particles/algorithms.h:270-309) with:
//   * a 2-D grid: blockIdx.x = block of i-particles, blockIdx.y = segment of j-tiles (j-split),
//     so small N still fills 148 SMs and large N has no tail wave; each (i-block, segment)
//     writes its partial sums, which a finish kernel adds up in a fixed order (deterministic);
//   * j-tiles of `jt` particles staged in shared memory by 1-D bulk copies (cp.async.bulk, no
//     multicast), double-buffered against the i-loop and completed on mbarriers;
//   * arrays padded to a multiple of kPad with inert particles (zero mass, far away), so every tile
//     is full and the reference's remainder-tile bug (algorithms.h:285-301) cannot arise.
#pragma once

#include "common.cuh"
#include "spatial.cuh"

namespace gsph {

// Two-stage pipeline over the j-tiles [t_begin, t_end) of up to 4 float4 streams.
template <int NS>
struct JTilePipe {
    float4* buf;          // shared: [2][NS][jt]
    uint64_t* bar;        // shared: [2]
    const float4* src[NS];
    int jt;
    int64_t t_begin, t_end;  // tiles t_begin .. t_end-1, or positions of `list` when it is set
    const int* list = nullptr;
    int* status;

    __device__ __forceinline__ int64_t tile_at(int64_t k) const { return list ? list[k] : k; }

    __device__ __forceinline__ void issue(int b, int64_t t) {
        mbar_expect_tx(&bar[b], static_cast<uint32_t>(NS * jt * sizeof(float4)));
#pragma unroll
        for (int s = 0; s < NS; ++s)
            bulk_g2s(buf + (static_cast<int64_t>(b) * NS + s) * jt, src[s] + t * jt,
                     static_cast<uint32_t>(jt * sizeof(float4)), &bar[b]);
    }

    // init barriers and start the first two tiles; all threads must call it
    __device__ __forceinline__ void start() {
        if (threadIdx.x == 0) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            fence_barrier_init();
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (t_begin < t_end) issue(0, tile_at(t_begin));
            if (t_begin + 1 < t_end) issue(1, tile_at(t_begin + 1));
        }
    }

    // for each tile: wait for it, run body(stage pointers), release the buffer and refill it
    template <typename Body>
    __device__ __forceinline__ void run(Body&& body) {
        int k = 0;
        for (int64_t t = t_begin; t < t_end; ++t, ++k) {
            const int b = k & 1;
            const bool ok = mbar_wait_bounded(&bar[b], static_cast<uint32_t>((k >> 1) & 1), status);
            if (__syncthreads_or(!ok)) {
                drain(k);
                return;
            }
            const float4* stage = buf + static_cast<int64_t>(b) * NS * jt;
            body(stage);
            __syncthreads();
            if (threadIdx.x == 0 && t + 2 < t_end) issue(b, tile_at(t + 2));
        }
    }

    // after a timed-out wait: give copies still in flight a bounded time to land before exit
    __device__ __forceinline__ void drain(int k) {
        if (threadIdx.x == 0) {
            for (int extra = 0; extra < 2; ++extra) {
                const int kk = k + extra;
                const int64_t t = t_begin + kk;
                if (t >= t_end) break;
                mbar_wait_bounded(&bar[kk & 1], static_cast<uint32_t>((kk >> 1) & 1), status);
            }
        }
        __syncthreads();
    }
};

// ---- culled passes: work items over the near-chunk lists ------------------------------------------
constexpr int kStageChunks = 4;  // chunks staged per pipeline stage (256 j-particles)
constexpr int kItemNb = 96;      // neighbour-list slots per lane and work item (density pass -> SPH passes)

// Work item w of the culled passes: i-group g, positions [c0, c1) of g's near-chunk list. Items are
// numbered group by group (item_start[g] .. item_start[g+1]-1), at most item_chunks chunks each.
struct CullView {
    const int* list;
    const int* count;
    const int* item_start;  // [ngroups + 2]: first item of each group, the number of items, the
                            // chunks per item (chosen on the device from the total near-chunk count)
    int ngroups;
    int64_t nchunks;        // row stride of `list`
    float* part;            // [item][field][kGroup]
    int* nb;                // nullable: per item, each lane's neighbour indices [item][kItemNb][kGroup] ...
    int* nbcnt;             // ... and their count [item][kGroup] (kItemNb + 1: the list overflowed) ...
    int* nbover;            // ... and per item whether any lane's list overflowed
    const float4* box_lo;   // per-chunk bounding boxes (the culled density pass skips, warp by warp, the
    const float4* box_hi;   // chunks of an item that are farther than h (1 + kMargin) from the warp's box)
    __device__ __forceinline__ int items() const { return item_start[ngroups]; }
    __device__ __forceinline__ void item(int w, int& g, int& c0, int& c1) const {
        int lo = 0, hi = ngroups;  // item_start[lo] <= w < item_start[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (item_start[mid] <= w) lo = mid;
            else hi = mid;
        }
        g = lo;
        const int ic = item_start[ngroups + 1];
        c0 = (w - item_start[g]) * ic;
        c1 = min(c0 + ic, count[g]);
    }
};

// Two-stage pipeline over a list of chunks, kStageChunks chunks per stage; the stage counter runs on
// across items so the mbarrier phases stay in step.
template <int NS>
struct ItemPipe {
    static constexpr int SJ = kStageChunks * kChunk;
    float4* buf;     // shared: [2][NS][SJ]
    uint64_t* bar;   // shared: [2]
    const float4* src[NS];
    int* status;
    uint32_t kst = 0;

    __device__ __forceinline__ void init() {
        if (threadIdx.x == 0) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            fence_barrier_init();
        }
        __syncthreads();
    }
    __device__ __forceinline__ void issue(int b, const int* chunks, int first, int nc) {
        mbar_expect_tx(&bar[b], static_cast<uint32_t>(NS * nc * kChunk * sizeof(float4)));
        for (int c = 0; c < nc; ++c) {
            const int64_t ch = chunks[first + c];
#pragma unroll
            for (int s = 0; s < NS; ++s)
                bulk_g2s(buf + (static_cast<int64_t>(b) * NS + s) * SJ + c * kChunk, src[s] + ch * kChunk,
                         static_cast<uint32_t>(kChunk * sizeof(float4)), &bar[b]);
        }
    }
    // body(stage, nj) for every stage of the n chunks chunks[0..n); false if a wait gave up
    template <typename Body>
    __device__ __forceinline__ bool run(const int* chunks, int n, Body&& body) {
        const int nst = (n + kStageChunks - 1) / kStageChunks;
        if (threadIdx.x == 0)
            for (int st = 0; st < 2 && st < nst; ++st)
                issue((kst + st) & 1, chunks, st * kStageChunks, min(kStageChunks, n - st * kStageChunks));
        for (int st = 0; st < nst; ++st) {
            const int b = kst & 1;
            const bool ok = mbar_wait_bounded(&bar[b], (kst >> 1) & 1, status);
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0 && st + 1 < nst)
                    mbar_wait_bounded(&bar[(kst + 1) & 1], ((kst + 1) >> 1) & 1, status);
                __syncthreads();
                return false;
            }
            const int nc = min(kStageChunks, n - st * kStageChunks);
            body(buf + static_cast<int64_t>(b) * NS * SJ, nc * kChunk);
            __syncthreads();
            if (threadIdx.x == 0 && st + 2 < nst)
                issue(b, chunks, (st + 2) * kStageChunks, min(kStageChunks, n - (st + 2) * kStageChunks));
            ++kst;
        }
        return true;
    }
};

// shared-memory bytes of a pipeline: 2 stages of NS streams plus the two barriers
__host__ __device__ inline size_t pipe_smem_bytes(int ns, int jt) {
    return static_cast<size_t>(2) * ns * jt * sizeof(float4) + 2 * sizeof(uint64_t);
}

// tile range of segment `seg` out of `nseg` over `ntiles` tiles (balanced to within one tile)
__device__ __forceinline__ void segment_tiles(int64_t ntiles, int seg, int nseg, int64_t& t0, int64_t& t1) {
    t0 = ntiles * seg / nseg;
    t1 = ntiles * (seg + 1) / nseg;
}

// ---- partial-sum fields of the SPH pair passes -----------------------------------------------
enum Field : int {
    F_GX = 0, F_GY, F_GZ,                    // gravity (G applied in the finish kernel)
    F_AX, F_AY, F_AZ,                        // stress + AV acceleration
    F_XV0, F_XV1, F_XV2,                     // XSPH
    F_E00, F_E11, F_E22, F_E01, F_E02, F_E12,  // strain rate (symmetric)
    F_W01, F_W02, F_W12,                     // rotation rate (antisymmetric)
    F_DIVV,                                  // velocity divergence
    F_C0, F_C1, F_C2,                        // velocity curl (fluid + Balsara)
    F_MAXV,                                  // max signal velocity (a max, not a sum)
    F_COUNT
};

enum Pass : int { PASS_VGRAD = 0, PASS_ACC = 1, PASS_FUSED = 2 };

template <int PASS, bool GRAV, bool SOLIDS>
__host__ __device__ constexpr uint32_t field_mask() {
    uint32_t m = 0;
    if (PASS != PASS_VGRAD) {
        m |= (1u << F_AX) | (1u << F_AY) | (1u << F_AZ) | (1u << F_XV0) | (1u << F_XV1) | (1u << F_XV2) |
             (1u << F_MAXV);
        if (GRAV) m |= (1u << F_GX) | (1u << F_GY) | (1u << F_GZ);
    }
    if (PASS != PASS_ACC) {
        m |= (1u << F_DIVV);
        if (SOLIDS)
            m |= (1u << F_E00) | (1u << F_E11) | (1u << F_E22) | (1u << F_E01) | (1u << F_E02) | (1u << F_E12) |
                 (1u << F_W01) | (1u << F_W02) | (1u << F_W12);
        else
            m |= (1u << F_C0) | (1u << F_C1) | (1u << F_C2);
    }
    return m;
}

__host__ __device__ constexpr int popc_c(uint32_t x) { return x == 0 ? 0 : int(x & 1u) + popc_c(x >> 1); }

template <uint32_t MASK>
__host__ __device__ constexpr int field_offset(int f) {
    return popc_c(MASK & ((1u << f) - 1u));
}

// Optional event pair bracketing one pair-kernel launch (per-kernel timing, graph-capturable).
struct KTimer {
    cudaEvent_t start = nullptr, stop = nullptr;
};
cudaError_t timer_record(cudaEvent_t ev, cudaStream_t s);

// host launchers (pairs.cu)
// How the finish kernels read a particle's gravity partials: segments 0 .. nseg-1 of the one-sided
// kernel ([segment][component][particle]), or (sym_G > 0) the symmetric kernel's G + 1 slots of the
// particle ([particle][slot][component]).
struct GravSum {
    int nseg = 0;
    int sym_G = 0;
};

struct Launch {
    bool cull;       // SPH passes over near-chunk lists (spatial.cuh) + separate all-pairs gravity
    int threads;     // threads per CTA of the SPH pair kernels
    int jt;          // j-tile
    int nseg;        // j-split of the SPH pair kernels
    int grav_threads;
    int grav_ipt;    // i per thread of the gravity kernel
    int grav_jt;     // j-tile of the gravity kernel
    bool grav_x2;    // paired FP32 (f32x2) form of the gravity kernel
    int grav_nseg;
    int grav_sym_G = 0;   // > 0: symmetric gravity kernel over G groups of grav_sym_gs blocks of 1024
    int grav_sym_gs = 0;
    int accum;       // GSPH_ACCUM_*
    int item_grid;   // persistent grid of the culled SPH kernel (its resident capacity)
    int density_grid;  // persistent grid of the culled density kernel
};

// the finish kernels' view of the gravity partials of launch shape L; nseg == 0: no gravity partials
inline GravSum grav_sum(const Launch& L, int nseg) {
    GravSum g;
    if (nseg <= 0) return g;
    if (L.grav_sym_G > 0) {
        g.sym_G = L.grav_sym_G;
    } else {
        g.nseg = nseg;
    }
    return g;
}
// the symmetric gravity kernel's group count for blocks of 1024 particles: groups of
// ceil(nblocks / target) blocks
inline void sym_groups(int64_t nblocks, int target, int& G, int& gs) {
    gs = static_cast<int>((nblocks + target - 1) / target);
    if (gs < 1) gs = 1;
    G = static_cast<int>((nblocks + gs - 1) / gs);
}

// With `sp`, the culled density pass also stores every lane's neighbour indices per work item
// (sp->item_nb), which the SPH passes of the same step then use instead of scanning the chunks again.
cudaError_t launch_density(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s,
                           const KTimer* t = nullptr, const SpatialArrays* sp = nullptr);
// near-chunk work items of the culled passes (item_start scan); needs launch_chunk_lists first.
// `target` items in total (plus at most one per group for rounding).
cudaError_t launch_work_items(const DevArrays& a, const SpatialArrays& sp, int target, cudaStream_t s);
cudaError_t launch_prepare(const DevArrays& a, const DevParams& p, cudaStream_t s);
// With `sp`, the SPH terms come from the near-chunk work items; the finish kernel then adds `gnseg`
// segments of gravity partials (a.gpart, from launch_gravity_partials), after waiting for `join`
// when it is given (the gravity kernel may run on another stream).
cudaError_t launch_pairs(int pass, const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s,
                         const KTimer* t = nullptr, const SpatialArrays* sp = nullptr, int gnseg = 0,
                         cudaEvent_t join = nullptr, bool lists = false);
cudaError_t launch_gravity_partials(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s,
                                    const KTimer* t = nullptr);
cudaError_t launch_gravity(const DevArrays& a, const DevParams& p, const Launch& L, cudaStream_t s,
                           const KTimer* t = nullptr);
cudaError_t launch_fp32_peak(int sm_count, int iters, float* sink, cudaStream_t s);
cudaError_t launch_gravity_raw(const float4* posm_padded, float* part, int64_t n_pad, int ipt, int jt, int nseg,
                               float eps2, int* status, cudaStream_t s);
int64_t fp32_peak_flops(int sm_count, int iters);
size_t partial_floats(const DevParams& p, const Launch& L, int64_t n_pad);
size_t gravity_partial_floats(const Launch& L, int64_t n_pad);
int gravity_blocks_per_sm(int ipt, int threads, int jt, bool comp);

}  // namespace gsph
