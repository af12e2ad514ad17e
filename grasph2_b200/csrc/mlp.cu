// mlp.cu -- the per-particle MLP of the learned surrogate on the tensor cores (tcgen05, BF16 operands,
// FP32 accumulation in tensor memory), and a tile-GEMM check of the operand encodings.
#include <cuda_bf16.h>

#include <cmath>
#include <new>
#include <string>

#include "umma.cuh"

void set_global_error(const std::string& msg);  // capi.cu

using namespace gsph;

namespace {

constexpr int kTileM = 128;  // rows (particles) per tile = tensor-memory lanes

// ---- tile GEMM check: D[128][N] = A[128][K] * B[N][K]^T --------------------------------------------
// A and B arrive row-major from global memory; a_mn / b_mn choose whether each is staged as a K-major
// operand (its rows) or as an MN-major operand (its transpose), so all four descriptor forms can be
// compared with a host product.
constexpr int kCheckSmem = 160 * 1024;
constexpr uint32_t kCheckB = 64 * 1024;  // byte offset of the B buffer

__global__ void __launch_bounds__(kTileM) k_tc_gemm_check(const __nv_bfloat16* __restrict__ A,
                                                          const __nv_bfloat16* __restrict__ B, float* __restrict__ D,
                                                          int N, int K, int a_mn, int b_mn, int* status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    unsigned char* sa = smem;
    unsigned char* sb = smem + kCheckB;
    for (int e = threadIdx.x; e < kTileM * K; e += blockDim.x) {
        const int m = e / K, k = e % K;
        const uint32_t o = a_mn ? umma::off(k, m, K) : umma::off(m, k, kTileM);
        *reinterpret_cast<__nv_bfloat16*>(sa + o) = A[e];
    }
    for (int e = threadIdx.x; e < N * K; e += blockDim.x) {
        const int n = e / K, k = e % K;
        const uint32_t o = b_mn ? umma::off(k, n, K) : umma::off(n, k, N);
        *reinterpret_cast<__nv_bfloat16*>(sb + o) = B[e];
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    umma::fence_smem_to_async();
    __syncthreads();
    if (threadIdx.x < 32) umma::tmem_alloc(&tslot, 256);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tbase = tslot;
    if (threadIdx.x == 0) {
        const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
        const uint32_t id = umma::idesc_bf16(kTileM, N, a_mn, b_mn);
        for (int s = 0; s < K / 16; ++s) {
            const uint64_t ad = a_mn ? umma::desc_mnmajor(a0, K, s) : umma::desc_kmajor(a0, kTileM, s);
            const uint64_t bd = b_mn ? umma::desc_mnmajor(b0, K, s) : umma::desc_kmajor(b0, N, s);
            umma::mma_bf16(tbase, ad, bd, id, s > 0);
        }
        umma::commit(&bar);
    }
    const bool ok = __syncthreads_and(umma::wait_mma(&bar, 0, status));
    umma::fence_after();
    if (ok) {
        for (int c = 0; c < N; c += 16) {
            float v[16];
            umma::ld16(umma::lane_addr(tbase, c), v);
#pragma unroll
            for (int k = 0; k < 16; ++k) D[threadIdx.x * N + c + k] = v[k];
        }
    }
    umma::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) umma::tmem_free(tbase, 256);
}

// ================================================================================================
// the surrogate's MLP: 32 -> 128 -> 128 -> 128 -> 13, SiLU, BF16 operands, FP32 accumulation
// ================================================================================================
constexpr int kIn = 32, kHid = 128, kOut = 13, kOutP = 16;
// flat FP32 parameter vector: W1[128][32] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] W4[13][128] b4[13]
constexpr int oW1 = 0, ob1 = oW1 + kHid * kIn, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid, oW3 = ob2 + kHid,
              ob3 = oW3 + kHid * kHid, oW4 = ob3 + kHid, ob4 = oW4 + kOut * kHid, kParams = ob4 + kOut;
// stride of the per-CTA gradient slices: a multiple of 4 floats, so the weight rows (which start at multiples
// of 4 within a slice) take 16-byte vector read-modify-writes
constexpr int kPartStride = (kParams + 3) & ~3;
static_assert(oW2 % 4 == 0 && oW3 % 4 == 0 && ob1 % 4 == 0 && ob2 % 4 == 0 && ob3 % 4 == 0 && kIn % 4 == 0 &&
                  kHid % 4 == 0, "vector gradient rows");
// packed BF16 weights (W4 padded to 16 rows) and FP32 biases (b4 padded to 16)
constexpr int qW1 = 0, qW2 = qW1 + kHid * kIn, qW3 = qW2 + kHid * kHid, qW4 = qW3 + kHid * kHid,
              kPacked = qW4 + kOutP * kHid;
constexpr int kBias = 3 * kHid + kOutP;

// shared-memory map (bytes)
constexpr uint32_t sW1 = 0, sW2 = sW1 + kHid * kIn * 2, sW3 = sW2 + kHid * kHid * 2, sW4 = sW3 + kHid * kHid * 2,
                   sX = sW4 + kOutP * kHid * 2, sH1 = sX + kTileM * kIn * 2;
// inference: per tile slot one buffer, holding the tile's inputs until the first layer's MMAs have read
// them and then its activations
constexpr int kSlots = 4;
constexpr uint32_t kSlotBytes = kTileM * kHid * 2;
constexpr uint32_t sBiasF = sX + kSlots * kSlotBytes, kFwdSmem = sBiasF + kBias * 4;
static_assert(kFwdSmem <= 227 * 1024, "forward kernel shared memory");
// training: three activation buffers, the output gradient, the layer gradient, a block of ones
constexpr uint32_t sH2 = sH1 + kTileM * kHid * 2, sH3 = sH2 + kTileM * kHid * 2, sG4 = sH3 + kTileM * kHid * 2,
                   sG = sG4 + kTileM * kOutP * 2, sOnes = sG + kTileM * kHid * 2, sBiasT = sOnes + kTileM * 16 * 2,
                   kTrainSmem = sBiasT + kBias * 4;
static_assert(kTrainSmem <= 227 * 1024, "training kernel shared memory");

// SiLU through one hardware tanh (tanh.approx.f32, PTX ISA 7.0; relative error about 2^-11, below the
// bf16 rounding of the activations): z sigmoid(z) = u + u tanh(u) with u = z / 2, and
// d/dz [z sigmoid(z)] = s (1 + z (1 - s)) with s = sigmoid(z) = 1/2 + tanh(u) / 2
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu(float z) {
    const float u = 0.5f * z;
    return fmaf(u, tanh_hw(u), u);
}
__device__ __forceinline__ float dsilu(float z) {
    const float s = fmaf(0.5f, tanh_hw(0.5f * z), 0.5f);
    return s * fmaf(z, 1.0f - s, 1.0f);
}

// named CTA barrier `id` over `n` threads (a multiple of 32), and the same with an AND over a predicate
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ bool named_and(int id, int n, bool v) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.and.pred p, %2, %3, q;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(r)
        : "r"(v ? 1u : 0u), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// stage the packed weights (row-major bf16) into the core-matrix layout, biases as FP32
__device__ void stage_weights(unsigned char* sm, const __nv_bfloat16* __restrict__ wq, const float* __restrict__ bq,
                              float* sbias) {
    struct M { uint32_t s; int q, R, C; };
    const M mats[4] = {{sW1, qW1, kHid, kIn}, {sW2, qW2, kHid, kHid}, {sW3, qW3, kHid, kHid}, {sW4, qW4, kOutP, kHid}};
    for (int m = 0; m < 4; ++m) {
        const int R = mats[m].R, C = mats[m].C;
        for (int e = threadIdx.x; e < R * C / 8; e += blockDim.x) {  // 8 consecutive columns per move
            const int r = e / (C / 8), c0 = (e % (C / 8)) * 8;
            *reinterpret_cast<uint4*>(sm + mats[m].s + umma::off(r, c0, R)) =
                *reinterpret_cast<const uint4*>(wq + mats[m].q + r * C + c0);
        }
    }
    for (int e = threadIdx.x; e < kBias; e += blockDim.x) sbias[e] = bq[e];
}

// one row of features (32 FP32) -> bf16 row t of the X buffer; zeros past the end
__device__ __forceinline__ void load_x(unsigned char* sm, const float* __restrict__ x, int64_t p, int64_t n) {
    float v[kIn];
    if (p < n) {
        const float4* src = reinterpret_cast<const float4*>(x + p * kIn);
#pragma unroll
        for (int k = 0; k < kIn / 4; ++k) {
            const float4 q = src[k];
            v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kIn; ++k) v[k] = 0.0f;
    }
#pragma unroll
    for (int c = 0; c < kIn; c += 8) umma::st8(sm + sX, threadIdx.x, c, kTileM, v + c);
}

// thread 0: D(tD) = A * B^T, operands in shared memory (K-major: buffer rows = M/N; MN-major: buffer
// rows = K), K in steps of 16
__device__ __forceinline__ void issue(uint32_t tD, uint32_t a0, int aR, bool a_mn, uint32_t b0, int bR, bool b_mn,
                                      int N, int K) {
    const uint32_t id = umma::idesc_bf16(kTileM, N, a_mn, b_mn);
    for (int s = 0; s < K / 16; ++s)
        umma::mma_bf16(tD, a_mn ? umma::desc_mnmajor(a0, aR, s) : umma::desc_kmajor(a0, aR, s),
                       b_mn ? umma::desc_mnmajor(b0, bR, s) : umma::desc_kmajor(b0, bR, s), id, s > 0);
}
// D(tD)[128][N] = ones[128][K] * B^T: every row holds the column sums of B over K (bias gradients)
__device__ __forceinline__ void issue_colsum(uint32_t tD, uint32_t ones, uint32_t b0, int bR, int N, int K) {
    const uint32_t id = umma::idesc_bf16(kTileM, N, false, true);
    for (int s = 0; s < K / 16; ++s)
        umma::mma_bf16(tD, umma::desc_kmajor(ones, kTileM, 0), umma::desc_mnmajor(b0, bR, s), id, s > 0);
}
// every thread: shared-memory writes and earlier tensor-memory reads are ordered before the MMAs that
// thread 0 issues next
__device__ __forceinline__ void before_issue() {
    umma::fence_smem_to_async();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
}
// every thread: wait for the MMAs of the last commit; uniform result
__device__ __forceinline__ bool after_commit(uint64_t* bar, uint32_t& phase, int* status) {
    const bool ok = __syncthreads_and(umma::wait_mma(bar, phase, status));
    phase ^= 1u;
    umma::fence_after();
    return ok;
}
// hidden-layer epilogue of row t: h = SiLU(D + b) into the activation buffer at `buf`
__device__ __forceinline__ void hidden_out(uint32_t tD, const float* bias, unsigned char* buf) {
#pragma unroll 1
    for (int c0 = 0; c0 < kHid; c0 += 32) {
        float v[32];
        umma::ld32(umma::lane_addr(tD, c0), v);
#pragma unroll
        for (int k = 0; k < 32; ++k) v[k] = silu(v[k] + bias[c0 + k]);
#pragma unroll
        for (int k = 0; k < 32; k += 8) umma::st8(buf, threadIdx.x, c0 + k, kTileM, v + k);
    }
}

// Forward over tiles of 128 rows (persistent grid): y[n][13] = MLP(x[n][32]). A CTA runs four
// independent tile pipelines (slots) of one warpgroup each; a slot has its own buffer (inputs, then
// activations), 128 tensor-memory columns (all 512 in use), MMA barrier and named CTA barrier, so while
// one slot drains an accumulator (bias, SiLU, bf16 pack) the tensor cores run other slots' layers and
// their input loads are in flight. Slot s takes tiles 4 b + s, 4 (b + grid) + s, ... of CTA b. Thread t
// of a slot owns row t: warp w drains tensor-memory lanes 32 (w % 4) .. + 31, all columns.
constexpr int kSlotThreads = kTileM, kFwdThreads = kSlots * kSlotThreads;

__global__ void __launch_bounds__(kFwdThreads, 1) k_mlp_forward(const float* __restrict__ x, float* __restrict__ y,
                                                               int64_t n, const __nv_bfloat16* __restrict__ wq,
                                                               const float* __restrict__ bq, int* status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar[kSlots];
    __shared__ uint32_t tslot;
    float* sbias = reinterpret_cast<float*>(sm + sBiasF);
    stage_weights(sm, wq, bq, sbias);
    if (threadIdx.x == 0) {
        for (int k = 0; k < kSlots; ++k) mbar_init(&bar[k], 1);
        fence_barrier_init();
    }
    if (threadIdx.x < 32) umma::tmem_alloc(&tslot, 128 * kSlots);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const int slot = threadIdx.x / kSlotThreads, row = threadIdx.x % kSlotThreads;
    const int bid = 1 + slot;  // named barrier of the slot (0 is __syncthreads)
    const uint32_t T = tslot + 128 * slot;
    const uint32_t base = smem_u32(sm);
    const uint32_t xo = sX + slot * kSlotBytes, ho = xo;  // the inputs, then the activations
    uint64_t* mbar = &bar[slot];
    uint32_t phase = 0;
    // shared-memory writes and tensor-memory reads of the slot before the MMAs its first thread issues
    auto slot_sync = [&] {
        umma::fence_smem_to_async();
        umma::fence_before();
        named_sync(bid, kSlotThreads);
        umma::fence_after();
    };
    // every thread of the slot waits for the last commit; uniform result
    auto slot_wait = [&]() -> bool {
        const bool ok = named_and(bid, kSlotThreads, umma::wait_mma(mbar, phase, status));
        phase ^= 1u;
        umma::fence_after();
        return ok;
    };
    auto layer = [&](uint32_t a, uint32_t b, int N, int K) {
        slot_sync();
        if (row == 0) {
            issue(T, base + a, kTileM, false, base + b, N, false, N, K);
            umma::commit(mbar);
        }
        return slot_wait();
    };
    // hidden epilogue of this thread's row: h = SiLU(D + b)
    auto hidden = [&](const float* bias) {
#pragma unroll 1
        for (int c0 = 0; c0 < kHid; c0 += 32) {
            float v[32];
            umma::ld32(umma::lane_addr(T, c0), v);
#pragma unroll
            for (int k = 0; k < 32; ++k) v[k] = silu(v[k] + bias[c0 + k]);
#pragma unroll
            for (int k = 0; k < 32; k += 8) umma::st8(sm + ho, row, c0 + k, kTileM, v + k);
        }
    };
    const int64_t tiles = (n + kTileM - 1) / kTileM;
    for (int64_t tile = static_cast<int64_t>(blockIdx.x) * kSlots + slot; tile < tiles;
         tile += static_cast<int64_t>(gridDim.x) * kSlots) {
        const int64_t p = tile * kTileM + row;
        {  // inputs: the 32 columns of this thread's row
            float v[kIn];
            if (p < n) {
                const float4* src = reinterpret_cast<const float4*>(x + p * kIn);
#pragma unroll
                for (int k = 0; k < kIn / 4; ++k) {
                    const float4 q = src[k];
                    v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
                }
            } else {
#pragma unroll
                for (int k = 0; k < kIn; ++k) v[k] = 0.0f;
            }
#pragma unroll
            for (int c = 0; c < kIn; c += 8) umma::st8(sm + xo, row, c, kTileM, v + c);
        }
        if (!layer(xo, sW1, kHid, kIn)) break;
        hidden(sbias);
        if (!layer(ho, sW2, kHid, kHid)) break;
        hidden(sbias + kHid);
        if (!layer(ho, sW3, kHid, kHid)) break;
        hidden(sbias + 2 * kHid);
        if (!layer(ho, sW4, kOutP, kHid)) break;
        {
            float v[16];
            umma::ld16(umma::lane_addr(T, 0), v);
            if (p < n) {
#pragma unroll
                for (int o = 0; o < kOut; ++o) y[p * kOut + o] = v[o] + sbias[3 * kHid + o];
            }
        }
    }
    umma::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) umma::tmem_free(tslot, 128 * kSlots);
}

// ---- training: gradient of L = (1/n) sum_p sum_o w_o (y_po - t_po)^2 --------------------------------
// Tile k goes to CTA k % grid; each CTA adds its tiles' weight and bias gradients into its own FP32
// slice part[cta][kPartStride] (no atomics) and its loss into loss_part[cta]; a second kernel sums the
// slices in CTA order, so the gradient is deterministic.
__device__ __forceinline__ void rmw(float* a, float v) { *a += v; }
// a[0..N) += v[0..N), a 16-byte aligned: N/4 vector loads and stores instead of N scalar ones (same sums)
template <int N>
__device__ __forceinline__ void rmw_row(float* a, const float* v) {
    static_assert(N % 4 == 0, "whole vectors");
    float4* q = reinterpret_cast<float4*>(a);
#pragma unroll
    for (int k = 0; k < N / 4; ++k) {
        float4 r = q[k];
        r.x += v[4 * k];
        r.y += v[4 * k + 1];
        r.z += v[4 * k + 2];
        r.w += v[4 * k + 3];
        q[k] = r;
    }
}

__global__ void __launch_bounds__(kTileM, 1) k_mlp_train(const float* __restrict__ x, const float* __restrict__ t,
                                                        const float* __restrict__ wout, int64_t n,
                                                        const __nv_bfloat16* __restrict__ wq,
                                                        const float* __restrict__ bq, float* __restrict__ part,
                                                        double* __restrict__ loss_part, int* status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    __shared__ double red[kTileM / 32];
    float* sbias = reinterpret_cast<float*>(sm + sBiasT);
    stage_weights(sm, wq, bq, sbias);
    for (int e = threadIdx.x; e < kTileM * 16 / 8; e += blockDim.x) {  // ones[128][16]
        const uint4 one = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);  // bf16 1.0 x 8
        *reinterpret_cast<uint4*>(sm + sOnes + e * 16) = one;
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    if (threadIdx.x < 32) umma::tmem_alloc(&tslot, 512);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    // tensor-memory columns: z1 [0,128) z2 [128,256) z3 / dH [256,384) y / dW [384,512)
    const uint32_t T1 = tslot, T2 = tslot + 128, T3 = tslot + 256, T4 = tslot + 384;
    const uint32_t base = smem_u32(sm);
    float* g = part + static_cast<int64_t>(blockIdx.x) * kPartStride;
    const float inv_n = 1.0f / static_cast<float>(n);
    uint32_t phase = 0;
    double lsum = 0.0;
    const int t_id = threadIdx.x;
    const int64_t tiles = (n + kTileM - 1) / kTileM;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t p = tile * kTileM + t_id;
        const bool valid = p < n;
        load_x(sm, x, p, n);
        // ---- forward, keeping z1 z2 z3 in tensor memory and h1 h2 h3 in shared memory
        before_issue();
        if (t_id == 0) { issue(T1, base + sX, kTileM, false, base + sW1, kHid, false, kHid, kIn); umma::commit(&bar); }
        if (!after_commit(&bar, phase, status)) break;
        hidden_out(T1, sbias, sm + sH1);
        before_issue();
        if (t_id == 0) { issue(T2, base + sH1, kTileM, false, base + sW2, kHid, false, kHid, kHid); umma::commit(&bar); }
        if (!after_commit(&bar, phase, status)) break;
        hidden_out(T2, sbias + kHid, sm + sH2);
        before_issue();
        if (t_id == 0) { issue(T3, base + sH2, kTileM, false, base + sW3, kHid, false, kHid, kHid); umma::commit(&bar); }
        if (!after_commit(&bar, phase, status)) break;
        hidden_out(T3, sbias + 2 * kHid, sm + sH3);
        before_issue();
        if (t_id == 0) { issue(T4, base + sH3, kTileM, false, base + sW4, kOutP, false, kOutP, kHid); umma::commit(&bar); }
        if (!after_commit(&bar, phase, status)) break;
        {  // output, loss, output gradient g4 = dL/dy
            float v[16], gv[16];
            umma::ld16(umma::lane_addr(T4, 0), v);
#pragma unroll
            for (int o = 0; o < kOutP; ++o) {
                gv[o] = 0.0f;
                if (o < kOut && valid) {
                    const float d = v[o] + sbias[3 * kHid + o] - t[p * kOut + o];
                    lsum += static_cast<double>(wout[o]) * d * d;
                    gv[o] = 2.0f * wout[o] * d * inv_n;
                }
            }
            umma::st8(sm + sG4, t_id, 0, kTileM, gv);
            umma::st8(sm + sG4, t_id, 8, kTileM, gv + 8);
        }
        // z3 into registers (its columns take dH3)
        float z[kHid];
#pragma unroll
        for (int c0 = 0; c0 < kHid; c0 += 32) umma::ld32(umma::lane_addr(T3, c0), z + c0);
#pragma unroll
        for (int c = 0; c < kHid; ++c) z[c] += sbias[2 * kHid + c];
        // ---- layer 4: dH3 = g4 W4, dW4^T = h3^T g4, db4 = colsum(g4)
        before_issue();
        if (t_id == 0) {
            issue(T3, base + sG4, kTileM, false, base + sW4, kOutP, true, kHid, kOutP);
            issue(T4, base + sH3, kTileM, true, base + sG4, kTileM, true, kOutP, kTileM);
            issue_colsum(T4 + 16, base + sOnes, base + sG4, kTileM, kOutP, kTileM);
            umma::commit(&bar);
        }
        if (!after_commit(&bar, phase, status)) break;
        {
            float v[16];
            umma::ld16(umma::lane_addr(T4, 0), v);  // row t = input feature t of layer 4
#pragma unroll
            for (int o = 0; o < kOut; ++o) rmw(g + oW4 + o * kHid + t_id, v[o]);
            umma::ld16(umma::lane_addr(T4 + 16, 0), v);
            if (t_id == 0) {
#pragma unroll
                for (int o = 0; o < kOut; ++o) rmw(g + ob4 + o, v[o]);
            }
        }
#pragma unroll 1
        for (int c0 = 0; c0 < kHid; c0 += 32) {  // dZ3 = dH3 * SiLU'(z3)
            float v[32];
            umma::ld32(umma::lane_addr(T3, c0), v);
#pragma unroll
            for (int k = 0; k < 32; ++k) v[k] *= dsilu(z[c0 + k]);
#pragma unroll
            for (int k = 0; k < 32; k += 8) umma::st8(sm + sG, t_id, c0 + k, kTileM, v + k);
        }
        // z2 into registers (its columns take db3)
#pragma unroll
        for (int c0 = 0; c0 < kHid; c0 += 32) umma::ld32(umma::lane_addr(T2, c0), z + c0);
#pragma unroll
        for (int c = 0; c < kHid; ++c) z[c] += sbias[kHid + c];
        // ---- layers 3, 2: dH = dZ W, dW = dZ^T h, db = colsum(dZ)
        bool ok = true;
#pragma unroll 1
        for (int layer = 3; layer >= 2 && ok; --layer) {
            const uint32_t sW = layer == 3 ? sW3 : sW2, sHin = layer == 3 ? sH2 : sH1;
            const int oW = layer == 3 ? oW3 : oW2, ob = layer == 3 ? ob3 : ob2;
            before_issue();
            if (t_id == 0) {
                issue(T3, base + sG, kTileM, false, base + sW, kHid, true, kHid, kHid);
                issue(T4, base + sG, kTileM, true, base + sHin, kTileM, true, kHid, kTileM);
                issue_colsum(T2, base + sOnes, base + sG, kTileM, kHid, kTileM);
                umma::commit(&bar);
            }
            if (!after_commit(&bar, phase, status)) { ok = false; break; }
#pragma unroll 1
            for (int c0 = 0; c0 < kHid; c0 += 32) {
                float v[32];
                umma::ld32(umma::lane_addr(T4, c0), v);  // row t = output unit t
                rmw_row<32>(g + oW + t_id * kHid + c0, v);
                umma::ld32(umma::lane_addr(T2, c0), v);
                if (t_id == 0) rmw_row<32>(g + ob + c0, v);
            }
            if (layer == 2) {  // z1 from its columns
#pragma unroll
                for (int c0 = 0; c0 < kHid; c0 += 32) umma::ld32(umma::lane_addr(T1, c0), z + c0);
#pragma unroll
                for (int c = 0; c < kHid; ++c) z[c] += sbias[c];
            }
            umma::fence_before();
            __syncthreads();  // every read of the dZ buffer by the MMAs is complete: overwrite it
#pragma unroll 1
            for (int c0 = 0; c0 < kHid; c0 += 32) {
                float v[32];
                umma::ld32(umma::lane_addr(T3, c0), v);
#pragma unroll
                for (int k = 0; k < 32; ++k) v[k] *= dsilu(z[c0 + k]);
#pragma unroll
                for (int k = 0; k < 32; k += 8) umma::st8(sm + sG, t_id, c0 + k, kTileM, v + k);
            }
            if (layer == 3) {  // z2 was loaded above; nothing to do
            }
        }
        if (!ok) break;
        // ---- layer 1: dW1 = dZ1^T x, db1 = colsum(dZ1)
        before_issue();
        if (t_id == 0) {
            issue(T4, base + sG, kTileM, true, base + sX, kTileM, true, kIn, kTileM);
            issue_colsum(T2, base + sOnes, base + sG, kTileM, kHid, kTileM);
            umma::commit(&bar);
        }
        if (!after_commit(&bar, phase, status)) break;
        {
            float v[32];
            umma::ld32(umma::lane_addr(T4, 0), v);
            rmw_row<kIn>(g + oW1 + t_id * kIn, v);
#pragma unroll 1
            for (int c0 = 0; c0 < kHid; c0 += 32) {
                umma::ld32(umma::lane_addr(T2, c0), v);
                if (t_id == 0) rmw_row<32>(g + ob1 + c0, v);
            }
        }
        umma::fence_before();
        __syncthreads();  // the next tile overwrites X and the activation buffers
    }
    // loss of this CTA
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((t_id & 31) == 0) red[t_id >> 5] = lsum;
    umma::fence_before();
    __syncthreads();
    if (t_id == 0) {
        double s = 0.0;
        for (int w = 0; w < kTileM / 32; ++w) s += red[w];
        loss_part[blockIdx.x] = s;
    }
    if (t_id < 32) umma::tmem_free(tslot, 512);
}

// grad[i] = sum over CTAs c of part[c][i] (fixed order); loss = sum of loss_part / n
__global__ void k_mlp_reduce(const float* __restrict__ part, int ncta, float* __restrict__ grad,
                             const double* __restrict__ loss_part, double* loss, int64_t n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kParams) {
        float s = 0.0f;
        for (int c = 0; c < ncta; ++c) s += part[static_cast<int64_t>(c) * kPartStride + i];
        grad[i] = s;
    }
    if (i == 0) {
        double s = 0.0;
        for (int c = 0; c < ncta; ++c) s += loss_part[c];
        *loss = s / static_cast<double>(n);
    }
}

// the squared global norm of the gradient (one block, fixed summation order) for gradient clipping
constexpr int kNormThreads = 1024;
__global__ void __launch_bounds__(kNormThreads) k_mlp_grad_norm(const float* __restrict__ grad, double* __restrict__ out) {
    __shared__ double sh[kNormThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < kParams; i += kNormThreads) s += static_cast<double>(grad[i]) * grad[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = kNormThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; with clip > 0 the gradient is first scaled by
// min(1, clip / ||g||_2) (global-norm clipping, Pascanu, Mikolov & Bengio 2013)
__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2,
                           float clip, const double* __restrict__ norm2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    float gi = grad[i];
    if (clip > 0.0f) {
        const double nrm = sqrt(*norm2);
        if (nrm > static_cast<double>(clip)) gi = static_cast<float>(gi * (static_cast<double>(clip) / nrm));
    }
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// FP32 master -> packed bf16 weights (W4 padded with zero rows) and FP32 biases
__global__ void k_mlp_pack(const float* __restrict__ w, __nv_bfloat16* __restrict__ wq, float* __restrict__ bq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kPacked) {
        float val = 0.0f;
        if (i < qW2) val = w[oW1 + i];
        else if (i < qW3) val = w[oW2 + (i - qW2)];
        else if (i < qW4) val = w[oW3 + (i - qW3)];
        else if (i - qW4 < kOut * kHid) val = w[oW4 + (i - qW4)];
        wq[i] = __float2bfloat16_rn(val);
    }
    if (i < kBias) {
        float b = 0.0f;
        if (i < kHid) b = w[ob1 + i];
        else if (i < 2 * kHid) b = w[ob2 + i - kHid];
        else if (i < 3 * kHid) b = w[ob3 + i - 2 * kHid];
        else if (i - 3 * kHid < kOut) b = w[ob4 + i - 3 * kHid];
        bq[i] = b;
    }
}

}  // namespace

// ---- the MLP object --------------------------------------------------------------------------------
struct gsph_mlp {
    float* w = nullptr;      // FP32 master parameters [kParams]
    float* m = nullptr;      // Adam moments
    float* v = nullptr;
    float* grad = nullptr;
    float* part = nullptr;   // [grid][kPartStride]
    double* loss_part = nullptr;
    double* loss = nullptr;
    __nv_bfloat16* wq = nullptr;
    float* bq = nullptr;
    int* status = nullptr;
    double* norm2 = nullptr;  // squared gradient norm (clipping)
    float clip = 0.0f;        // global-norm clipping threshold of the Adam step (0: off)
    int grid = 0;
    int64_t step = 0;
    std::string err;
};

namespace {

int mfail(gsph_mlp* m, int code, const std::string& msg) {
    if (m) m->err = msg;
    else set_global_error(msg);
    return code;
}
#define MLP_CK(mm, call, what)                                                              \
    do {                                                                                    \
        cudaError_t c_ = (call);                                                            \
        if (c_ != cudaSuccess) return mfail(mm, GSPH_E_CUDA, std::string(what) + ": " + cudaGetErrorString(c_)); \
    } while (0)

void mlp_release(gsph_mlp* m) {
    void* ptrs[] = {m->w, m->m, m->v, m->grad, m->part, m->loss_part, m->loss, m->wq, m->bq, m->status, m->norm2};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

int mlp_status(gsph_mlp* m, cudaStream_t s) {
    int st = 0;
    MLP_CK(m, cudaMemcpyAsync(&st, m->status, sizeof(int), cudaMemcpyDeviceToHost, s), "status read");
    MLP_CK(m, cudaStreamSynchronize(s), "stream synchronize");
    if (st) return mfail(m, GSPH_E_TIMEOUT, "a tensor-core completion wait gave up");
    return GSPH_OK;
}

}  // namespace

extern "C" {

int64_t gsph_mlp_param_count(void) { return kParams; }

int gsph_mlp_create(const float* params, gsph_mlp** out) {
    if (!out) return mfail(nullptr, GSPH_E_INVALID, "out is NULL");
    *out = nullptr;
    gsph_mlp* m = new (std::nothrow) gsph_mlp();
    if (!m) return mfail(nullptr, GSPH_E_NOMEM, "host allocation failed");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    m->grid = sms > 0 ? sms : 1;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    A(reinterpret_cast<void**>(&m->w), kParams * sizeof(float));
    A(reinterpret_cast<void**>(&m->m), kParams * sizeof(float));
    A(reinterpret_cast<void**>(&m->v), kParams * sizeof(float));
    A(reinterpret_cast<void**>(&m->grad), kParams * sizeof(float));
    A(reinterpret_cast<void**>(&m->part), static_cast<size_t>(m->grid) * kPartStride * sizeof(float));
    A(reinterpret_cast<void**>(&m->loss_part), static_cast<size_t>(m->grid) * sizeof(double));
    A(reinterpret_cast<void**>(&m->loss), sizeof(double));
    A(reinterpret_cast<void**>(&m->wq), kPacked * sizeof(__nv_bfloat16));
    A(reinterpret_cast<void**>(&m->bq), kBias * sizeof(float));
    A(reinterpret_cast<void**>(&m->status), sizeof(int));
    A(reinterpret_cast<void**>(&m->norm2), sizeof(double));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
    if (e == cudaSuccess && params) e = cudaMemcpy(m->w, params, kParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_mlp_pack<<<(kPacked + 255) / 256, 256>>>(m->w, m->wq, m->bq);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        const std::string msg = std::string("gsph_mlp_create: ") + cudaGetErrorString(e);
        mlp_release(m);
        delete m;
        return mfail(nullptr, GSPH_E_CUDA, msg);
    }
    *out = m;
    return GSPH_OK;
}

int gsph_mlp_destroy(gsph_mlp* m) {
    if (!m) return GSPH_E_INVALID;
    cudaDeviceSynchronize();
    mlp_release(m);
    delete m;
    return GSPH_OK;
}

int gsph_mlp_get_params(gsph_mlp* m, float* params) {
    if (!m || !params) return mfail(m, GSPH_E_INVALID, "NULL argument");
    MLP_CK(m, cudaMemcpy(params, m->w, kParams * sizeof(float), cudaMemcpyDeviceToHost), "copy");
    return GSPH_OK;
}

int gsph_mlp_set_params(gsph_mlp* m, const float* params) {
    if (!m || !params) return mfail(m, GSPH_E_INVALID, "NULL argument");
    MLP_CK(m, cudaMemcpy(m->w, params, kParams * sizeof(float), cudaMemcpyHostToDevice), "copy");
    MLP_CK(m, cudaMemset(m->m, 0, kParams * sizeof(float)), "reset");
    MLP_CK(m, cudaMemset(m->v, 0, kParams * sizeof(float)), "reset");
    m->step = 0;
    k_mlp_pack<<<(kPacked + 255) / 256, 256>>>(m->w, m->wq, m->bq);
    MLP_CK(m, cudaGetLastError(), "pack");
    MLP_CK(m, cudaDeviceSynchronize(), "pack");
    return GSPH_OK;
}

int gsph_mlp_forward(gsph_mlp* m, const float* x, float* y, int64_t n, void* stream) {
    if (!m || (!x && n) || (!y && n) || n < 0) return mfail(m, GSPH_E_INVALID, "bad argument");
    // the kernel reads each input row as 16-byte vectors
    if (reinterpret_cast<uintptr_t>(x) % 16) return mfail(m, GSPH_E_INVALID, "x must be 16-byte aligned");
    if (n == 0) return GSPH_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t tiles = (n + kTileM - 1) / kTileM;
    const int64_t pairs = (tiles + kSlots - 1) / kSlots;  // a CTA takes kSlots tiles at a time
    const int grid = static_cast<int>(pairs < m->grid ? pairs : m->grid);
    k_mlp_forward<<<grid, kFwdThreads, kFwdSmem, s>>>(x, y, n, m->wq, m->bq, m->status);
    MLP_CK(m, cudaGetLastError(), "forward launch");
    return GSPH_OK;
}

int gsph_mlp_gradient(gsph_mlp* m, const float* x, const float* target, const float* wout, int64_t n, float* grad,
                      double* loss, void* stream) {
    if (!m || !x || !target || !wout || n <= 0) return mfail(m, GSPH_E_INVALID, "bad argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t tiles = (n + kTileM - 1) / kTileM;
    const int grid = static_cast<int>(tiles < m->grid ? tiles : m->grid);
    MLP_CK(m, cudaMemsetAsync(m->part, 0, static_cast<size_t>(grid) * kPartStride * sizeof(float), s), "clear");
    k_mlp_train<<<grid, kTileM, kTrainSmem, s>>>(x, target, wout, n, m->wq, m->bq, m->part, m->loss_part, m->status);
    MLP_CK(m, cudaGetLastError(), "gradient launch");
    k_mlp_reduce<<<(kParams + 255) / 256, 256, 0, s>>>(m->part, grid, m->grad, m->loss_part, m->loss, n);
    MLP_CK(m, cudaGetLastError(), "reduce launch");
    if (grad) MLP_CK(m, cudaMemcpyAsync(grad, m->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, s), "grad copy");
    if (loss) MLP_CK(m, cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, s), "loss copy");
    if (grad || loss) return mlp_status(m, s);
    return GSPH_OK;
}

int gsph_mlp_adam(gsph_mlp* m, float lr, float beta1, float beta2, float eps, void* stream) {
    if (!m) return GSPH_E_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    m->step += 1;
    const float c1 = 1.0f - powf(beta1, static_cast<float>(m->step));
    const float c2 = 1.0f - powf(beta2, static_cast<float>(m->step));
    if (m->clip > 0.0f) {
        k_mlp_grad_norm<<<1, kNormThreads, 0, s>>>(m->grad, m->norm2);
        MLP_CK(m, cudaGetLastError(), "gradient norm launch");
    }
    k_mlp_adam<<<(kParams + 255) / 256, 256, 0, s>>>(m->w, m->m, m->v, m->grad, lr, beta1, beta2, eps, c1, c2, m->clip,
                                                     m->norm2);
    MLP_CK(m, cudaGetLastError(), "adam launch");
    k_mlp_pack<<<(kPacked + 255) / 256, 256, 0, s>>>(m->w, m->wq, m->bq);
    MLP_CK(m, cudaGetLastError(), "pack launch");
    return GSPH_OK;
}

int gsph_mlp_set_grad_clip(gsph_mlp* m, float max_norm) {
    if (!m) return GSPH_E_INVALID;
    if (!(max_norm >= 0.0f)) return mfail(m, GSPH_E_INVALID, "max_norm must be >= 0");
    m->clip = max_norm;
    return GSPH_OK;
}

const char* gsph_mlp_last_error(const gsph_mlp* m) { return m ? m->err.c_str() : gsph_last_error(nullptr); }


// D[128][N] (FP32, row-major) = A[128][K] * B[N][K]^T from bf16 row-major device arrays, on the tensor
// cores; N in {16, 32, ..., 128}, K in {16, 32, ..., 128}. Synchronises the device; status as gsph_*.
int gsph_tc_gemm_check(const void* A, const void* B, float* D, int32_t N, int32_t K, int32_t a_mn, int32_t b_mn) {
    if (!A || !B || !D || N < 16 || N > 128 || N % 16 || K < 16 || K > 128 || K % 16) {
        set_global_error("gsph_tc_gemm_check: N and K must be multiples of 16 in [16, 128], pointers non-NULL");
        return GSPH_E_INVALID;
    }
    int* status = nullptr;
    cudaError_t e = cudaMalloc(&status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_tc_gemm_check, cudaFuncAttributeMaxDynamicSharedMemorySize, kCheckSmem);
    if (e == cudaSuccess) {
        k_tc_gemm_check<<<1, kTileM, kCheckSmem>>>(static_cast<const __nv_bfloat16*>(A),
                                                    static_cast<const __nv_bfloat16*>(B), D, N, K, a_mn != 0,
                                                    b_mn != 0, status);
        e = cudaGetLastError();
    }
    int st = 0;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost);
    if (status) cudaFree(status);
    if (e != cudaSuccess) {
        set_global_error(std::string("gsph_tc_gemm_check: ") + cudaGetErrorString(e));
        return GSPH_E_CUDA;
    }
    if (st) {
        set_global_error("gsph_tc_gemm_check: the MMA completion wait gave up");
        return GSPH_E_TIMEOUT;
    }
    return GSPH_OK;
}

}  // extern "C"
