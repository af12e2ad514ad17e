// mlp.cu -- the per-particle MLP of the learned surrogate on the tensor cores (tcgen05, BF16 operands,
// FP32 accumulation in tensor memory), and a tile-GEMM check of the operand encodings.
#include <cuda_bf16.h>

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

}  // namespace

extern "C" {

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
