// noalloc.cu -- softened all-pairs gravity for callers that cannot allocate device memory.
//
// Some callers may not call cudaMalloc: a host application that hands out all device memory from a
// pool fixed at start-up (an allocation from inside a library would break its budget), or a loop
// that must never stall, since cudaMalloc/cudaFree may synchronise the whole device. For them,
// gsph_gravity_accel_static computes the same accelerations as the gravity pass of
// gsph_compute_derivatives from caller-owned device arrays, keeping its scratch -- the padded
// j-records and the j-split partial sums -- in one file-scope device array of a fixed size.
#include <algorithm>
#include <initializer_list>
#include <atomic>
#include <mutex>
#include <string>

#include "pairs.cuh"

void set_global_error(const std::string& msg);

namespace {

using namespace gsph;

constexpr int64_t kStaticMaxN = 524288;                 // most particles one call accepts
constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB, held by every device that loads the library
constexpr size_t kStatusBytes = 256;                    // status word, padded to the array's alignment
constexpr int kMaxDevices = 64;

// Shared by every call on a device and left holding the last call's data. Layout:
// [status int | padding to 256 B][n_pad j-records (float4)][nseg x 3 x n_pad partial sums (float)]
static __device__ __align__(256) unsigned char g_gravity_scratch[kStaticScratchBytes];

std::mutex g_lock;
void* g_scratch_addr[kMaxDevices] = {};
std::atomic<int> g_inject_timeout{0};  // test hook: the next call starts with the timeout bit set

// The device address of the array for the current device. In host code the array's name stands for
// a host-side shadow, not a device address, so the address is looked up with cudaGetSymbolAddress:
// afresh on every call outside stream capture (a device reset reloads the module and moves the
// array), and from the last lookup while `s` is capturing (the first call on a device must come
// before any capture).
int scratch_address(cudaStream_t s, void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_global_error(std::string("no usable CUDA device: ") + cudaGetErrorString(e));
        return GSPH_E_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_global_error("device index out of range for the static scratch table");
        return GSPH_E_UNSUPPORTED;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) {
        set_global_error(std::string("cudaStreamIsCapturing failed: ") + cudaGetErrorString(e));
        return GSPH_E_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_lock);
    if (cap == cudaStreamCaptureStatusNone || !g_scratch_addr[dev]) {
        if (cap != cudaStreamCaptureStatusNone) {
            set_global_error("the first call on a device must come before any stream capture");
            return GSPH_E_INVALID;
        }
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_gravity_scratch);
        if (e != cudaSuccess || !p) {
            set_global_error(std::string("cudaGetSymbolAddress of the static scratch failed: ") +
                             cudaGetErrorString(e));
            return GSPH_E_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return GSPH_OK;
}

// the caller's n records, then inert padding (zero mass, far away) up to n_pad; the status word
// starts at `status0`
__global__ void k_static_pad(const float4* __restrict__ in, float4* __restrict__ out, int64_t n, int64_t n_pad,
                             int* status, int status0) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i == 0) *status = status0;
    if (i >= n_pad) return;
    out[i] = (i < n) ? in[i] : make_float4(1e18f, 1e18f, 1e18f, 0.0f);
}

// a_i = G * (sum of the segments, fixed order). If a bounded wait of the gravity kernel gave up
// (timeout bit in the status word), some j-tiles were never summed: every output is NaN instead, so a
// partial result cannot pass for a correct one.
__global__ void k_static_finish(const float* __restrict__ part, float4* __restrict__ acc, int64_t n, int64_t n_pad,
                                int nseg, float G, const int* __restrict__ status) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (*status & GSPH_DEV_ERR_TIMEOUT) {
        const float q = __int_as_float(0x7fc00000);
        acc[i] = make_float4(q, q, q, q);
        return;
    }
    float s[3] = {0.0f, 0.0f, 0.0f};
    for (int k = 0; k < nseg; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) s[c] += part[(static_cast<int64_t>(k) * 3 + c) * n_pad + i];
    acc[i] = make_float4(G * s[0], G * s[1], G * s[2], 0.0f);
}

}  // namespace

extern "C" int gsph_gravity_accel_static(const void* posm, int64_t n, double G, double eps, void* acc, void* stream) {
    if (!posm || !acc) {
        set_global_error("posm and acc must be device pointers");
        return GSPH_E_INVALID;
    }
    if ((reinterpret_cast<uintptr_t>(posm) | reinterpret_cast<uintptr_t>(acc)) & 15u) {
        set_global_error("posm and acc must be 16-byte aligned float4 arrays");
        return GSPH_E_INVALID;
    }
    if (n < 1 || n > kStaticMaxN) {
        set_global_error("n must be in [1, 524288] (the static scratch holds at most 524288 particles)");
        return GSPH_E_INVALID;
    }
    if (!(eps >= 0.0) || !(G == G)) {
        set_global_error("eps must be >= 0 and G a number");
        return GSPH_E_INVALID;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    void* base = nullptr;
    const int rc = scratch_address(s, &base);
    if (rc != GSPH_OK) return rc;

    const int64_t n_pad = (n + kPad - 1) / kPad * kPad;
    const bool small = n_pad < 65536;
    const int ipt = small ? 2 : 4;
    const int jt = small ? 64 : 256;
    const size_t rec_bytes = static_cast<size_t>(n_pad) * sizeof(float4);
    const size_t seg_bytes = static_cast<size_t>(3) * n_pad * sizeof(float);
    const int64_t fit = static_cast<int64_t>((kStaticScratchBytes - kStatusBytes - rec_bytes) / seg_bytes);
    const int nseg = static_cast<int>(std::min(std::min<int64_t>(16, fit), n_pad / jt));  // fit >= 1 for n <= kStaticMaxN

    unsigned char* b = static_cast<unsigned char*>(base);
    int* status = reinterpret_cast<int*>(b);
    float4* rec = reinterpret_cast<float4*>(b + kStatusBytes);
    float* part = reinterpret_cast<float*>(b + kStatusBytes + rec_bytes);

    // the status word starts at zero (or, for the failure-path test, with the timeout bit set)
    const int status0 = g_inject_timeout.exchange(0) ? GSPH_DEV_ERR_TIMEOUT : 0;
    k_static_pad<<<static_cast<unsigned>((n_pad + 255) / 256), 256, 0, s>>>(static_cast<const float4*>(posm), rec, n,
                                                                             n_pad, status, status0);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = launch_gravity_raw(rec, part, n_pad, ipt, jt, nseg, static_cast<float>(eps * eps), status, s);
    if (e == cudaSuccess) {
        k_static_finish<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(part, static_cast<float4*>(acc), n, n_pad,
                                                                                nseg, static_cast<float>(G), status);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_global_error(std::string("gravity launch failed: ") + cudaGetErrorString(e));
        return GSPH_E_CUDA;
    }
    return GSPH_OK;
}

extern "C" int gsph_gravity_accel_static_status(void* stream) {
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    void* base = nullptr;
    const int rc = scratch_address(s, &base);
    if (rc != GSPH_OK) return rc;
    int st = 0;
    cudaError_t e = cudaMemcpyAsync(&st, base, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_global_error(std::string("status read failed: ") + cudaGetErrorString(e));
        return GSPH_E_CUDA;
    }
    if (st & GSPH_DEV_ERR_TIMEOUT) {
        set_global_error("a device-side wait of gsph_gravity_accel_static gave up; its accelerations are NaN");
        return GSPH_E_TIMEOUT;
    }
    return GSPH_OK;
}

extern "C" int gsph_inject_static_timeout(int on) {
    g_inject_timeout.store(on ? 1 : 0);
    return GSPH_OK;
}
