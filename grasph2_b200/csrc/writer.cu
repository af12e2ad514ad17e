// writer.cu -- asynchronous snapshot output (the reference's ResultStorageManager: printToFile copies
// the device buffers to a duplicate and a worker thread downloads and writes them,
// src/ResultStorageManager.h:140-148, src/ResultStorageManager.cu:102-186).
//
// gsph_writer_write() copies the context's state on the device into one of `depth` slots, ordered on
// the caller's stream (later steps do not disturb it), then unpacks it to the host layout and copies it
// into the slot's pinned host buffers on the writer's own copy stream, and returns. A worker thread
// waits for each slot's copy event and writes the tsv file (the reference's format and order). When
// every slot is busy, write() waits for the oldest one (a bounded queue). The worker never touches the
// context, so the simulation keeps stepping while snapshots are written.
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/grasph2_b200.hpp"
#include "integrate.cuh"

void set_global_error(const std::string& msg);                                       // capi.cu
bool gsph_ctx_state(gsph_ctx* c, gsph::DevArrays* a, const int** ext);                // capi.cu

using namespace gsph;

struct gsph_writer {
    struct Slot {
        DevArrays a{};
        int* ext = nullptr;
        float* staging = nullptr;       // device, 9 n floats
        float* host[11] = {};           // pinned
        cudaEvent_t copied = nullptr;   // device copy of the state done (on the caller's stream)
        cudaEvent_t done = nullptr;     // host buffers complete (copy stream)
        std::string file;
        bool busy = false;
    };
    gsph_ctx* ctx = nullptr;
    uint32_t mask = 0;
    int64_t n = 0;
    cudaStream_t copy = nullptr;
    std::vector<Slot> slots;
    int next = 0;
    std::deque<int> queue;
    std::mutex m;
    std::condition_variable cv_job, cv_free;
    std::thread worker;
    bool stop = false;
    int first_err = GSPH_OK;
    std::string err;
    int64_t written = 0;
};

namespace {

constexpr int kComps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};

int wfail(gsph_writer* w, int code, const std::string& msg) {
    if (w) {
        std::lock_guard<std::mutex> lk(w->m);
        w->err = msg;
        if (w->first_err == GSPH_OK) w->first_err = code;
    } else {
        set_global_error(msg);
    }
    return code;
}

void worker_loop(gsph_writer* w) {
    for (;;) {
        int k;
        {
            std::unique_lock<std::mutex> lk(w->m);
            w->cv_job.wait(lk, [&] { return w->stop || !w->queue.empty(); });
            if (w->queue.empty()) return;  // stop requested and nothing left
            k = w->queue.front();
        }
        gsph_writer::Slot& s = w->slots[k];
        int code = GSPH_OK;
        std::string msg;
        const cudaError_t e = cudaEventSynchronize(s.done);
        if (e != cudaSuccess) {
            code = GSPH_E_CUDA;
            msg = std::string("snapshot copy: ") + cudaGetErrorString(e);
        } else {
            gsph_host_particles v{s.host[0], s.host[1], s.host[2], s.host[3], s.host[4], s.host[5],
                                  s.host[6], s.host[7], s.host[8], s.host[9], s.host[10]};
            const bool h5 = s.file.size() > 3 && s.file.compare(s.file.size() - 3, 3, ".h5") == 0;
            if (h5) {  // the reference's STORE_HDF5 output (ResultStorageManager.cu:191-227)
                code = gsph_h5_write(s.file.c_str(), w->n, &v, w->mask);
                if (code != GSPH_OK) msg = gsph_last_error(nullptr);
            } else {
                try {
                    printTextFile(v, static_cast<size_t>(w->n), s.file, w->mask);
                } catch (const std::exception& ex) {
                    code = GSPH_E_INVALID;
                    msg = ex.what();
                }
            }
        }
        {
            std::lock_guard<std::mutex> lk(w->m);
            w->queue.pop_front();
            s.busy = false;
            if (code != GSPH_OK) {
                if (w->first_err == GSPH_OK) w->first_err = code;
                w->err = msg;
            } else {
                ++w->written;
            }
        }
        w->cv_free.notify_all();
    }
}

void release(gsph_writer* w) {
    for (auto& s : w->slots) {
        void* dev[] = {s.a.posm, s.a.velrho, s.a.acc, s.a.xvel, s.a.sA, s.a.sB, s.a.dA, s.a.dB, s.a.rhodot,
                       s.a.balsara, s.ext, s.staging};
        for (void* p : dev)
            if (p) cudaFree(p);
        for (float* h : s.host)
            if (h) cudaFreeHost(h);
        if (s.copied) cudaEventDestroy(s.copied);
        if (s.done) cudaEventDestroy(s.done);
    }
    if (w->copy) cudaStreamDestroy(w->copy);
}

}  // namespace

extern "C" {

int gsph_writer_create(gsph_ctx* ctx, uint32_t mask, int32_t depth, gsph_writer** out) {
    if (!out) return wfail(nullptr, GSPH_E_INVALID, "out is NULL");
    *out = nullptr;
    DevArrays a{};
    const int* ext = nullptr;
    if (!ctx || !gsph_ctx_state(ctx, &a, &ext))
        return wfail(nullptr, GSPH_E_UNSUPPORTED, "the writer needs a single-precision context");
    if (mask == 0 || (mask & ~GSPH_ALL_ATTRIBS) || depth < 1 || depth > 16)
        return wfail(nullptr, GSPH_E_INVALID, "mask must name attributes; depth in [1, 16]");
    gsph_writer* w = new (std::nothrow) gsph_writer();
    if (!w) return wfail(nullptr, GSPH_E_NOMEM, "host allocation failed");
    w->ctx = ctx;
    w->mask = mask;
    w->n = a.n;
    const int64_t np = a.n_pad;
    cudaError_t e = cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking);
    w->slots.resize(depth);
    for (auto& s : w->slots) {
        auto D = [&](void** p, size_t bytes) {
            if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        };
        s.a = a;
        float4** f4[] = {&s.a.posm, &s.a.velrho, &s.a.acc, &s.a.xvel, &s.a.sA, &s.a.sB, &s.a.dA, &s.a.dB};
        for (float4** p : f4) {
            *p = nullptr;
            D(reinterpret_cast<void**>(p), np * sizeof(float4));
        }
        s.a.rhodot = s.a.balsara = nullptr;
        D(reinterpret_cast<void**>(&s.a.rhodot), np * sizeof(float));
        D(reinterpret_cast<void**>(&s.a.balsara), np * sizeof(float));
        if (ext) D(reinterpret_cast<void**>(&s.ext), np * sizeof(int));
        D(reinterpret_cast<void**>(&s.staging), 9 * a.n * sizeof(float));
        for (int k = 0; k < 11; ++k)
            if ((mask >> k & 1u) && e == cudaSuccess)
                e = cudaHostAlloc(reinterpret_cast<void**>(&s.host[k]), kComps[k] * a.n * sizeof(float),
                                  cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        const std::string msg = std::string("gsph_writer_create: ") + cudaGetErrorString(e);
        release(w);
        delete w;
        return wfail(nullptr, GSPH_E_NOMEM, msg);
    }
    w->worker = std::thread(worker_loop, w);
    *out = w;
    return GSPH_OK;
}

int gsph_writer_write(gsph_writer* w, const char* filename, void* stream) {
    if (!w || !filename) return wfail(w, GSPH_E_INVALID, "NULL argument");
    int k;
    {
        std::unique_lock<std::mutex> lk(w->m);
        w->cv_free.wait(lk, [&] {
            for (const auto& s : w->slots)
                if (!s.busy) return true;
            return false;
        });
        k = w->next;
        while (w->slots[k].busy) k = (k + 1) % static_cast<int>(w->slots.size());
        w->next = (k + 1) % static_cast<int>(w->slots.size());
    }
    gsph_writer::Slot& s = w->slots[k];
    DevArrays a{};
    const int* ext = nullptr;
    gsph_ctx_state(w->ctx, &a, &ext);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int64_t np = a.n_pad;
    struct C { void* dst; const void* src; size_t bytes; };
    const C copies[] = {{s.a.posm, a.posm, np * sizeof(float4)}, {s.a.velrho, a.velrho, np * sizeof(float4)},
                        {s.a.acc, a.acc, np * sizeof(float4)}, {s.a.xvel, a.xvel, np * sizeof(float4)},
                        {s.a.sA, a.sA, np * sizeof(float4)}, {s.a.sB, a.sB, np * sizeof(float4)},
                        {s.a.dA, a.dA, np * sizeof(float4)}, {s.a.dB, a.dB, np * sizeof(float4)},
                        {s.a.rhodot, a.rhodot, np * sizeof(float)}, {s.a.balsara, a.balsara, np * sizeof(float)},
                        {s.ext, ext, np * sizeof(int)}};
    cudaError_t e = cudaSuccess;
    for (const C& c : copies)
        if (c.dst && c.src && e == cudaSuccess) e = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(s.copied, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(w->copy, s.copied, 0);
    for (int b = 0; b < 11 && e == cudaSuccess; ++b) {
        if (!(w->mask >> b & 1u)) continue;
        e = launch_unpack(s.a, b, s.staging, s.ext, w->copy);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s.host[b], s.staging, kComps[b] * a.n * sizeof(float), cudaMemcpyDeviceToHost, w->copy);
    }
    if (e == cudaSuccess) e = cudaEventRecord(s.done, w->copy);
    if (e != cudaSuccess) return wfail(w, GSPH_E_CUDA, std::string("gsph_writer_write: ") + cudaGetErrorString(e));
    {
        std::lock_guard<std::mutex> lk(w->m);
        s.file = filename;
        s.busy = true;
        w->queue.push_back(k);
    }
    w->cv_job.notify_one();
    return GSPH_OK;
}

int gsph_writer_flush(gsph_writer* w, int64_t* written) {
    if (!w) return GSPH_E_INVALID;
    std::unique_lock<std::mutex> lk(w->m);
    w->cv_free.wait(lk, [&] { return w->queue.empty(); });
    if (written) *written = w->written;
    return w->first_err;
}

const char* gsph_writer_last_error(gsph_writer* w) {
    if (!w) return gsph_last_error(nullptr);
    std::lock_guard<std::mutex> lk(w->m);
    return w->err.c_str();
}

int gsph_writer_destroy(gsph_writer* w) {
    if (!w) return GSPH_E_INVALID;
    gsph_writer_flush(w, nullptr);
    {
        std::lock_guard<std::mutex> lk(w->m);
        w->stop = true;
    }
    w->cv_job.notify_all();
    if (w->worker.joinable()) w->worker.join();
    const int rc = w->first_err;
    release(w);
    delete w;
    return rc;
}

}  // extern "C"
