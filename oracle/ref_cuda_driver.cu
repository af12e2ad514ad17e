/*
 * ref_cuda_driver.cu -- TEST INFRASTRUCTURE ONLY. Builds GraSPH2's own CUDA hot path for sm_100a:
 * computeDerivatives(pb) (src/computeDerivatives.h:315-328) with its three jobs run by the
 * reference's tile kernel do_for_each_pair_fast_impl (src/particles/algorithms.h:270-309), and
 * integrate(pb, notFirstStep) (src/integration.h:219-244) with the fixed-step job or the two
 * variable-step kernels (:130-217), all #included unchanged from the reference tree. The particle
 * engine and mpUtils are the stand-ins of oracle/ref_shim_cuda/. Compiled by oracle/build_ref.py
 * (nvcc, per-thread default stream as the reference's CMakeLists.txt:148) into
 * oracle/_ref/libref_cuda_<variant>.so, one per physics variant. The tests compare the product with
 * it; bench.py times it beside the CPU arm.
 *
 * The reference's tile loop is only correct for N a multiple of its 256-thread block
 * (algorithms.h:285-301 re-reads stale shared memory on the last tile otherwise); callers keep to
 * such N. This driver adds only the host side: upload/download between the caller's host layout
 * (pos[3n], mass[n], vel[3n], ..., dstress[9n] row-major) and the reference's device layout, and
 * event timing of whole steps.
 */
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "settings.h"
#include "computeDerivatives.h"

/* the caller's host arrays: the layout of oracle_particles (oracle/oracle.cpp) */
struct refcu_particles {
    f1_t* pos;
    f1_t* mass;
    f1_t* vel;
    f1_t* acc;
    f1_t* balsara;
    f1_t* xvel;
    f1_t* density;
    f1_t* density_dt;
    f1_t* dstress;
    f1_t* dstress_dt;
    f1_t* maxvsig;
};

namespace {
std::string g_err;

using Buffer = DeviceParticleBuffer<>;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        assert_cuda(cudaDeviceSynchronize());
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

template <typename T>
void put(T* dst, const std::vector<T>& src) {
    assert_cuda(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
}
template <typename T>
void get(std::vector<T>& dst, const T* src) {
    assert_cuda(cudaMemcpy(dst.data(), src, dst.size() * sizeof(T), cudaMemcpyDeviceToHost));
}
}  // namespace

extern "C" {

const char* refcu_last_error(void) { return g_err.c_str(); }
int refcu_precision(void) { return static_cast<int>(sizeof(f1_t)); }

void* refcu_create(int64_t n) {
    Buffer* b = nullptr;
    if (guarded([&] { b = new Buffer(static_cast<size_t>(n)); }) != 0) return nullptr;
    return b;
}

void refcu_destroy(void* h) { delete static_cast<Buffer*>(h); }

int refcu_upload(void* h, const refcu_particles* s) {
    Buffer* b = static_cast<Buffer*>(h);
    if (!b || !s) return -1;
    return guarded([&] {
        const size_t n = b->size();
        const gsph_dev_arrays& a = b->ref.a;
        std::vector<f4_t> posm(n), vel(n), acc(n), xvel(n);
        std::vector<f1_t> bal(n), rho(n), rhodt(n), vsig(n);
        std::vector<m3_t> S(n), dS(n);
        for (size_t i = 0; i < n; ++i) {
            posm[i] = f4_t{s->pos[3 * i], s->pos[3 * i + 1], s->pos[3 * i + 2], s->mass[i]};
            vel[i] = f4_t{s->vel[3 * i], s->vel[3 * i + 1], s->vel[3 * i + 2], 0};
            acc[i] = f4_t{s->acc[3 * i], s->acc[3 * i + 1], s->acc[3 * i + 2], 0};
            xvel[i] = f4_t{s->xvel[3 * i], s->xvel[3 * i + 1], s->xvel[3 * i + 2], 0};
            bal[i] = s->balsara[i];
            rho[i] = s->density[i];
            rhodt[i] = s->density_dt[i];
            vsig[i] = s->maxvsig[i];
            for (int e = 0; e < 9; ++e) {
                S[i](e) = s->dstress[9 * i + e];
                dS[i](e) = s->dstress_dt[9 * i + e];
            }
        }
        put(a.posm, posm); put(a.vel, vel); put(a.acc, acc); put(a.xvel, xvel);
        put(a.balsara, bal); put(a.density, rho); put(a.density_dt, rhodt); put(a.maxvsig, vsig);
        put(a.dstress, S); put(a.dstress_dt, dS);
    });
}

int refcu_download(void* h, refcu_particles* s) {
    Buffer* b = static_cast<Buffer*>(h);
    if (!b || !s) return -1;
    return guarded([&] {
        const size_t n = b->size();
        const gsph_dev_arrays& a = b->ref.a;
        std::vector<f4_t> posm(n), vel(n), acc(n), xvel(n);
        std::vector<f1_t> bal(n), rho(n), rhodt(n), vsig(n);
        std::vector<m3_t> S(n), dS(n);
        get(posm, a.posm); get(vel, a.vel); get(acc, a.acc); get(xvel, a.xvel);
        get(bal, a.balsara); get(rho, a.density); get(rhodt, a.density_dt); get(vsig, a.maxvsig);
        get(S, a.dstress); get(dS, a.dstress_dt);
        for (size_t i = 0; i < n; ++i) {
            s->pos[3 * i] = posm[i].x; s->pos[3 * i + 1] = posm[i].y; s->pos[3 * i + 2] = posm[i].z;
            s->mass[i] = posm[i].w;
            s->vel[3 * i] = vel[i].x; s->vel[3 * i + 1] = vel[i].y; s->vel[3 * i + 2] = vel[i].z;
            s->acc[3 * i] = acc[i].x; s->acc[3 * i + 1] = acc[i].y; s->acc[3 * i + 2] = acc[i].z;
            s->xvel[3 * i] = xvel[i].x; s->xvel[3 * i + 1] = xvel[i].y; s->xvel[3 * i + 2] = xvel[i].z;
            s->balsara[i] = bal[i];
            s->density[i] = rho[i];
            s->density_dt[i] = rhodt[i];
            s->maxvsig[i] = vsig[i];
            for (int e = 0; e < 9; ++e) {
                s->dstress[9 * i + e] = S[i](e);
                s->dstress_dt[9 * i + e] = dS[i](e);
            }
        }
    });
}

/* computeDerivatives(pb) */
int refcu_compute_derivatives(void* h) {
    Buffer* b = static_cast<Buffer*>(h);
    if (!b) return -1;
    return guarded([&] { computeDerivatives(*b); });
}

/* integrate(pb, notFirstStep) */
int refcu_integrate(void* h, int not_first_step) {
    Buffer* b = static_cast<Buffer*>(h);
    if (!b) return -1;
    return guarded([&] { integrate(*b, not_first_step != 0); });
}

/* getCurrentTimestep() */
double refcu_current_timestep(void) {
    double dt = 0;
    guarded([&] { dt = static_cast<double>(getCurrentTimestep()); });
    return dt;
}

/* the reference's device time-step symbols currentTS / nextTS (src/integration.h:127-128), which keep
 * their values between calls in one process: set both (zero before a fresh variable-step run) */
int refcu_set_timestep(double current, double next) {
    return guarded([&] {
#if defined(VARIABLE_TIMESTEP_LEAPFROG)
        const f1_t c = static_cast<f1_t>(current), x = static_cast<f1_t>(next);
        assert_cuda(cudaMemcpyToSymbol(currentTS, &c, sizeof(f1_t)));
        assert_cuda(cudaMemcpyToSymbol(nextTS, &x, sizeof(f1_t)));
#else
        (void)current;
        (void)next;
#endif
    });
}

/* `steps` x {computeDerivatives(pb); integrate(pb, true)}, the loop body of src/main.cu:249-273
 * without I/O, timed with CUDA events on the per-thread default stream; *ms = total device time */
int refcu_time_steps(void* h, int steps, double* ms) {
    Buffer* b = static_cast<Buffer*>(h);
    if (!b || !ms || steps < 1) return -1;
    return guarded([&] {
        cudaEvent_t e0, e1;
        assert_cuda(cudaEventCreate(&e0));
        assert_cuda(cudaEventCreate(&e1));
        assert_cuda(cudaEventRecord(e0, cudaStreamPerThread));
        for (int k = 0; k < steps; ++k) {
            computeDerivatives(*b);
            integrate(*b, true);
        }
        assert_cuda(cudaEventRecord(e1, cudaStreamPerThread));
        assert_cuda(cudaEventSynchronize(e1));
        float t = 0;
        assert_cuda(cudaEventElapsedTime(&t, e0, e1));
        *ms = t;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    });
}

}  // extern "C"
