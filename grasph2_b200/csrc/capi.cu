// capi.cu -- the C-ABI of include/grasph2_b200.h: context (the DeviceParticleBuffer analogue),
// upload/download in the reference's attribute layout, computeDerivatives / integrate dispatch,
// the CUDA-graph step loop and the FP64 diagnostics.
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "fp64.cuh"
#include "surrogate.cuh"
#include "integrate.cuh"
#include "pairs.cuh"
#include "spatial.cuh"

using namespace gsph;

constexpr int kSnapSlots = 4;
// floats per particle of the transfer staging buffer: the components of all 11 attributes
// (pos 3, mass 1, vel 3, acc 3, balsara 1, xvel 3, density 1, density_dt 1, dstress 9, dstress_dt 9, maxvsig 1)
constexpr int kStagingFloats = 35;

struct gsph_ctx {
    gsph_params params;
    gsph_options opt;
    DevParams dp;
    Launch L;
    DevArrays a;
    SpatialArrays sp{};
    int64_t steps_since_sort = 0;
    cudaStream_t side = nullptr;   // gravity runs here, concurrent with the SPH chain (culled path)
    bool fp64 = false;             // GSPH_PRECISION_DOUBLE: every pass on a64 (fp64.cu)
    DevArrays64 a64{};
    DevParams64 dp64{};
    double* diag64 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int device = 0;
    int sm_count = 148;
    std::vector<void*> allocations;
    float* staging = nullptr;     // kStagingFloats * n floats: every attribute its own region
    double* staging64 = nullptr;  // 9 * n doubles
    double* diag_out = nullptr;   // device, 12 doubles
    size_t part_cap = 0, gpart_cap = 0, item_cap = 0;  // floats allocated for a.part, a.gpart, sp.item_part
    size_t item_nb_items = 0;                          // work items the neighbour-list buffers hold
    std::vector<void*> snap[4];    // gsph_snapshot slots: saved copies of the state arrays (allocated on first save)
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int64_t graph_kernels = 0;
    int64_t launches = 0;
    // per-kernel timing (gsph_profile_*)
    bool profiling = false;
    KTimer timers[GSPH_KSLOTS];
    bool pending[GSPH_KSLOTS] = {};
    uint32_t graph_slots = 0;      // slots recorded inside the captured step graph
    double prof_ms[GSPH_KSLOTS] = {};
    int64_t prof_launches[GSPH_KSLOTS] = {};
    std::string err;
};

namespace {

thread_local std::string g_create_error;

}  // namespace

// message of a failed call that has no context (read back with gsph_last_error(NULL))
void set_global_error(const std::string& msg) { g_create_error = msg; }

namespace {

int fail(gsph_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}
int cuda_fail(gsph_ctx* c, cudaError_t e, const char* what) {
    return fail(c, GSPH_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define GSPH_CK(ctx, call, what)                          \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

double spline_prefactor(int dim, double h) {  // src/sph/kernel.h:44-60
    if (dim == 1) return 4.0 / (3.0 * h);
    if (dim == 2) return 40.0 / (7.0 * M_PI * h * h);
    return 8.0 / (M_PI * h * h * h);
}
double dspline_prefactor(int dim, double h) {  // src/sph/kernel.h:71-87
    if (dim == 1) return 24.0 / (3.0 * h * h);
    if (dim == 2) return 240.0 / (7.0 * M_PI * h * h * h);
    return 48.0 / (M_PI * h * h * h * h);
}

DevParams make_dev_params(const gsph_params& p) {
    DevParams d{};
    d.flags = p.flags;
    d.dim = p.dimension;
    d.H = static_cast<float>(p.H);
    d.H2 = static_cast<float>(p.H * p.H);
    d.inv_h = static_cast<float>(1.0 / p.H);
    d.eps2 = static_cast<float>(p.grav_eps * p.grav_eps);
    d.G = static_cast<float>(p.grav_G);
    d.w_pref = static_cast<float>(spline_prefactor(p.dimension, p.H));
    d.dw_pref = static_cast<float>(dspline_prefactor(p.dimension, p.H));
    d.rho0 = static_cast<float>(p.rho0);
    d.bulk = static_cast<float>(p.bulk);
    d.dbulk = static_cast<float>(p.dbulk_dp);
    d.c = static_cast<float>(p.soundspeed);
    d.c2 = static_cast<float>(p.soundspeed * p.soundspeed);
    d.shear = static_cast<float>(p.shear);
    d.Y = static_cast<float>(p.Y);
    d.tanfr = static_cast<float>(p.tanfr);
    d.cohesion = static_cast<float>(p.cohesion);
    d.alpha = static_cast<float>(p.av_alpha);
    d.beta = static_cast<float>(p.av_beta);
    d.mateps = static_cast<float>(p.mateps);
    d.matexp = static_cast<float>(p.matexp);
    {  // 1 / W(normalsep) of the artificial stress (computeDerivatives.h:265)
        const double q = p.normalsep / p.H;
        double w = 0.0;
        if (q <= 1.0) w = (q < 0.5) ? (6 * q * q * q - 6 * q * q + 1) : 2 * (1 - q) * (1 - q) * (1 - q);
        w *= spline_prefactor(p.dimension, p.H);
        d.inv_w_normalsep = static_cast<float>(w > 0 ? 1.0 / w : 0.0);
    }
    d.xsph = static_cast<float>(p.xsph_factor);
    d.fixed_dt = static_cast<float>(p.fixed_dt);
    d.initial_dt = static_cast<float>(p.initial_dt);
    d.min_dt = static_cast<float>(p.min_dt);
    d.max_dt = static_cast<float>(p.max_dt);
    d.accel_acc = static_cast<float>(p.accel_accuracy);
    d.vel_acc = static_cast<float>(p.velocity_accuracy);
    d.cw_n = static_cast<float>(p.cw_n);
    for (int k = 0; k < 3; ++k) {
        d.const_acc[k] = static_cast<float>(p.const_acc[k]);
        d.box_min[k] = static_cast<float>(p.box_min[k]);
        d.box_max[k] = static_cast<float>(p.box_max[k]);
    }
    d.box_refl = static_cast<float>(p.box_reflectiveness);
    d.balsara_floor = static_cast<float>(0.0001 * p.soundspeed / p.H);
    d.eps2_d = p.grav_eps * p.grav_eps;
    d.G_d = p.grav_G;
    return d;
}

// smallest j-split whose last wave is at least 95 % full (or the best one up to `cap`)
int pick_split(int64_t iblocks, int slots, int cap) {
    int best = 1;
    double best_eff = 0.0;
    for (int s = 1; s <= cap; ++s) {
        const double w = static_cast<double>(iblocks) * s / slots;
        const double eff = w / std::ceil(w);
        if (eff >= 0.95 && w >= 1.0) return s;
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = s;
        }
    }
    return best;
}

bool is_pow2_in(int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

void* dalloc(gsph_ctx* c, size_t bytes, cudaError_t& e) {
    if (e != cudaSuccess) return nullptr;  // an earlier allocation failed: keep its error
    void* p = nullptr;
    e = cudaMalloc(&p, bytes == 0 ? 16 : bytes);
    if (e == cudaSuccess) c->allocations.push_back(p);
    return p;
}

void drop_graph(gsph_ctx* c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    c->graph_slots = 0;
}

void release(gsph_ctx* c) {
    drop_graph(c);
    if (c->side) cudaStreamSynchronize(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->side) cudaStreamDestroy(c->side);
    c->side = nullptr;
    c->ev_fork = c->ev_join = nullptr;
    for (auto& t : c->timers) {
        if (t.start) cudaEventDestroy(t.start);
        if (t.stop) cudaEventDestroy(t.stop);
        t.start = t.stop = nullptr;
    }
    if (c->capture_stream) cudaStreamDestroy(c->capture_stream);
    for (void* p : c->allocations) cudaFree(p);
    c->allocations.clear();
    for (auto& sl : c->snap) {
        for (void* p : sl)
            if (p) cudaFree(p);
        sl.clear();
    }
}

int check_status(gsph_ctx* c, cudaStream_t s) {
    int st = 0;
    GSPH_CK(c, cudaMemcpyAsync(&st, c->a.status, sizeof(int), cudaMemcpyDeviceToHost, s), "status read");
    GSPH_CK(c, cudaStreamSynchronize(s), "stream synchronize");
    if (st & GSPH_DEV_ERR_TIMEOUT) {  // report once: this call's results are incomplete, the context stays usable
        const int cleared = st & ~GSPH_DEV_ERR_TIMEOUT;
        cudaMemcpyAsync(c->a.status, &cleared, sizeof(int), cudaMemcpyHostToDevice, s);
        cudaStreamSynchronize(s);
        return fail(c, GSPH_E_TIMEOUT, "a device-side wait gave up (j-tile pipeline)");
    }
    if (st & 2) {  // a host-requested scan: report once, then clear the flag
        const int cleared = st & ~2;
        cudaMemcpyAsync(c->a.status, &cleared, sizeof(int), cudaMemcpyHostToDevice, s);
        cudaStreamSynchronize(s);
        return fail(c, GSPH_E_NUMERIC, "non-finite particle state");
    }
    return GSPH_OK;
}

// timer of `slot` when profiling, and mark it pending (collected by gsph_profile_collect)
const KTimer* slot_timer(gsph_ctx* c, int slot) {
    if (!c->profiling) return nullptr;
    c->pending[slot] = true;
    return &c->timers[slot];
}

int derivatives(gsph_ctx* c, cudaStream_t s) {
    const DevParams& p = c->dp;
    cudaError_t e;
    if (c->fp64) {
        int launches = 0;
        e = launch64_derivatives(c->a64, c->dp64, s, launches);
        c->launches += launches;
        if (e != cudaSuccess) return cuda_fail(c, e, "FP64 derivatives");
        return GSPH_OK;
    }
    if (has(p, GSPH_SPH)) {
        const SpatialArrays* sp = c->L.cull ? &c->sp : nullptr;
        const bool grav_kernel = sp && has(p, GSPH_SELF_GRAVITY);
        cudaEvent_t join = nullptr;
        if (grav_kernel) {  // fork: all-pairs gravity on the side stream, joined before the finish
            e = cudaEventRecord(c->ev_fork, s);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(c->side, c->ev_fork, 0);
            if (e == cudaSuccess) e = launch_gravity_partials(c->a, p, c->L, c->side, slot_timer(c, GSPH_KSLOT_GRAVITY));
            if (e == cudaSuccess) e = cudaEventRecord(c->ev_join, c->side);
            if (e != cudaSuccess) return cuda_fail(c, e, "gravity pass");
            join = c->ev_join;
            c->launches += 1;
        }
        if (sp) {  // bounds of every chunk at the current positions, each group's near chunks, work items
            e = launch_chunk_bounds(c->a, c->sp, s);
            if (e == cudaSuccess) e = launch_chunk_lists(c->a, c->sp, p.H, s);
            if (e == cudaSuccess) e = launch_work_items(c->a, c->sp, c->sp.item_target, s);
            if (e != cudaSuccess) return cuda_fail(c, e, "chunk lists");
            c->launches += 3;
        }
        if (!has(p, GSPH_INTEGRATE_DENSITY)) {
            e = launch_density(c->a, p, c->L, s, slot_timer(c, GSPH_KSLOT_DENSITY), sp);
            if (e != cudaSuccess) return cuda_fail(c, e, "density pass");
            c->launches += 2;
        } else {
            e = launch_prepare(c->a, p, s);
            if (e != cudaSuccess) return cuda_fail(c, e, "j-record pass");
            c->launches += 1;
        }
        const bool vgrad = has(p, GSPH_SOLIDS) || has(p, GSPH_INTEGRATE_DENSITY) || has(p, GSPH_BALSARA_SWITCH);
        const int gnseg = grav_kernel ? c->L.grav_nseg : 0;
        const bool lists = sp && !has(p, GSPH_INTEGRATE_DENSITY);  // the density pass stored neighbour lists
        if (vgrad && has(p, GSPH_BALSARA_SWITCH)) {
            e = launch_pairs(PASS_VGRAD, c->a, p, c->L, s, slot_timer(c, GSPH_KSLOT_VGRAD), sp, 0, nullptr, lists);
            if (e != cudaSuccess) return cuda_fail(c, e, "velocity-gradient pass");
            e = launch_pairs(PASS_ACC, c->a, p, c->L, s, slot_timer(c, GSPH_KSLOT_PAIRS), sp, gnseg, join, lists);
            if (e != cudaSuccess) return cuda_fail(c, e, "acceleration pass");
            c->launches += 4;
        } else {
            e = launch_pairs(vgrad ? PASS_FUSED : PASS_ACC, c->a, p, c->L, s, slot_timer(c, GSPH_KSLOT_PAIRS), sp, gnseg,
                             join, lists);
            if (e != cudaSuccess) return cuda_fail(c, e, "pair pass");
            c->launches += 2;
        }
    } else {
        e = launch_gravity(c->a, p, c->L, s,
                           has(p, GSPH_SELF_GRAVITY) ? slot_timer(c, GSPH_KSLOT_GRAVITY) : nullptr);
        if (e != cudaSuccess) return cuda_fail(c, e, "gravity pass");
        c->launches += has(p, GSPH_SELF_GRAVITY) ? 2 : 1;
    }
    return GSPH_OK;
}

int reorder(gsph_ctx* c, cudaStream_t s) {
    if (!c->L.cull) return GSPH_OK;
    int launches = 0;
    const cudaError_t e = reorder_particles(c->a, c->sp, s, launches);
    c->launches += launches;
    c->steps_since_sort = 0;
    if (e != cudaSuccess) return cuda_fail(c, e, "particle reorder");
    return GSPH_OK;
}

const int* ext_map(const gsph_ctx* c) { return c->L.cull ? c->sp.ext_of_int : nullptr; }

int integrate(gsph_ctx* c, int not_first_step, cudaStream_t s) {
    if (c->fp64) {
        int launches = 0;
        const cudaError_t e = launch64_leapfrog(c->a64, c->dp64, not_first_step, s, launches);
        c->launches += launches;
        if (e != cudaSuccess) return cuda_fail(c, e, "FP64 leapfrog");
        return GSPH_OK;
    }
    const KTimer* t = slot_timer(c, GSPH_KSLOT_INTEGRATE);
    cudaError_t e = t ? timer_record(t->start, s) : cudaSuccess;
    if (e == cudaSuccess) e = launch_leapfrog(c->a, c->dp, not_first_step, s);
    if (e == cudaSuccess && t) e = timer_record(t->stop, s);
    if (e != cudaSuccess) return cuda_fail(c, e, "leapfrog");
    c->launches += has(c->dp, GSPH_VARIABLE_TIMESTEP) ? 3 : 1;
    return GSPH_OK;
}

}  // namespace

// the parameter block of the kernels, for the other translation units (ensemble.cu)
DevParams gsph_dev_params(const gsph_params& p) { return make_dev_params(p); }

// the device arrays and the slot -> caller order map of a single-precision context (writer.cu)
bool gsph_ctx_state(gsph_ctx* c, DevArrays* a, const int** ext) {
    if (!c || c->fp64) return false;
    *a = c->a;
    *ext = ext_map(c);
    return true;
}

extern "C" {

int gsph_params_reference_defaults(gsph_params* p) {
    if (!p) return GSPH_E_INVALID;
    std::memset(p, 0, sizeof(*p));
    const double pradius = 0.1 * std::pow(double(1 << 14), -1.0 / 3.0);  // settings.h:97-98
    p->flags = GSPH_SELF_GRAVITY | GSPH_SPH | GSPH_INTEGRATE_DENSITY | GSPH_SOLIDS | GSPH_VARIABLE_TIMESTEP |
               GSPH_ACCELERATION_CRITERION | GSPH_VELOCITY_CRITERION | GSPH_PLASTICITY_MC |
               GSPH_ARTIFICIAL_VISCOSITY | GSPH_BALSARA_SWITCH;
    p->dimension = 3;
    p->H = pradius * 2.5;
    p->grav_eps = p->H;
    p->grav_G = 1.0;
    p->rho0 = 1.0 / (1 << 14) / (4.0 / 3.0 * pradius * pradius * pradius * M_PI);
    p->bulk = 1024;
    p->dbulk_dp = 1;
    p->soundspeed = std::sqrt(p->bulk / p->rho0);
    p->shear = 128;
    p->Y = 0.5;
    p->tanfr = std::tan(45.0 * M_PI / 180.0);
    p->cohesion = 0.0;
    p->av_alpha = 1.0;
    p->av_beta = 3.0;
    p->mateps = 0.4;
    p->matexp = 4.0;
    p->normalsep = p->H * 0.3;
    p->xsph_factor = 0.5;
    p->fixed_dt = 0.002;
    p->initial_dt = 0.002;
    p->min_dt = 0.00002;
    p->max_dt = 0.02;
    p->accel_accuracy = 0.01;
    p->velocity_accuracy = 0.09;
    p->cw_n = std::sqrt(1.0 / 3.0);
    p->const_acc[1] = -1.0;
    for (int k = 0; k < 3; ++k) {
        p->box_min[k] = -1.2;
        p->box_max[k] = 1.2;
    }
    p->box_reflectiveness = 0.5;
    return GSPH_OK;
}

int gsph_params_validate(const gsph_params* p, char* msg, size_t msg_len) {
    auto bad = [&](int code, const char* why) {
        if (msg && msg_len) std::snprintf(msg, msg_len, "%s", why);
        return code;
    };
    if (!p) return bad(GSPH_E_INVALID, "params is NULL");
    if (p->flags & ~GSPH_ALL_FLAGS) return bad(GSPH_E_INVALID, "unknown flag bits");
    if (p->dimension < 1 || p->dimension > 3) return bad(GSPH_E_INVALID, "dimension must be 1, 2 or 3");
    if (!(p->H > 0) || !std::isfinite(p->H)) return bad(GSPH_E_INVALID, "H must be positive and finite");
    if (!(p->grav_eps >= 0) || !std::isfinite(p->grav_eps)) return bad(GSPH_E_INVALID, "grav_eps must be >= 0");
    if ((p->flags & GSPH_PLASTICITY_MIESE) && (p->flags & GSPH_PLASTICITY_MC))
        return bad(GSPH_E_INVALID, "choose up to one plasticity model (settings.h:203-205)");
    if (p->flags & GSPH_SPH) {
        if (!(p->rho0 > 0)) return bad(GSPH_E_INVALID, "rho0 must be positive");
        if ((p->flags & GSPH_SOLIDS) && !(p->dbulk_dp != 0)) return bad(GSPH_E_INVALID, "dbulk_dp must be nonzero");
    }
    if (!(p->flags & GSPH_VARIABLE_TIMESTEP) && !(p->fixed_dt > 0)) return bad(GSPH_E_INVALID, "fixed_dt must be > 0");
    if ((p->flags & GSPH_VARIABLE_TIMESTEP) && !(p->min_dt > 0 && p->max_dt >= p->min_dt && p->initial_dt > 0))
        return bad(GSPH_E_INVALID, "variable step needs 0 < min_dt <= max_dt and initial_dt > 0");
    if (msg && msg_len) msg[0] = 0;
    return GSPH_OK;
}

int gsph_options_defaults(gsph_options* o) {
    if (!o) return GSPH_E_INVALID;
    std::memset(o, 0, sizeof(*o));
    o->accum = GSPH_ACCUM_PLAIN;
    return GSPH_OK;
}

int gsph_create(const gsph_params* p, const gsph_options* opt, int64_t n, gsph_ctx** out) {
    if (!out) return fail(nullptr, GSPH_E_INVALID, "out is NULL");
    *out = nullptr;
    char why[160];
    const int v = gsph_params_validate(p, why, sizeof why);
    if (v != GSPH_OK) return fail(nullptr, v, why);
    if (n < 1 || n > (int64_t(1) << 31)) return fail(nullptr, GSPH_E_INVALID, "n must be in [1, 2^31]");
    gsph_options o;
    if (opt) o = *opt;
    else gsph_options_defaults(&o);
    if (o.accum != GSPH_ACCUM_PLAIN && o.accum != GSPH_ACCUM_COMPENSATED)
        return fail(nullptr, GSPH_E_INVALID, "options.accum must be GSPH_ACCUM_PLAIN or GSPH_ACCUM_COMPENSATED");
    if (o.j_tile && !is_pow2_in(o.j_tile, 64, 1024)) return fail(nullptr, GSPH_E_INVALID, "j_tile: power of 2 in [64,1024]");
    if (o.gravity_form < GSPH_GRAVITY_AUTO || o.gravity_form > GSPH_GRAVITY_SYMMETRIC || o.gravity_groups < 0 ||
        o.gravity_groups > 1024)
        return fail(nullptr, GSPH_E_INVALID, "options.gravity_form must be a GSPH_GRAVITY_* value, gravity_groups in [0, 1024]");
    if (o.threads && o.threads != 64 && o.threads != 128 && o.threads != 256)
        return fail(nullptr, GSPH_E_INVALID, "threads: 64, 128 or 256");
    if (o.i_per_thread && o.i_per_thread != 1 && o.i_per_thread != 2 && o.i_per_thread != 4 && o.i_per_thread != 8)
        return fail(nullptr, GSPH_E_INVALID, "i_per_thread: 1, 2, 4 or 8");
    if (o.j_split < 0 || o.j_split > kMaxSplit) return fail(nullptr, GSPH_E_INVALID, "j_split out of range");
    if (o.precision != GSPH_PRECISION_SINGLE && o.precision != GSPH_PRECISION_DOUBLE)
        return fail(nullptr, GSPH_E_INVALID, "precision must be GSPH_PRECISION_SINGLE or GSPH_PRECISION_DOUBLE");

    gsph_ctx* c = new (std::nothrow) gsph_ctx();
    if (!c) return fail(nullptr, GSPH_E_NOMEM, "host allocation failed");
    c->params = *p;
    c->opt = o;
    c->dp = make_dev_params(*p);
    cudaError_t e = cudaGetDevice(&c->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    if (e != cudaSuccess) {
        delete c;
        return fail(nullptr, GSPH_E_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
    }
    const int64_t n_pad = (n + kPad - 1) / kPad * kPad;
    c->a.n = n;
    c->a.n_pad = n_pad;

    // launch shape
    Launch& L = c->L;
    L.accum = o.accum;
    c->fp64 = o.precision == GSPH_PRECISION_DOUBLE;
    L.cull = (p->flags & GSPH_SPH) && !o.no_cull && !c->fp64;
    L.threads = o.threads ? o.threads : 128;
    L.jt = o.j_tile ? o.j_tile : 256;
    const int64_t ntiles = n_pad / L.jt;
    const int cap = static_cast<int>(std::min<int64_t>(kMaxSplit, std::max<int64_t>(1, ntiles)));
    L.nseg = o.j_split ? std::min(o.j_split, cap) : pick_split(n_pad / L.threads, c->sm_count * 4, cap);
    // gravity kernel: the most i-blocking (and the largest j-tile) that still gives two waves of CTAs
    L.grav_threads = 128;
    L.grav_x2 = !o.scalar_fp32;
    {
        const bool comp = o.accum == GSPH_ACCUM_COMPENSATED;
        const int ipts[3] = {4, 2, 1};
        const int jts[3] = {256, 128, 64};
        int best_i = 1, best_jt = 64;
        bool found = false;
        for (int a = 0; a < 3 && !found; ++a)
            for (int b = 0; b < 3 && !found; ++b) {
                const int64_t iblocks = n_pad / (int64_t(L.grav_threads) * ipts[a]);
                const int64_t maxseg = std::min<int64_t>(kMaxSplit, n_pad / jts[b]);
                const int slots = c->sm_count * gravity_blocks_per_sm(ipts[a], L.grav_threads, jts[b], comp);
                if (iblocks * maxseg >= 2 * slots) {
                    best_i = ipts[a];
                    best_jt = jts[b];
                    found = true;
                }
            }
        L.grav_ipt = o.i_per_thread ? o.i_per_thread : best_i;
        L.grav_jt = o.j_tile ? o.j_tile : best_jt;
        const int64_t gt = n_pad / L.grav_jt;
        const int gcap = static_cast<int>(std::min<int64_t>(kMaxSplit, std::max<int64_t>(1, gt)));
        const int slots = c->sm_count * gravity_blocks_per_sm(L.grav_ipt, L.grav_threads, L.grav_jt, comp);
        L.grav_nseg = o.j_split ? std::min(o.j_split, gcap)
                                : pick_split(n_pad / (int64_t(L.grav_threads) * L.grav_ipt), slots, gcap);
        // the symmetric form: enough tasks (G(G+1)/2 with G up to 64) to fill the GPU twice
        const int64_t nblocks = n_pad / 1024;
        const bool sym = o.gravity_form == GSPH_GRAVITY_SYMMETRIC ||
                         (o.gravity_form == GSPH_GRAVITY_AUTO && !o.scalar_fp32 && nblocks >= 24);
        const bool own_kernel = !(p->flags & GSPH_SPH) || L.cull;  // gravity has a kernel of its own
        if (sym && own_kernel && !c->fp64) sym_groups(nblocks, o.gravity_groups ? o.gravity_groups : 64, L.grav_sym_G, L.grav_sym_gs);
    }

    cudaError_t ae = cudaSuccess;
    auto F4 = [&](void) { return static_cast<float4*>(dalloc(c, n_pad * sizeof(float4), ae)); };
    DevArrays& a = c->a;
    a.posm = F4(); a.velrho = F4(); a.acc = F4(); a.xvel = F4();
    a.sA = F4(); a.sB = F4(); a.dA = F4(); a.dB = F4(); a.jA = F4(); a.jB = F4();
    a.pos64 = static_cast<double*>(dalloc(c, 3 * n_pad * sizeof(double), ae));
    a.rhodot = static_cast<float*>(dalloc(c, n_pad * sizeof(float), ae));
    a.balsara = static_cast<float*>(dalloc(c, n_pad * sizeof(float), ae));
    c->part_cap = partial_floats(c->dp, L, n_pad);
    c->gpart_cap = L.cull ? gravity_partial_floats(L, n_pad) : 4;
    a.part = static_cast<float*>(dalloc(c, c->part_cap * sizeof(float), ae));
    a.gpart = static_cast<float*>(dalloc(c, c->gpart_cap * sizeof(float), ae));
    a.gfold = static_cast<double*>(dalloc(c, (L.cull ? 3 * n_pad : 4) * sizeof(double), ae));
    if (L.cull) {
        SpatialArrays& sp = c->sp;
        const int64_t nchunks = n_pad / kChunk, ngroups = n_pad / kGroup;
        L.item_grid = c->sm_count * 5;      // 41 KB of shared memory and at most 102 registers: 5 per SM
        L.density_grid = c->sm_count * 12;  // 40 registers (launch bound) and 8 KB of shared memory: 12 per SM
        sp.item_target = 6 * L.item_grid;
        sp.item_start = static_cast<int*>(dalloc(c, (ngroups + 2) * sizeof(int), ae));
        // worst case fields per item: fused solids pass without gravity, compensated (x2); items are at
        // most target + one per group (rounding up per group)
        const size_t kk = 2 * static_cast<size_t>(popc_c(field_mask<PASS_FUSED, false, true>()));
        const size_t cap = static_cast<size_t>(sp.item_target) + static_cast<size_t>(ngroups);
        c->item_cap = cap * kk * kGroup;
        sp.item_part = static_cast<float*>(dalloc(c, c->item_cap * sizeof(float), ae));
        c->item_nb_items = cap;
        sp.item_nb = static_cast<int*>(dalloc(c, cap * kItemNb * kGroup * sizeof(int), ae));
        sp.item_nbcnt = static_cast<int*>(dalloc(c, cap * kGroup * sizeof(int), ae));
        sp.item_nbover = static_cast<int*>(dalloc(c, cap * sizeof(int), ae));
        a.jrec = static_cast<float4*>(dalloc(c, 4 * n_pad * sizeof(float4), ae));
        if (ae == cudaSuccess) ae = cudaMemset(a.jrec, 0, 4 * n_pad * sizeof(float4));
        sp.box_lo = static_cast<float4*>(dalloc(c, nchunks * sizeof(float4), ae));
        sp.box_hi = static_cast<float4*>(dalloc(c, nchunks * sizeof(float4), ae));
        sp.list = static_cast<int*>(dalloc(c, static_cast<size_t>(ngroups) * nchunks * sizeof(int), ae));
        sp.count = static_cast<int*>(dalloc(c, ngroups * sizeof(int), ae));
        sp.ext_of_int = static_cast<int*>(dalloc(c, n_pad * sizeof(int), ae));
        sp.order = static_cast<int*>(dalloc(c, n_pad * sizeof(int), ae));
        sp.order_out = static_cast<int*>(dalloc(c, n_pad * sizeof(int), ae));
        sp.keys = static_cast<unsigned*>(dalloc(c, 2 * n_pad * sizeof(unsigned), ae));
        sp.sort_tmp_bytes = spatial_sort_tmp_bytes(n_pad);
        sp.sort_tmp = dalloc(c, sp.sort_tmp_bytes, ae);
        sp.bbox = static_cast<int*>(dalloc(c, 8 * sizeof(int), ae));
        sp.tmp4 = static_cast<float4*>(dalloc(c, n_pad * sizeof(float4), ae));
        sp.tmp8 = static_cast<double*>(dalloc(c, n_pad * sizeof(double), ae));
    }
    a.dt_state = static_cast<float*>(dalloc(c, 4 * sizeof(float), ae));
    a.diag = static_cast<double*>(dalloc(c, diag_scratch_doubles(n) * sizeof(double), ae));
    a.status = static_cast<int*>(dalloc(c, sizeof(int) * 4, ae));
    a.grav = static_cast<float4*>(dalloc(c, n_pad * sizeof(float4), ae));
    if (c->fp64) {
        DevArrays64& b = c->a64;
        b.n = n;
        b.n_pad = n_pad;
        auto D4 = [&](void) { return static_cast<double4*>(dalloc(c, n_pad * sizeof(double4), ae)); };
        b.posm = D4(); b.velrho = D4(); b.acc = D4(); b.xvel = D4(); b.sA = D4(); b.sB = D4();
        b.dA = D4(); b.dB = D4(); b.jA = D4(); b.jB = D4();
        b.rhodot = static_cast<double*>(dalloc(c, n_pad * sizeof(double), ae));
        b.balsara = static_cast<double*>(dalloc(c, n_pad * sizeof(double), ae));
        b.dt_state = static_cast<double*>(dalloc(c, 4 * sizeof(double), ae));
        c->diag64 = static_cast<double*>(dalloc(c, diag64_scratch_doubles(n_pad) * sizeof(double), ae));
        const double q = p->normalsep / p->H;
        double wn = 0.0;
        if (q <= 1.0) wn = (q < 0.5) ? (6 * q * q * q - 6 * q * q + 1) : 2 * (1 - q) * (1 - q) * (1 - q);
        wn *= spline_prefactor(p->dimension, p->H);
        c->dp64 = make_dev_params64(*p, spline_prefactor(p->dimension, p->H), dspline_prefactor(p->dimension, p->H),
                                    wn > 0 ? 1.0 / wn : 0.0);
    }
    c->staging = static_cast<float*>(dalloc(c, kStagingFloats * n * sizeof(float), ae));
    c->staging64 = static_cast<double*>(dalloc(c, 9 * n * sizeof(double), ae));
    c->diag_out = static_cast<double*>(dalloc(c, 16 * sizeof(double), ae));
    if (ae != cudaSuccess) {
        release(c);
        delete c;
        return fail(nullptr, GSPH_E_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(ae));
    }
    e = cudaMemset(a.dt_state, 0, 4 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(a.status, 0, 4 * sizeof(int));
    if (e == cudaSuccess) e = launch_init_padding(a, 0);
    if (e == cudaSuccess && L.cull) e = launch_identity_order(c->sp, n_pad, 0);
    if (e == cudaSuccess && c->fp64) {
        e = launch64_init(c->a64, 0);
        if (e == cudaSuccess) e = cudaMemset(c->a64.dt_state, 0, 4 * sizeof(double));
    }
    if (e == cudaSuccess && L.cull) {
        e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        release(c);
        delete c;
        return fail(nullptr, GSPH_E_CUDA, std::string("context initialisation: ") + cudaGetErrorString(e));
    }
    c->launches = 1;
    *out = c;
    return GSPH_OK;
}

int gsph_destroy(gsph_ctx* c) {
    if (!c) return GSPH_E_INVALID;
    release(c);
    delete c;
    return GSPH_OK;
}

namespace {
int upload_any(gsph_ctx* c, uint32_t mask, const gsph_host_particles* src, void* stream, cudaMemcpyKind kind);
}  // namespace

int gsph_upload(gsph_ctx* c, uint32_t mask, const gsph_host_particles* src, void* stream) {
    return upload_any(c, mask, src, stream, cudaMemcpyHostToDevice);
}

int gsph_upload_device(gsph_ctx* c, uint32_t mask, const gsph_host_particles* src, void* stream) {
    return upload_any(c, mask, src, stream, cudaMemcpyDeviceToDevice);
}

}  // extern "C"

namespace {
int upload_any(gsph_ctx* c, uint32_t mask, const gsph_host_particles* src, void* stream, cudaMemcpyKind kind) {
    if (!c) return GSPH_E_INVALID;
    if (!src) return fail(c, GSPH_E_INVALID, "src is NULL");
    if (mask & ~GSPH_ALL_ATTRIBS) return fail(c, GSPH_E_INVALID, "unknown attribute bits in mask");
    const float* ptrs[11] = {src->pos, src->mass, src->vel, src->acc, src->balsara, src->xvel,
                             src->density, src->density_dt, src->dstress, src->dstress_dt, src->maxvsig};
    static const int comps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};
    for (int k = 0; k < 11; ++k)
        if ((mask >> k & 1u) && !ptrs[k]) return fail(c, GSPH_E_INVALID, "attribute pointer is NULL for a set mask bit");
    cudaStream_t s = as_stream(stream);
    // every attribute into its own staging region, all copies first: they run back to back on the copy
    // engine instead of each waiting for the previous attribute's pack kernel
    int64_t off[11];
    int64_t o = 0;
    for (int k = 0; k < 11; ++k) {
        off[k] = o;
        if (!(mask >> k & 1u)) continue;
        GSPH_CK(c, cudaMemcpyAsync(c->staging + o, ptrs[k], comps[k] * c->a.n * sizeof(float), kind, s), "upload copy");
        o += comps[k] * c->a.n;
    }
    for (int k = 0; k < 11; ++k) {
        if (!(mask >> k & 1u)) continue;
        if (c->fp64) GSPH_CK(c, launch64_pack(c->a64, k, c->staging + off[k], s), "upload pack");
        else GSPH_CK(c, launch_pack(c->a, k, c->staging + off[k], ext_map(c), s), "upload pack");
        c->launches += 1;
    }
    if (mask & GSPH_POS) {
        const int rc = reorder(c, s);
        if (rc != GSPH_OK) return rc;
    }
    if (c->opt.check_finite) {
        GSPH_CK(c, launch_check_finite(c->a, s), "finite check");
        c->launches += 1;
        return check_status(c, s);
    }
    return GSPH_OK;
}
}  // namespace

extern "C" {

int gsph_download(gsph_ctx* c, uint32_t mask, gsph_host_particles* dst, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (!dst) return fail(c, GSPH_E_INVALID, "dst is NULL");
    if (mask & ~GSPH_ALL_ATTRIBS) return fail(c, GSPH_E_INVALID, "unknown attribute bits in mask");
    float* ptrs[11] = {dst->pos, dst->mass, dst->vel, dst->acc, dst->balsara, dst->xvel,
                       dst->density, dst->density_dt, dst->dstress, dst->dstress_dt, dst->maxvsig};
    static const int comps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};
    for (int k = 0; k < 11; ++k)
        if ((mask >> k & 1u) && !ptrs[k]) return fail(c, GSPH_E_INVALID, "attribute pointer is NULL for a set mask bit");
    cudaStream_t s = as_stream(stream);
    // all unpack kernels into their own staging regions first, then the copies back to back
    int64_t off[11];
    int64_t o = 0;
    for (int k = 0; k < 11; ++k) {
        off[k] = o;
        if (!(mask >> k & 1u)) continue;
        if (c->fp64) GSPH_CK(c, launch64_unpack(c->a64, k, c->staging + o, s), "download unpack");
        else GSPH_CK(c, launch_unpack(c->a, k, c->staging + o, ext_map(c), s), "download unpack");
        c->launches += 1;
        o += comps[k] * c->a.n;
    }
    for (int k = 0; k < 11; ++k) {
        if (!(mask >> k & 1u)) continue;
        GSPH_CK(c, cudaMemcpyAsync(ptrs[k], c->staging + off[k], comps[k] * c->a.n * sizeof(float),
                                   cudaMemcpyDeviceToHost, s),
                "download copy");
    }
    return check_status(c, s);
}

int gsph_upload_f64(gsph_ctx* c, uint32_t mask, const gsph_host_particles64* src, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (!src) return fail(c, GSPH_E_INVALID, "src is NULL");
    if (mask & ~GSPH_ALL_ATTRIBS) return fail(c, GSPH_E_INVALID, "unknown attribute bits in mask");
    const double* ptrs[11] = {src->pos, src->mass, src->vel, src->acc, src->balsara, src->xvel,
                              src->density, src->density_dt, src->dstress, src->dstress_dt, src->maxvsig};
    static const int comps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};
    for (int k = 0; k < 11; ++k)
        if ((mask >> k & 1u) && !ptrs[k]) return fail(c, GSPH_E_INVALID, "attribute pointer is NULL for a set mask bit");
    cudaStream_t s = as_stream(stream);
    for (int k = 0; k < 11; ++k) {
        if (!(mask >> k & 1u)) continue;
        const int64_t cnt = comps[k] * c->a.n;
        GSPH_CK(c, cudaMemcpyAsync(c->staging64, ptrs[k], cnt * sizeof(double), cudaMemcpyHostToDevice, s),
                "upload copy");
        if (c->fp64) {
            GSPH_CK(c, launch64_pack_f64(c->a64, k, c->staging64, s), "upload pack");
        } else {
            GSPH_CK(c, launch_narrow(c->staging64, c->staging, cnt, s), "upload narrow");
            GSPH_CK(c, launch_pack(c->a, k, c->staging, ext_map(c), s), "upload pack");
            if (k == 0) GSPH_CK(c, launch_pack_pos64(c->a, c->staging64, ext_map(c), s), "upload pack");
            c->launches += 1 + (k == 0);
        }
        c->launches += 1;
    }
    if (mask & GSPH_POS) return reorder(c, s);
    return GSPH_OK;
}

int gsph_download_f64(gsph_ctx* c, uint32_t mask, gsph_host_particles64* dst, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (!dst) return fail(c, GSPH_E_INVALID, "dst is NULL");
    if (mask & ~GSPH_ALL_ATTRIBS) return fail(c, GSPH_E_INVALID, "unknown attribute bits in mask");
    double* ptrs[11] = {dst->pos, dst->mass, dst->vel, dst->acc, dst->balsara, dst->xvel,
                        dst->density, dst->density_dt, dst->dstress, dst->dstress_dt, dst->maxvsig};
    static const int comps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};
    for (int k = 0; k < 11; ++k)
        if ((mask >> k & 1u) && !ptrs[k]) return fail(c, GSPH_E_INVALID, "attribute pointer is NULL for a set mask bit");
    cudaStream_t s = as_stream(stream);
    for (int k = 0; k < 11; ++k) {
        if (!(mask >> k & 1u)) continue;
        const int64_t cnt = comps[k] * c->a.n;
        if (c->fp64) {
            GSPH_CK(c, launch64_unpack_f64(c->a64, k, c->staging64, s), "download unpack");
        } else if (k == 0) {
            GSPH_CK(c, launch_unpack_pos64(c->a, c->staging64, ext_map(c), s), "download unpack");
        } else {
            GSPH_CK(c, launch_unpack(c->a, k, c->staging, ext_map(c), s), "download unpack");
            GSPH_CK(c, launch_widen(c->staging, c->staging64, cnt, s), "download widen");
            c->launches += 1;
        }
        c->launches += 1;
        GSPH_CK(c, cudaMemcpyAsync(ptrs[k], c->staging64, cnt * sizeof(double), cudaMemcpyDeviceToHost, s),
                "download copy");
    }
    return check_status(c, s);
}

int gsph_upload_pos64(gsph_ctx* c, const double* pos, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (!pos) return fail(c, GSPH_E_INVALID, "pos is NULL");
    cudaStream_t s = as_stream(stream);
    GSPH_CK(c, cudaMemcpyAsync(c->staging64, pos, 3 * c->a.n * sizeof(double), cudaMemcpyHostToDevice, s), "upload copy");
    if (c->fp64) GSPH_CK(c, launch64_pack_pos(c->a64, c->staging64, s), "upload pack");
    else GSPH_CK(c, launch_pack_pos64(c->a, c->staging64, ext_map(c), s), "upload pack");
    c->launches += 1;
    return reorder(c, s);
}

int gsph_download_pos64(gsph_ctx* c, double* pos, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (!pos) return fail(c, GSPH_E_INVALID, "pos is NULL");
    cudaStream_t s = as_stream(stream);
    if (c->fp64) GSPH_CK(c, launch64_unpack_d(c->a64, 0, c->staging64, s), "download unpack");
    else GSPH_CK(c, launch_unpack_pos64(c->a, c->staging64, ext_map(c), s), "download unpack");
    c->launches += 1;
    GSPH_CK(c, cudaMemcpyAsync(pos, c->staging64, 3 * c->a.n * sizeof(double), cudaMemcpyDeviceToHost, s), "download copy");
    return check_status(c, s);
}

int gsph_compute_derivatives(gsph_ctx* c, void* stream) {
    if (!c) return GSPH_E_INVALID;
    return derivatives(c, as_stream(stream));
}

int gsph_integrate(gsph_ctx* c, int not_first_step, void* stream) {
    if (!c) return GSPH_E_INVALID;
    return integrate(c, not_first_step, as_stream(stream));
}

int gsph_step(gsph_ctx* c, int32_t nsteps, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (nsteps < 0) return fail(c, GSPH_E_INVALID, "nsteps < 0");
    if (nsteps == 0) return GSPH_OK;
    cudaStream_t s = as_stream(stream);
    if (!c->graph_exec) {
        if (!c->capture_stream) GSPH_CK(c, cudaStreamCreateWithFlags(&c->capture_stream, cudaStreamNonBlocking), "stream");
        const int64_t before = c->launches;
        bool was_pending[GSPH_KSLOTS];
        for (int k = 0; k < GSPH_KSLOTS; ++k) {
            was_pending[k] = c->pending[k];
            c->pending[k] = false;
        }
        GSPH_CK(c, cudaStreamBeginCapture(c->capture_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = GSPH_OK;
        const KTimer* st = slot_timer(c, GSPH_KSLOT_STEP);
        if (st) {
            const cudaError_t te = timer_record(st->start, c->capture_stream);
            if (te != cudaSuccess) rc = cuda_fail(c, te, "timer");
        }
        if (rc == GSPH_OK) rc = derivatives(c, c->capture_stream);
        if (rc == GSPH_OK) rc = integrate(c, 1, c->capture_stream);
        if (rc == GSPH_OK && st) {
            const cudaError_t te = timer_record(st->stop, c->capture_stream);
            if (te != cudaSuccess) rc = cuda_fail(c, te, "timer");
        }
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(c->capture_stream, &g);
        c->launches = before;
        uint32_t slots = 0;
        for (int k = 0; k < GSPH_KSLOTS; ++k) {
            if (c->pending[k]) slots |= 1u << k;
            c->pending[k] = was_pending[k];
        }
        if (rc != GSPH_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ee != cudaSuccess) return cuda_fail(c, ee, "end capture");
        cudaGraphExec_t ex = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
        if (ie != cudaSuccess) {
            cudaGraphDestroy(g);
            return cuda_fail(c, ie, "graph instantiate");
        }
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        int64_t kernels = 0;
        if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
        for (auto nd : nodes) {
            cudaGraphNodeType ty;
            if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++kernels;
        }
        c->graph = g;
        c->graph_exec = ex;
        c->graph_kernels = kernels;
        c->graph_slots = slots;
    }
    for (int32_t k = 0; k < nsteps; ++k) {
        if (c->L.cull && c->opt.resort_interval > 0 && c->steps_since_sort >= c->opt.resort_interval) {
            const int rc = reorder(c, s);  // permutes in place: the graph's pointers stay valid
            if (rc != GSPH_OK) return rc;
        }
        GSPH_CK(c, cudaGraphLaunch(c->graph_exec, s), "graph launch");
        c->launches += c->graph_kernels;
        c->steps_since_sort += 1;
    }
    for (int k = 0; k < GSPH_KSLOTS; ++k)
        if (c->graph_slots >> k & 1u) c->pending[k] = true;
    return GSPH_OK;
}

int gsph_current_timestep(gsph_ctx* c, double* dt, void* stream) {
    if (!c || !dt) return c ? fail(c, GSPH_E_INVALID, "dt is NULL") : GSPH_E_INVALID;
    if (!(c->params.flags & GSPH_VARIABLE_TIMESTEP)) {
        // f1_t fixed_timestep: float, or double in the double-precision mode
        *dt = c->fp64 ? c->params.fixed_dt : static_cast<float>(c->params.fixed_dt);
        return GSPH_OK;
    }
    cudaStream_t s = as_stream(stream);
    if (c->fp64) {
        double d = 0.0;
        GSPH_CK(c, cudaMemcpyAsync(&d, c->a64.dt_state, sizeof(double), cudaMemcpyDeviceToHost, s), "timestep read");
        GSPH_CK(c, cudaStreamSynchronize(s), "stream synchronize");
        *dt = d;
        return GSPH_OK;
    }
    float v = 0.0f;
    GSPH_CK(c, cudaMemcpyAsync(&v, c->a.dt_state, sizeof(float), cudaMemcpyDeviceToHost, s), "timestep read");
    GSPH_CK(c, cudaStreamSynchronize(s), "stream synchronize");
    *dt = v;
    return GSPH_OK;
}

namespace {
int diagnostics(gsph_ctx* c, double half_kick, gsph_diag* out, void* stream, bool fast) {
    if (!c) return GSPH_E_INVALID;
    if (!out) return fail(c, GSPH_E_INVALID, "out is NULL");
    cudaStream_t s = as_stream(stream);
    if (c->fp64) GSPH_CK(c, launch64_diagnostics(c->a64, c->dp64, half_kick, c->diag64, c->diag_out, s), "diagnostics");
    else if (fast) GSPH_CK(c, launch_diagnostics_fast(c->a, c->dp, half_kick, c->diag_out, s), "diagnostics");
    else GSPH_CK(c, launch_diagnostics(c->a, c->dp, half_kick, c->diag_out, s), "diagnostics");
    c->launches += 2;
    double h[12];
    GSPH_CK(c, cudaMemcpyAsync(h, c->diag_out, sizeof h, cudaMemcpyDeviceToHost, s), "diagnostics read");
    const int rc = check_status(c, s);
    if (rc != GSPH_OK) return rc;
    out->e_kin = h[0];
    out->e_grav = h[1];
    out->e_int = h[2];
    out->e_shear = h[3];
    for (int k = 0; k < 3; ++k) {
        out->momentum[k] = h[4 + k];
        out->ang_mom[k] = h[7 + k];
    }
    out->mass = h[10];
    return GSPH_OK;
}
}  // namespace

int gsph_diagnostics(gsph_ctx* c, double half_kick, gsph_diag* out, void* stream) {
    return diagnostics(c, half_kick, out, stream, false);
}

int gsph_diagnostics_fast(gsph_ctx* c, double half_kick, gsph_diag* out, void* stream) {
    return diagnostics(c, half_kick, out, stream, true);
}

int gsph_reorder(gsph_ctx* c, void* stream) {
    if (!c) return GSPH_E_INVALID;
    return reorder(c, as_stream(stream));
}

int gsph_surrogate_features(gsph_ctx* c, const float* mu, const float* sigma, float* feat, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (!feat || (!mu) != (!sigma)) return fail(c, GSPH_E_INVALID, "feat is NULL, or only one of mu / sigma given");
    if (c->fp64 || !c->L.cull || !(c->params.flags & GSPH_SPH))
        return fail(c, GSPH_E_UNSUPPORTED, "features need an SPH context in single precision with culling");
    cudaStream_t s = as_stream(stream);
    GSPH_CK(c, launch_chunk_bounds(c->a, c->sp, s), "chunk bounds");
    GSPH_CK(c, launch_chunk_lists(c->a, c->sp, c->dp.H, s), "chunk lists");
    GSPH_CK(c, launch_features(c->a, c->dp, c->sp, mu, sigma, feat, s), "features");
    c->launches += 3;
    return GSPH_OK;
}

int gsph_surrogate_apply(gsph_ctx* c, const float* delta, const float* out_mu, const float* out_sigma, int32_t K,
                         void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (K < 1 || (delta && (!out_mu || !out_sigma))) return fail(c, GSPH_E_INVALID, "K < 1, or delta without scales");
    if (c->fp64 || (c->params.flags & GSPH_VARIABLE_TIMESTEP))
        return fail(c, GSPH_E_UNSUPPORTED, "proposals need the fixed step in single precision");
    GSPH_CK(c, launch_apply(c->a, c->dp, ext_map(c), delta, out_mu, out_sigma, K, as_stream(stream)), "apply");
    c->launches += 1;
    return GSPH_OK;
}

int gsph_snapshot(gsph_ctx* c, int32_t slot, int32_t restore, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (c->fp64) return fail(c, GSPH_E_UNSUPPORTED, "snapshots are single-precision only");
    if (slot < 0 || slot >= kSnapSlots) return fail(c, GSPH_E_INVALID, "snapshot slot out of range");
    std::vector<void*>& snap = c->snap[slot];
    const int64_t np = c->a.n_pad;
    struct Arr { void* p; size_t bytes; };
    const Arr arrs[] = {
        {c->a.posm, np * sizeof(float4)}, {c->a.velrho, np * sizeof(float4)}, {c->a.acc, np * sizeof(float4)},
        {c->a.xvel, np * sizeof(float4)}, {c->a.sA, np * sizeof(float4)}, {c->a.sB, np * sizeof(float4)},
        {c->a.dA, np * sizeof(float4)}, {c->a.dB, np * sizeof(float4)}, {c->a.jA, np * sizeof(float4)},
        {c->a.jB, np * sizeof(float4)}, {c->a.pos64, 3 * np * sizeof(double)}, {c->a.rhodot, np * sizeof(float)},
        {c->a.balsara, np * sizeof(float)}, {c->a.dt_state, 4 * sizeof(float)},
        {c->L.cull ? c->sp.ext_of_int : nullptr, np * sizeof(int)}};
    const int na = static_cast<int>(sizeof(arrs) / sizeof(arrs[0]));
    cudaStream_t s = as_stream(stream);
    if (!restore && snap.empty()) {
        for (int k = 0; k < na; ++k) {
            void* p = nullptr;
            if (arrs[k].p) {
                const cudaError_t e = cudaMalloc(&p, arrs[k].bytes);
                if (e != cudaSuccess) {
                    for (void* q : snap) cudaFree(q);
                    snap.clear();
                    return fail(c, GSPH_E_NOMEM, "snapshot allocation failed");
                }
            }
            snap.push_back(p);
        }
    }
    if (restore && snap.empty()) return fail(c, GSPH_E_STATE, "no snapshot saved");
    for (int k = 0; k < na; ++k) {
        if (!arrs[k].p) continue;
        GSPH_CK(c, cudaMemcpyAsync(restore ? arrs[k].p : snap[k], restore ? snap[k] : arrs[k].p, arrs[k].bytes,
                                   cudaMemcpyDeviceToDevice, s), "snapshot copy");
    }
    return GSPH_OK;
}

}  // extern "C"

namespace {

// replace the tracked allocation *p by one of `floats` floats when it holds fewer (contents are scratch)
int grow(gsph_ctx* c, float** p, size_t& cap, size_t floats) {
    if (floats <= cap) return GSPH_OK;
    float* q = nullptr;
    GSPH_CK(c, cudaMalloc(&q, floats * sizeof(float)), "autotune allocation");
    for (auto& a : c->allocations)
        if (a == *p) a = q;
    cudaFree(*p);
    *p = q;
    cap = floats;
    return GSPH_OK;
}

// median over `reps` launches of f(stream), in ms (events on the stream, after one warm-up)
template <typename F>
int time_ms(gsph_ctx* c, cudaStream_t s, int reps, F&& f, float& ms) {
    cudaEvent_t e0, e1;
    GSPH_CK(c, cudaEventCreate(&e0), "event");
    GSPH_CK(c, cudaEventCreate(&e1), "event");
    std::vector<float> t;
    int rc = f();
    for (int r = 0; r < reps && rc == GSPH_OK; ++r) {
        cudaEventRecord(e0, s);
        rc = f();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float x = 0.0f;
        cudaEventElapsedTime(&x, e0, e1);
        t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != GSPH_OK) return rc;
    std::sort(t.begin(), t.end());
    ms = t.empty() ? 0.0f : t[t.size() / 2];
    return check_status(c, s);
}

}  // namespace

extern "C" {

int gsph_autotune(gsph_ctx* c, int32_t reps, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (c->fp64) return GSPH_OK;  // the double-precision passes have a fixed shape
    if (reps < 1) reps = 3;
    cudaStream_t s = as_stream(stream);
    Launch& L = c->L;
    const int64_t np = c->a.n_pad;
    const bool comp = L.accum == GSPH_ACCUM_COMPENSATED;
    const bool sph = has(c->dp, GSPH_SPH), grav = has(c->dp, GSPH_SELF_GRAVITY);
    const bool profiling = c->profiling;
    c->profiling = false;
    int rc = GSPH_OK;
    // 1. the all-pairs gravity kernel (its own pass in the culled and the gravity-only paths)
    if (grav && (L.cull || !sph)) {
        Launch best = L;
        float best_ms = 1e30f;
        const int ipts[3] = {2, 4, 8};
        const int jts[3] = {128, 256, 512};
        for (int ip : ipts)
            for (int jt : jts) {
                if (np % (int64_t(L.grav_threads) * ip) || np % jt) continue;
                const int64_t iblocks = np / (int64_t(L.grav_threads) * ip);
                const int gcap = static_cast<int>(std::min<int64_t>(kMaxSplit, np / jt));
                const int slots = c->sm_count * gravity_blocks_per_sm(ip, L.grav_threads, jt, comp);
                const int s0 = pick_split(iblocks, slots, gcap);
                const int segs[3] = {std::max(1, s0 / 2), s0, std::min(gcap, 2 * s0)};
                for (int k = 0; k < 3; ++k) {
                    if (k > 0 && segs[k] == segs[k - 1]) continue;
                    Launch t = L;
                    t.grav_sym_G = t.grav_sym_gs = 0;
                    t.grav_ipt = ip;
                    t.grav_jt = jt;
                    t.grav_nseg = segs[k];
                    if (L.cull) rc = grow(c, &c->a.gpart, c->gpart_cap, gravity_partial_floats(t, np));
                    else rc = grow(c, &c->a.part, c->part_cap, partial_floats(c->dp, t, np));
                    if (rc != GSPH_OK) break;
                    float ms = 0.0f;
                    rc = time_ms(c, s, reps, [&]() {
                        const cudaError_t e = L.cull ? launch_gravity_partials(c->a, c->dp, t, s)
                                                     : launch_gravity(c->a, c->dp, t, s);
                        return e == cudaSuccess ? GSPH_OK : cuda_fail(c, e, "autotune gravity");
                    }, ms);
                    if (rc != GSPH_OK) break;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = t;
                    }
                }
                if (rc != GSPH_OK) break;
            }
        // the symmetric form (unless one-sided was asked for) with 32, 64 and 128 groups at most
        const int64_t nblocks = np / 1024;
        const int form = c->opt.gravity_form;
        if (rc == GSPH_OK && form != GSPH_GRAVITY_ONE_SIDED && (form == GSPH_GRAVITY_SYMMETRIC || nblocks >= 8)) {
            int last_G = -1;
            for (int target : {32, 64, 128}) {
                Launch t = best;
                sym_groups(nblocks, c->opt.gravity_groups ? c->opt.gravity_groups : target, t.grav_sym_G, t.grav_sym_gs);
                if (t.grav_sym_G == last_G) continue;
                last_G = t.grav_sym_G;
                if (L.cull) rc = grow(c, &c->a.gpart, c->gpart_cap, gravity_partial_floats(t, np));
                else rc = grow(c, &c->a.part, c->part_cap, partial_floats(c->dp, t, np));
                if (rc != GSPH_OK) break;
                float ms = 0.0f;
                rc = time_ms(c, s, reps, [&]() {
                    const cudaError_t e = L.cull ? launch_gravity_partials(c->a, c->dp, t, s) : launch_gravity(c->a, c->dp, t, s);
                    return e == cudaSuccess ? GSPH_OK : cuda_fail(c, e, "autotune gravity");
                }, ms);
                if (rc != GSPH_OK) break;
                if (ms < best_ms || form == GSPH_GRAVITY_SYMMETRIC && best.grav_sym_G == 0) {
                    best_ms = ms;
                    best = t;
                }
            }
        }
        if (rc == GSPH_OK) {
            L.grav_ipt = best.grav_ipt;
            L.grav_jt = best.grav_jt;
            L.grav_nseg = best.grav_nseg;
            L.grav_sym_G = best.grav_sym_G;
            L.grav_sym_gs = best.grav_sym_gs;
        }
    }
    // 2. the SPH passes: work items of the culled kernels, or the all-pairs tile shape
    if (rc == GSPH_OK && sph) {
        Launch best = L;
        float best_ms = 1e30f;
        std::vector<Launch> cands;
        if (L.cull) {
            for (int f : {3, 6, 12, 24}) {
                Launch t = L;
                t.item_grid = L.item_grid;
                cands.push_back(t);
                cands.back().nseg = -f;  // marks the item multiple (restored below)
            }
        } else {
            for (int th : {64, 128, 256})
                for (int jt : {128, 256, 512}) {
                    if (np % jt || np % th) continue;
                    const int cap = static_cast<int>(std::min<int64_t>(kMaxSplit, np / jt));
                    const int s0 = pick_split(np / th, c->sm_count * 4, cap);
                    for (int sg : {std::max(1, s0 / 2), s0, std::min(cap, 2 * s0)}) {
                        Launch t = L;
                        t.threads = th;
                        t.jt = jt;
                        t.nseg = sg;
                        cands.push_back(t);
                    }
                }
        }
        const int ngroups = static_cast<int>(np / kGroup);
        const size_t kk = 2 * static_cast<size_t>(popc_c(field_mask<PASS_FUSED, false, true>()));
        for (Launch t : cands) {
            const int target_mult = t.nseg < 0 ? -t.nseg : 0;
            if (target_mult) {
                t.nseg = L.nseg;
                const size_t items = static_cast<size_t>(target_mult) * L.item_grid + ngroups;
                rc = grow(c, &c->sp.item_part, c->item_cap, items * kk * kGroup);
                if (rc == GSPH_OK && items > c->item_nb_items) {
                    size_t cap_nb = c->item_nb_items * kItemNb * kGroup, cap_cnt = c->item_nb_items * kGroup,
                           cap_over = c->item_nb_items;
                    rc = grow(c, reinterpret_cast<float**>(&c->sp.item_nb), cap_nb, items * kItemNb * kGroup);
                    if (rc == GSPH_OK)
                        rc = grow(c, reinterpret_cast<float**>(&c->sp.item_nbcnt), cap_cnt, items * kGroup);
                    if (rc == GSPH_OK)
                        rc = grow(c, reinterpret_cast<float**>(&c->sp.item_nbover), cap_over, items);
                    if (rc == GSPH_OK) c->item_nb_items = items;
                }
                if (rc != GSPH_OK) break;
                c->sp.item_target = target_mult * L.item_grid;
            } else {
                rc = grow(c, &c->a.part, c->part_cap, partial_floats(c->dp, t, np));
                if (rc != GSPH_OK) break;
            }
            const Launch saved = L;
            L = t;
            float ms = 0.0f;
            rc = time_ms(c, s, reps, [&]() { return derivatives(c, s); }, ms);
            L = saved;
            if (rc != GSPH_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = t;
                if (target_mult) best.item_grid = -target_mult;  // remembered as a multiple
            }
        }
        if (rc == GSPH_OK) {
            if (L.cull) {
                c->sp.item_target = -best.item_grid * L.item_grid;
            } else {
                L.threads = best.threads;
                L.jt = best.jt;
                L.nseg = best.nseg;
            }
        }
    }
    c->profiling = profiling;
    drop_graph(c);  // the next gsph_step captures the new shapes
    return rc;
}

int gsph_launch_shape_get(gsph_ctx* c, gsph_launch_shape* out) {
    if (!c || !out) return GSPH_E_INVALID;
    std::memset(out, 0, sizeof *out);
    out->cull = c->L.cull;
    out->grav_ipt = c->L.grav_ipt;
    out->grav_jt = c->L.grav_jt;
    out->grav_nseg = c->L.grav_nseg;
    out->grav_x2 = c->L.grav_x2;
    out->grav_sym_groups = c->L.grav_sym_G;
    out->sph_threads = c->L.threads;
    out->sph_jt = c->L.jt;
    out->sph_nseg = c->L.nseg;
    out->items = c->L.cull ? c->sp.item_target : 0;
    return GSPH_OK;
}

}  // extern "C"

namespace {
// gsph_state_compare and gsph_state_compare_parts: the first `nout` (<= 8) fields of k_state_compare
int state_compare(gsph_ctx* c, int32_t slot_p, int32_t slot_0, double* out, int nout, void* stream) {
    if (!c || !out) return c ? fail(c, GSPH_E_INVALID, "out is NULL") : GSPH_E_INVALID;
    if (c->fp64) return fail(c, GSPH_E_UNSUPPORTED, "single precision only");
    if (slot_p < 0 || slot_p >= kSnapSlots || slot_0 < 0 || slot_0 >= kSnapSlots || c->snap[slot_p].empty() ||
        c->snap[slot_0].empty())
        return fail(c, GSPH_E_STATE, "both snapshot slots must hold a saved state");
    auto view = [&](int slot) {  // the saved arrays, in gsph_snapshot's order
        DevArrays v = c->a;
        const std::vector<void*>& sn = c->snap[slot];
        v.posm = static_cast<float4*>(sn[0]);
        v.velrho = static_cast<float4*>(sn[1]);
        v.acc = static_cast<float4*>(sn[2]);
        v.sA = static_cast<float4*>(sn[4]);
        v.sB = static_cast<float4*>(sn[5]);
        v.pos64 = static_cast<double*>(sn[10]);
        return v;
    };
    cudaStream_t s = as_stream(stream);
    GSPH_CK(c, launch_state_compare(c->a, view(slot_p), view(slot_0), c->dp, c->a.diag, c->diag_out, s), "compare");
    c->launches += 2;
    double h[8];
    GSPH_CK(c, cudaMemcpyAsync(h, c->diag_out, sizeof h, cudaMemcpyDeviceToHost, s), "compare read");
    const int rc = check_status(c, s);
    if (rc != GSPH_OK) return rc;
    for (int k = 0; k < nout; ++k) out[k] = h[k];
    return GSPH_OK;
}
}  // namespace

extern "C" {

int gsph_state_compare(gsph_ctx* c, int32_t slot_p, int32_t slot_0, double* out, void* stream) {
    return state_compare(c, slot_p, slot_0, out, 4, stream);
}

int gsph_state_compare_parts(gsph_ctx* c, int32_t slot_p, int32_t slot_0, double* out, void* stream) {
    return state_compare(c, slot_p, slot_0, out, 8, stream);
}

int gsph_energy_adjust(gsph_ctx* c, double d_kin, double d_shear, void* stream) {
    if (!c) return GSPH_E_INVALID;
    if (c->fp64) return fail(c, GSPH_E_UNSUPPORTED, "single precision only");
    if (!std::isfinite(d_kin) || !std::isfinite(d_shear)) return fail(c, GSPH_E_INVALID, "energy changes must be finite");
    GSPH_CK(c, launch_energy_adjust(c->a, c->dp, d_kin, d_shear, c->diag_out, as_stream(stream)), "energy adjust");
    c->launches += 3;
    return GSPH_OK;
}

int gsph_size(gsph_ctx* c, int64_t* n) {
    if (!c || !n) return GSPH_E_INVALID;
    *n = c->a.n;
    return GSPH_OK;
}

const char* gsph_last_error(gsph_ctx* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int gsph_device_view_get(gsph_ctx* c, gsph_device_view* v) {
    if (!c || !v) return GSPH_E_INVALID;
    v->n = c->a.n;
    v->posm = c->a.posm;
    v->velrho = c->a.velrho;
    v->acc = c->a.acc;
    v->pos64 = c->a.pos64;
    return GSPH_OK;
}

int gsph_launch_count(gsph_ctx* c, int64_t* count) {
    if (!c || !count) return GSPH_E_INVALID;
    *count = c->launches;
    return GSPH_OK;
}

int gsph_profile_enable(gsph_ctx* c, int on) {
    if (!c) return GSPH_E_INVALID;
    if ((on != 0) == c->profiling) return GSPH_OK;
    drop_graph(c);
    if (on)
        for (auto& t : c->timers) {
            if (!t.start) GSPH_CK(c, cudaEventCreate(&t.start), "event create");
            if (!t.stop) GSPH_CK(c, cudaEventCreate(&t.stop), "event create");
        }
    c->profiling = on != 0;
    for (bool& b : c->pending) b = false;
    return GSPH_OK;
}

int gsph_profile_collect(gsph_ctx* c) {
    if (!c) return GSPH_E_INVALID;
    for (int k = 0; k < GSPH_KSLOTS; ++k) {
        if (!c->pending[k] || !c->timers[k].stop) continue;
        GSPH_CK(c, cudaEventSynchronize(c->timers[k].stop), "event synchronize");
        float ms = 0.0f;
        GSPH_CK(c, cudaEventElapsedTime(&ms, c->timers[k].start, c->timers[k].stop), "event elapsed");
        c->prof_ms[k] += ms;
        c->prof_launches[k] += 1;
        c->pending[k] = false;
    }
    return GSPH_OK;
}

int gsph_profile_read(gsph_ctx* c, gsph_profile* out) {
    if (!c || !out) return GSPH_E_INVALID;
    for (int k = 0; k < GSPH_KSLOTS; ++k) {
        out->ms[k] = c->prof_ms[k];
        out->launches[k] = c->prof_launches[k];
    }
    return GSPH_OK;
}

int gsph_profile_reset(gsph_ctx* c) {
    if (!c) return GSPH_E_INVALID;
    for (int k = 0; k < GSPH_KSLOTS; ++k) {
        c->prof_ms[k] = 0.0;
        c->prof_launches[k] = 0;
    }
    return GSPH_OK;
}

int gsph_measure_fp32_peak(double seconds, double* tflops) {
    if (!tflops || !(seconds > 0)) return fail(nullptr, GSPH_E_INVALID, "bad arguments");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float* sink = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&sink, 4096 * sizeof(float));
    cudaEvent_t a = nullptr, b = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    int iters = 256;
    double best = 0.0;
    for (int round = 0; e == cudaSuccess && round < 12; ++round) {
        e = cudaEventRecord(a, 0);
        if (e == cudaSuccess) e = launch_fp32_peak(sms, iters, sink, 0);
        if (e == cudaSuccess) e = cudaEventRecord(b, 0);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e != cudaSuccess) break;
        const double tf = static_cast<double>(fp32_peak_flops(sms, iters)) / (ms * 1e-3) / 1e12;
        if (ms > 0.25 * seconds * 1e3) best = std::max(best, tf);
        if (ms < 0.25 * seconds * 1e3) iters = static_cast<int>(std::min<double>(iters * 4.0, 1 << 28));
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (sink) cudaFree(sink);
    if (e != cudaSuccess) return fail(nullptr, GSPH_E_CUDA, std::string("fp32 peak: ") + cudaGetErrorString(e));
    *tflops = best;
    return GSPH_OK;
}

}  // extern "C"
