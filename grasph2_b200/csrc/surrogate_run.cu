// surrogate_run.cu -- the learned K-substep surrogate as a native object: its MLP, the standardisation
// of the MLP's inputs and outputs, and the proposal / judge / window loop, built only on the public
// entry points (gsph_compute_derivatives, gsph_surrogate_features, gsph_mlp_forward,
// gsph_surrogate_apply, gsph_snapshot, gsph_step, gsph_state_compare, gsph_diagnostics_fast), so a
// C or C++ host drives the learned path without Python.
//
// Window rule: M proposals of K substeps; the plain integrator re-advances the last one from the same
// state as judge. The window is accepted when that proposal is within pos_tol of the plain result in
// position (norm over all particles, relative to the plain displacement over the K substeps) and within
// e_tol in total energy (relative to the energy scale e_ref); the state then continues from the plain
// result. Otherwise the window's proposals are discarded and the window is re-run by the plain
// integrator from its start (snapshot slot 0). Slots 1 and 2 hold the judge's start and proposal.
//
// Energy correction (optional): an MSE-trained network under-predicts the spread of what it cannot
// predict, so its proposals lose a little kinetic and shear energy against the plain integrator, the
// same way every time; over many windows that bias adds up although each judged proposal passes. With
// the correction on, every proposal is followed by gsph_energy_adjust(-b_kin, -b_shear), and every
// judged window whose position error passes updates the estimates from the judge's own comparison:
// b += gain * (E_P - E_Q) per part. The judged proposal is corrected like the others, so the judge
// measures the residual bias and checks the corrected method.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/grasph2_b200.h"

void set_global_error(const std::string& msg);  // capi.cu

namespace {
constexpr int kIn = GSPH_MLP_IN, kOut = GSPH_MLP_OUT;
constexpr int kStats = 2 * kIn + 2 * kOut;  // in_mu, in_sigma, out_mu, out_sigma
constexpr char kMagic[8] = {'G', 'S', 'P', 'H', 'S', 'U', 'R', '1'};
}  // namespace

struct gsph_surrogate {
    int32_t K = 0;
    gsph_mlp* net = nullptr;
    float host_stats[kStats] = {};
    float* stats = nullptr;    // device copy of host_stats
    float* feat = nullptr;     // [cap][32]
    float* out = nullptr;      // [cap][13]
    int64_t cap = 0;
    int64_t launches = 0;      // MLP forward launches
    bool ecorr = false;        // energy correction
    double gain = 0.5;
    double bias[2] = {0.0, 0.0};  // estimated kinetic and shear energy bias of one proposal
    std::string err;
};

namespace {

int sfail(gsph_surrogate* s, int code, const std::string& msg) {
    if (s)
        s->err = msg;
    else
        set_global_error(msg);
    return code;
}

// a failed context call: its own message, prefixed
int ctx_fail(gsph_surrogate* s, gsph_ctx* ctx, int code, const char* what) {
    return sfail(s, code, std::string(what) + ": " + gsph_last_error(ctx));
}

void release(gsph_surrogate* s) {
    if (s->net) gsph_mlp_destroy(s->net);
    if (s->stats) cudaFree(s->stats);
    if (s->feat) cudaFree(s->feat);
    if (s->out) cudaFree(s->out);
}

int reserve(gsph_surrogate* s, int64_t n) {
    if (n <= s->cap) return GSPH_OK;
    if (s->feat) cudaFree(s->feat);
    if (s->out) cudaFree(s->out);
    s->feat = s->out = nullptr;
    s->cap = 0;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&s->feat), static_cast<size_t>(n) * kIn * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s->out), static_cast<size_t>(n) * kOut * sizeof(float));
    if (e != cudaSuccess) return sfail(s, GSPH_E_NOMEM, std::string("surrogate buffers: ") + cudaGetErrorString(e));
    s->cap = n;
    return GSPH_OK;
}

// the energy correction after a proposal (nothing when off or before the first estimate)
int correct(gsph_surrogate* s, gsph_ctx* ctx, void* stream) {
    if (!s->ecorr || (s->bias[0] == 0.0 && s->bias[1] == 0.0)) return GSPH_OK;
    const int rc = gsph_energy_adjust(ctx, -s->bias[0], -s->bias[1], stream);
    return rc == GSPH_OK ? GSPH_OK : ctx_fail(s, ctx, rc, "propose: energy correction");
}

}  // namespace

extern "C" {

int gsph_surrogate_create(const float* params, const float* in_mu, const float* in_sigma, const float* out_mu,
                          const float* out_sigma, int32_t K, gsph_surrogate** out) {
    if (!out) return sfail(nullptr, GSPH_E_INVALID, "gsph_surrogate_create: out is NULL");
    *out = nullptr;
    if (K < 1) return sfail(nullptr, GSPH_E_INVALID, "gsph_surrogate_create: K < 1");
    const float* src[4] = {in_mu, in_sigma, out_mu, out_sigma};
    const int len[4] = {kIn, kIn, kOut, kOut};
    gsph_surrogate* s = new (std::nothrow) gsph_surrogate();
    if (!s) return sfail(nullptr, GSPH_E_NOMEM, "gsph_surrogate_create: host allocation failed");
    s->K = K;
    for (int b = 0, o = 0; b < 4; o += len[b], ++b)
        for (int k = 0; k < len[b]; ++k) {
            const float v = src[b] ? src[b][k] : (b % 2 ? 1.0f : 0.0f);  // default: identity scaling
            if (!std::isfinite(v) || (b % 2 == 1 && !(v > 0.0f))) {
                delete s;
                return sfail(nullptr, GSPH_E_INVALID, "gsph_surrogate_create: scales must be finite, sigmas > 0");
            }
            s->host_stats[o + k] = v;
        }
    int rc = gsph_mlp_create(params, &s->net);
    if (rc != GSPH_OK) {
        delete s;
        return rc;  // message set by gsph_mlp_create
    }
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&s->stats), kStats * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(s->stats, s->host_stats, kStats * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        const std::string msg = std::string("gsph_surrogate_create: ") + cudaGetErrorString(e);
        release(s);
        delete s;
        return sfail(nullptr, GSPH_E_CUDA, msg);
    }
    *out = s;
    return GSPH_OK;
}

int gsph_surrogate_destroy(gsph_surrogate* s) {
    if (!s) return GSPH_E_INVALID;
    cudaDeviceSynchronize();
    release(s);
    delete s;
    return GSPH_OK;
}

gsph_mlp* gsph_surrogate_mlp(gsph_surrogate* s) { return s ? s->net : nullptr; }

int32_t gsph_surrogate_substeps(const gsph_surrogate* s) { return s ? s->K : 0; }

int gsph_surrogate_stats(const gsph_surrogate* s, float* stats) {
    if (!s || !stats) return GSPH_E_INVALID;
    std::memcpy(stats, s->host_stats, sizeof(s->host_stats));
    return GSPH_OK;
}

int gsph_surrogate_save(gsph_surrogate* s, const char* path) {
    if (!s || !path) return sfail(s, GSPH_E_INVALID, "NULL argument");
    const int64_t np = gsph_mlp_param_count();
    std::vector<float> params(static_cast<size_t>(np));
    int rc = gsph_mlp_get_params(s->net, params.data());
    if (rc != GSPH_OK) return sfail(s, rc, std::string("save: ") + gsph_mlp_last_error(s->net));
    FILE* f = std::fopen(path, "wb");
    if (!f) return sfail(s, GSPH_E_INVALID, std::string("cannot open ") + path);
    const int32_t head[2] = {s->K, static_cast<int32_t>(np)};
    bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(head, sizeof(int32_t), 2, f) == 2 &&
              std::fwrite(params.data(), sizeof(float), params.size(), f) == params.size() &&
              std::fwrite(s->host_stats, sizeof(float), kStats, f) == static_cast<size_t>(kStats);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? GSPH_OK : sfail(s, GSPH_E_INVALID, std::string("write failed: ") + path);
}

int gsph_surrogate_load(const char* path, gsph_surrogate** out) {
    if (!path || !out) return sfail(nullptr, GSPH_E_INVALID, "gsph_surrogate_load: NULL argument");
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return sfail(nullptr, GSPH_E_INVALID, std::string("gsph_surrogate_load: cannot open ") + path);
    char magic[8];
    int32_t head[2] = {0, 0};
    const int64_t np = gsph_mlp_param_count();
    std::vector<float> params(static_cast<size_t>(np));
    float stats[kStats];
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
              std::fread(head, sizeof(int32_t), 2, f) == 2 && head[1] == np &&
              std::fread(params.data(), sizeof(float), params.size(), f) == params.size() &&
              std::fread(stats, sizeof(float), kStats, f) == static_cast<size_t>(kStats) && std::fgetc(f) == EOF;
    std::fclose(f);
    if (!ok) return sfail(nullptr, GSPH_E_INVALID, std::string("gsph_surrogate_load: not a surrogate model file: ") + path);
    return gsph_surrogate_create(params.data(), stats, stats + kIn, stats + 2 * kIn, stats + 2 * kIn + kOut, head[0],
                                 out);
}

}  // extern "C"

namespace {
// a proposal from a state whose derivatives are already computed: features, MLP, apply, correction
int propose_from_derivatives(gsph_surrogate* s, gsph_ctx* ctx, int32_t use_net, void* stream) {
    int rc;
    if (!use_net) {
        rc = gsph_surrogate_apply(ctx, nullptr, nullptr, nullptr, s->K, stream);
        if (rc != GSPH_OK) return ctx_fail(s, ctx, rc, "propose: apply");
        return correct(s, ctx, stream);
    }
    int64_t n = 0;
    gsph_size(ctx, &n);
    rc = reserve(s, n);
    if (rc != GSPH_OK) return rc;
    rc = gsph_surrogate_features(ctx, s->stats, s->stats + kIn, s->feat, stream);
    if (rc != GSPH_OK) return ctx_fail(s, ctx, rc, "propose: features");
    rc = gsph_mlp_forward(s->net, s->feat, s->out, n, stream);
    if (rc != GSPH_OK) return sfail(s, rc, std::string("propose: MLP: ") + gsph_mlp_last_error(s->net));
    ++s->launches;
    rc = gsph_surrogate_apply(ctx, s->out, s->stats + 2 * kIn, s->stats + 2 * kIn + kOut, s->K, stream);
    if (rc != GSPH_OK) return ctx_fail(s, ctx, rc, "propose: apply");
    return correct(s, ctx, stream);
}
}  // namespace

extern "C" {

int gsph_surrogate_propose(gsph_surrogate* s, gsph_ctx* ctx, int32_t use_net, void* stream) {
    if (!s || !ctx) return sfail(s, GSPH_E_INVALID, "NULL argument");
    const int rc = gsph_compute_derivatives(ctx, stream);
    if (rc != GSPH_OK) return ctx_fail(s, ctx, rc, "propose: derivatives");
    return propose_from_derivatives(s, ctx, use_net, stream);
}

int gsph_surrogate_judge(gsph_surrogate* s, gsph_ctx* ctx, int32_t use_net, double e_ref, gsph_surrogate_window* out,
                         void* stream) {
    if (!s || !ctx || !out) return sfail(s, GSPH_E_INVALID, "NULL argument");
    int rc;
    if (!(std::isfinite(e_ref) && e_ref != 0.0)) {
        gsph_diag d;
        rc = gsph_diagnostics_fast(ctx, 0.0, &d, stream);
        if (rc != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: energy");
        e_ref = d.e_kin + d.e_grav + d.e_int + d.e_shear;
    }
    // the start state is saved with its derivatives, which the proposal and the plain integrator's first
    // step share: the plain path is one integrate and K - 1 full steps (the same arithmetic as K steps)
    if ((rc = gsph_compute_derivatives(ctx, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: derivatives");
    if ((rc = gsph_snapshot(ctx, 1, 0, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: snapshot");
    if ((rc = propose_from_derivatives(s, ctx, use_net, stream)) != GSPH_OK) return rc;
    if ((rc = gsph_snapshot(ctx, 2, 0, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: snapshot");
    if ((rc = gsph_snapshot(ctx, 1, 1, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: restore");
    if ((rc = gsph_integrate(ctx, 1, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: plain steps");
    if ((rc = gsph_step(ctx, s->K - 1, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: plain steps");
    double c[8];
    if ((rc = gsph_state_compare_parts(ctx, 2, 1, c, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "judge: compare");
    out->pos_error = c[2] > 0.0 ? std::sqrt(c[1] / c[2]) : HUGE_VAL;
    out->energy_error = std::fabs(c[0]) / std::fabs(e_ref);
    for (int k = 0; k < 4; ++k) out->energy_parts[k] = c[4 + k] / std::fabs(e_ref);
    out->accepted = 0;
    out->reserved = 0;
    return GSPH_OK;
}

int gsph_surrogate_advance(gsph_surrogate* s, gsph_ctx* ctx, int32_t nwin, int32_t M, double pos_tol, double e_tol,
                           int32_t use_net, gsph_surrogate_window* windows, int32_t* accepted, void* stream) {
    if (!s || !ctx || nwin < 0 || M < 1) return sfail(s, GSPH_E_INVALID, "bad argument");
    gsph_diag d;
    int rc = gsph_diagnostics_fast(ctx, 0.0, &d, stream);
    if (rc != GSPH_OK) return ctx_fail(s, ctx, rc, "advance: energy");
    const double e_ref = d.e_kin + d.e_grav + d.e_int + d.e_shear;  // the scale of the energy criterion
    int32_t acc = 0;
    for (int32_t w = 0; w < nwin; ++w) {
        if ((rc = gsph_snapshot(ctx, 0, 0, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "advance: snapshot");
        for (int32_t k = 0; k + 1 < M; ++k)
            if ((rc = gsph_surrogate_propose(s, ctx, use_net, stream)) != GSPH_OK) return rc;
        gsph_surrogate_window r;
        if ((rc = gsph_surrogate_judge(s, ctx, use_net, e_ref, &r, stream)) != GSPH_OK) return rc;
        r.accepted = (r.pos_error <= pos_tol && r.energy_error <= e_tol) ? 1 : 0;
        if (s->ecorr && r.pos_error <= pos_tol) {  // the judge's residual kinetic and shear bias
            s->bias[0] += s->gain * r.energy_parts[0] * std::fabs(e_ref);
            s->bias[1] += s->gain * r.energy_parts[2] * std::fabs(e_ref);
        }
        if (r.accepted) {
            ++acc;
        } else {  // discard the window's proposals: the plain integrator from the window's start
            if ((rc = gsph_snapshot(ctx, 0, 1, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "advance: restore");
            if ((rc = gsph_step(ctx, M * s->K, stream)) != GSPH_OK) return ctx_fail(s, ctx, rc, "advance: plain steps");
        }
        if (windows) windows[w] = r;
    }
    if (accepted) *accepted = acc;
    return GSPH_OK;
}

int gsph_surrogate_set_energy_correction(gsph_surrogate* s, int32_t on, double gain) {
    if (!s) return GSPH_E_INVALID;
    if (!(gain > 0.0 && gain <= 1.0)) return sfail(s, GSPH_E_INVALID, "gain must be in (0, 1]");
    s->ecorr = on != 0;
    s->gain = gain;
    s->bias[0] = s->bias[1] = 0.0;
    return GSPH_OK;
}

int gsph_surrogate_energy_bias(const gsph_surrogate* s, double* bias) {
    if (!s || !bias) return GSPH_E_INVALID;
    bias[0] = s->bias[0];
    bias[1] = s->bias[1];
    return GSPH_OK;
}

int gsph_surrogate_launch_count(const gsph_surrogate* s, int64_t* count) {
    if (!s || !count) return GSPH_E_INVALID;
    *count = s->launches;
    return GSPH_OK;
}

const char* gsph_surrogate_last_error(const gsph_surrogate* s) { return s ? s->err.c_str() : gsph_last_error(nullptr); }

}  // extern "C"
