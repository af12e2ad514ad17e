// grasph2_b200.hpp -- header-only C++ adapter over the C-ABI with GraSPH2's names, so a driver
// written against the reference's hot path (src/main.cu:249-273) ports line for line:
//
//     gsph::HostParticleBuffer hpb(n);                   // HostParticleBuffer<...>   (HostParticleBuffer.h:47-99)
//     gsph::DeviceParticleBuffer pb(params, hpb.size());  // DeviceParticleBuffer<...> (DeviceParticleBuffer.h:47-233)
//     pb = hpb;                                           // upload                    (Device_base.h:163-181)
//     computeDerivatives(pb);                             // src/computeDerivatives.h:315-328
//     integrate(pb, true);                                // src/integration.h:219-244
//     double dt = getCurrentTimestep(pb);                 // src/integration.h:246-255
//     hpb = pb;                                           // download
//     gsph::printTextFile(hpb, path);                     // ResultStorageManager::printTextFile (.cu:160-186)
//
// Errors throw gsph::Error (a std::runtime_error carrying the GSPH_E_* code); the reference's
// assert_cuda throws/aborts in the same places.
#ifndef GRASPH2_B200_HPP
#define GRASPH2_B200_HPP

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "grasph2_b200.h"

namespace gsph {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc, gsph_ctx* ctx) {
    if (rc != GSPH_OK) throw Error(rc, gsph_last_error(ctx));
}

// ---- precision types (settings/precisionSettings.h, src/types.h:32-56; the single-precision build) ----
using f1_t = float;
struct f3_t {
    f1_t x = 0, y = 0, z = 0;
};
struct f4_t {
    f1_t x = 0, y = 0, z = 0, w = 0;
};
inline f3_t operator+(f3_t a, f3_t b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline f3_t operator-(f3_t a, f3_t b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline f3_t operator*(f3_t a, f1_t s) { return {a.x * s, a.y * s, a.z * s}; }
inline f3_t operator*(f1_t s, f3_t a) { return a * s; }
inline f1_t dot(f3_t a, f3_t b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// 3x3 matrix, row-major; m(r, c) and m[r][c] as mpu::Mat's accessors
struct m3_t {
    f1_t v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    f1_t& operator()(int r, int c) { return v[3 * r + c]; }
    f1_t operator()(int r, int c) const { return v[3 * r + c]; }
    f1_t* operator[](int r) { return v + 3 * r; }
    const f1_t* operator[](int r) const { return v + 3 * r; }
};

// One particle with every attribute of the reference's DeviceParticlesType (settings/settings.h:184),
// the counterpart of Particle<...> (src/particles/Particle.h) for host-side access.
struct Particle {
    f3_t pos;
    f1_t mass = 0;
    f3_t vel, acc;
    f1_t balsara = 0;
    f3_t xvel;
    f1_t density = 0, density_dt = 0;
    m3_t dstress, dstress_dt;
    f1_t maxvsig = 0;
};

// Host particle attributes in the reference layout, one std::vector<float> per attribute.
class HostParticleBuffer {
public:
    HostParticleBuffer() = default;
    explicit HostParticleBuffer(size_t n) { resize(n); }
    void resize(size_t n) {
        n_ = n;
        pos.assign(3 * n, 0.f); mass.assign(n, 0.f); vel.assign(3 * n, 0.f); acc.assign(3 * n, 0.f);
        balsara.assign(n, 0.f); xvel.assign(3 * n, 0.f); density.assign(n, 0.f); density_dt.assign(n, 0.f);
        dstress.assign(9 * n, 0.f); dstress_dt.assign(9 * n, 0.f); maxvsig.assign(n, 0.f);
    }
    size_t size() const { return n_; }
    gsph_host_particles view() {
        return gsph_host_particles{pos.data(), mass.data(), vel.data(), acc.data(), balsara.data(), xvel.data(),
                                   density.data(), density_dt.data(), dstress.data(), dstress_dt.data(), maxvsig.data()};
    }
    std::vector<float> pos, mass, vel, acc, balsara, xvel, density, density_dt, dstress, dstress_dt, maxvsig;

    // HostParticleBuffer::loadParticle / storeParticle (src/particles/HostParticleBuffer.h:79-83); the
    // attributes written are chosen by a GSPH_* mask instead of the reference's template arguments
    Particle loadParticle(size_t i) const {
        Particle p;
        p.pos = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        p.mass = mass[i];
        p.vel = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
        p.acc = {acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]};
        p.balsara = balsara[i];
        p.xvel = {xvel[3 * i], xvel[3 * i + 1], xvel[3 * i + 2]};
        p.density = density[i];
        p.density_dt = density_dt[i];
        for (int k = 0; k < 9; ++k) {
            p.dstress.v[k] = dstress[9 * i + k];
            p.dstress_dt.v[k] = dstress_dt[9 * i + k];
        }
        p.maxvsig = maxvsig[i];
        return p;
    }
    void storeParticle(size_t i, const Particle& p, uint32_t mask = GSPH_ALL_ATTRIBS) {
        auto put3 = [&](std::vector<float>& a, const f3_t& v) {
            a[3 * i] = v.x;
            a[3 * i + 1] = v.y;
            a[3 * i + 2] = v.z;
        };
        if (mask & GSPH_POS) put3(pos, p.pos);
        if (mask & GSPH_MASS) mass[i] = p.mass;
        if (mask & GSPH_VEL) put3(vel, p.vel);
        if (mask & GSPH_ACC) put3(acc, p.acc);
        if (mask & GSPH_BALSARA) balsara[i] = p.balsara;
        if (mask & GSPH_XVEL) put3(xvel, p.xvel);
        if (mask & GSPH_DENSITY) density[i] = p.density;
        if (mask & GSPH_DENSITY_DT) density_dt[i] = p.density_dt;
        for (int k = 0; k < 9; ++k) {
            if (mask & GSPH_DSTRESS) dstress[9 * i + k] = p.dstress.v[k];
            if (mask & GSPH_DSTRESS_DT) dstress_dt[9 * i + k] = p.dstress_dt.v[k];
        }
        if (mask & GSPH_MAXVSIG) maxvsig[i] = p.maxvsig;
    }

private:
    size_t n_ = 0;
};

// Owning device buffer of one simulation (RAII over gsph_create / gsph_destroy).
class DeviceParticleBuffer {
public:
    DeviceParticleBuffer(const gsph_params& p, int64_t n, const gsph_options* opt = nullptr) {
        check(gsph_create(&p, opt, n, &ctx_), nullptr);
    }
    ~DeviceParticleBuffer() {
        if (ctx_) gsph_destroy(ctx_);
    }
    DeviceParticleBuffer(const DeviceParticleBuffer&) = delete;
    DeviceParticleBuffer& operator=(const DeviceParticleBuffer&) = delete;
    DeviceParticleBuffer(DeviceParticleBuffer&& o) noexcept : ctx_(std::exchange(o.ctx_, nullptr)) {}
    DeviceParticleBuffer& operator=(DeviceParticleBuffer&& o) noexcept {
        if (this != &o) {
            if (ctx_) gsph_destroy(ctx_);
            ctx_ = std::exchange(o.ctx_, nullptr);
        }
        return *this;
    }
    // pb = hostBuffer: every attribute (Device_base.h:163-181)
    DeviceParticleBuffer& operator=(HostParticleBuffer& h) {
        upload(h, GSPH_ALL_ATTRIBS);
        return *this;
    }
    void upload(HostParticleBuffer& h, uint32_t mask, void* stream = nullptr) {
        gsph_host_particles v = h.view();
        check(gsph_upload(ctx_, mask, &v, stream), ctx_);
    }
    void download(HostParticleBuffer& h, uint32_t mask = GSPH_ALL_ATTRIBS, void* stream = nullptr) {
        if (h.size() != static_cast<size_t>(size())) h.resize(static_cast<size_t>(size()));
        gsph_host_particles v = h.view();
        check(gsph_download(ctx_, mask, &v, stream), ctx_);
    }
    int64_t size() const {
        int64_t n = 0;
        check(gsph_size(ctx_, &n), ctx_);
        return n;
    }
    void step(int nsteps, void* stream = nullptr) { check(gsph_step(ctx_, nsteps, stream), ctx_); }
    gsph_diag diagnostics(double half_kick = 0.0, void* stream = nullptr) {
        gsph_diag d{};
        check(gsph_diagnostics(ctx_, half_kick, &d, stream), ctx_);
        return d;
    }
    // time candidate launch shapes on the current state and keep the fastest
    gsph_launch_shape autotune(int reps = 3, void* stream = nullptr) {
        check(gsph_autotune(ctx_, reps, stream), ctx_);
        gsph_launch_shape s{};
        check(gsph_launch_shape_get(ctx_, &s), ctx_);
        return s;
    }
    gsph_ctx* get() const { return ctx_; }

private:
    gsph_ctx* ctx_ = nullptr;
};

// Many simulations of one physics setup, advanced together (RAII over gsph_ensemble_*). Host buffers
// hold the simulations back to back in the order of offsets().
class Ensemble {
public:
    Ensemble(const gsph_params& p, const std::vector<int64_t>& counts, const gsph_options* opt = nullptr) {
        int rc = gsph_ensemble_create(&p, opt, static_cast<int32_t>(counts.size()), counts.data(), &e_);
        if (rc != GSPH_OK) throw Error(rc, gsph_ensemble_last_error(nullptr));
        off_.resize(counts.size() + 1);
        chk(gsph_ensemble_offsets(e_, off_.data()));
    }
    ~Ensemble() {
        if (e_) gsph_ensemble_destroy(e_);
    }
    Ensemble(const Ensemble&) = delete;
    Ensemble& operator=(const Ensemble&) = delete;
    const std::vector<int64_t>& offsets() const { return off_; }
    int64_t size() const { return off_.back(); }
    void upload(HostParticleBuffer& h, uint32_t mask, void* stream = nullptr) {
        gsph_host_particles v = h.view();
        chk(gsph_ensemble_upload(e_, mask, &v, stream));
    }
    void download(HostParticleBuffer& h, uint32_t mask = GSPH_ALL_ATTRIBS, void* stream = nullptr) {
        if (h.size() != static_cast<size_t>(size())) h.resize(static_cast<size_t>(size()));
        gsph_host_particles v = h.view();
        chk(gsph_ensemble_download(e_, mask, &v, stream));
    }
    void step(int nsteps, void* stream = nullptr) { chk(gsph_ensemble_step(e_, nsteps, stream)); }
    std::vector<gsph_diag> diagnostics(double half_kick = 0.0, void* stream = nullptr) {
        std::vector<gsph_diag> d(off_.size() - 1);
        chk(gsph_ensemble_diagnostics(e_, half_kick, d.data(), stream));
        return d;
    }
    void autotune(int reps = 2, void* stream = nullptr) {
        chk(gsph_ensemble_autotune(e_, reps, nullptr, nullptr, stream));
    }
    gsph_ensemble* get() const { return e_; }

private:
    void chk(int rc) {
        if (rc != GSPH_OK) throw Error(rc, gsph_ensemble_last_error(e_));
    }
    gsph_ensemble* e_ = nullptr;
    std::vector<int64_t> off_;
};

// hostBuffer = deviceBuffer
inline HostParticleBuffer& operator<<(HostParticleBuffer& h, DeviceParticleBuffer& d) {
    d.download(h);
    return h;
}

inline void computeDerivatives(DeviceParticleBuffer& pb, void* stream = nullptr) {
    check(gsph_compute_derivatives(pb.get(), stream), pb.get());
}
inline void integrate(DeviceParticleBuffer& pb, bool notFirstStep, void* stream = nullptr) {
    check(gsph_integrate(pb.get(), notFirstStep ? 1 : 0, stream), pb.get());
}
inline double getCurrentTimestep(DeviceParticleBuffer& pb, void* stream = nullptr) {
    double dt = 0.0;
    check(gsph_current_timestep(pb.get(), &dt, stream), pb.get());
    return dt;
}

// ---- tsv snapshots -----------------------------------------------------------------------------
// One line per particle; the selected attributes in particle_bases order, every value followed by
// a tab; fixed notation with digits10 + 1 digits (ResultStorageManager::printTextFile,
// src/ResultStorageManager.cu:160-186; the stored attributes are HostDiscPT's, settings
// outputSettings.h:26: POS, MASS, VEL, DENSITY by default).
constexpr uint32_t kDefaultStoredAttributes = GSPH_POS | GSPH_MASS | GSPH_VEL | GSPH_DENSITY;

inline int attribute_components(int bit) {
    static const int comps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};
    return comps[bit];
}
inline const std::vector<float>& attribute_data(const HostParticleBuffer& h, int bit) {
    const std::vector<float>* a[11] = {&h.pos, &h.mass, &h.vel, &h.acc, &h.balsara, &h.xvel,
                                       &h.density, &h.density_dt, &h.dstress, &h.dstress_dt, &h.maxvsig};
    return *a[bit];
}
inline std::vector<float>& attribute_data(HostParticleBuffer& h, int bit) {
    return const_cast<std::vector<float>&>(attribute_data(static_cast<const HostParticleBuffer&>(h), bit));
}

// file name <directory><prefix><startTime>_<time>.tsv (ResultStorageManager.cu:162-163)
inline std::string snapshotFileName(const std::string& directory, const std::string& prefix,
                                    const std::string& startTime, float time, const char* ext = ".tsv") {
    std::ostringstream fn;
    fn << directory << prefix << startTime << "_" << std::fixed
       << std::setprecision(std::numeric_limits<float>::digits10 + 1) << time << ext;
    return fn.str();
}

// the same from raw host arrays (a gsph_host_particles view of n particles)
inline void printTextFile(const gsph_host_particles& v, size_t n, const std::string& filename,
                          uint32_t mask = kDefaultStoredAttributes) {
    const float* a[11] = {v.pos, v.mass, v.vel, v.acc, v.balsara, v.xvel, v.density, v.density_dt, v.dstress,
                          v.dstress_dt, v.maxvsig};
    std::ofstream file(filename);
    if (!file.is_open()) throw Error(GSPH_E_INVALID, "Could not open output file: " + filename);
    file << std::fixed << std::setprecision(std::numeric_limits<float>::digits10 + 1);
    for (size_t i = 0; i < n; ++i) {
        for (int b = 0; b < 11; ++b) {
            if (!(mask >> b & 1u)) continue;
            const int k = attribute_components(b);
            for (int c = 0; c < k; ++c) file << a[b][k * i + c] << "\t";
        }
        file << "\n";
    }
    if (file.fail()) throw Error(GSPH_E_INVALID, "Error writing output file: " + filename);
}

inline void printTextFile(const HostParticleBuffer& h, const std::string& filename,
                          uint32_t mask = kDefaultStoredAttributes) {
    gsph_host_particles v = const_cast<HostParticleBuffer&>(h).view();
    printTextFile(v, h.size(), filename, mask);
}

// Asynchronous snapshots (ResultStorageManager::printToFile, src/ResultStorageManager.cu:102-186): write()
// returns once the state is copied on the device; a worker thread writes the tsv file.
class SnapshotWriter {
public:
    SnapshotWriter(DeviceParticleBuffer& pb, uint32_t mask = kDefaultStoredAttributes, int depth = 2) {
        const int rc = gsph_writer_create(pb.get(), mask, depth, &w_);
        if (rc != GSPH_OK) throw Error(rc, gsph_last_error(nullptr));
    }
    ~SnapshotWriter() {
        if (w_) gsph_writer_destroy(w_);
    }
    SnapshotWriter(const SnapshotWriter&) = delete;
    SnapshotWriter& operator=(const SnapshotWriter&) = delete;
    void write(const std::string& filename, void* stream = nullptr) { chk(gsph_writer_write(w_, filename.c_str(), stream)); }
    int64_t flush() {
        int64_t n = 0;
        chk(gsph_writer_flush(w_, &n));
        return n;
    }

private:
    void chk(int rc) {
        if (rc != GSPH_OK) throw Error(rc, gsph_writer_last_error(w_));
    }
    gsph_writer* w_ = nullptr;
};

// The learned K-substep surrogate (gsph_surrogate_*): load a trained model file and advance a buffer
// by judged windows of proposals.
class Surrogate {
public:
    explicit Surrogate(const std::string& modelFile) {
        const int rc = gsph_surrogate_load(modelFile.c_str(), &s_);
        if (rc != GSPH_OK) throw Error(rc, gsph_last_error(nullptr));
    }
    ~Surrogate() {
        if (s_) gsph_surrogate_destroy(s_);
    }
    Surrogate(const Surrogate&) = delete;
    Surrogate& operator=(const Surrogate&) = delete;
    int substeps() const { return gsph_surrogate_substeps(s_); }
    void propose(DeviceParticleBuffer& pb, bool useNet = true, void* stream = nullptr) {
        chk(gsph_surrogate_propose(s_, pb.get(), useNet ? 1 : 0, stream));
    }
    // nwin windows of M proposals; returns the per-window errors and acceptance
    std::vector<gsph_surrogate_window> advance(DeviceParticleBuffer& pb, int nwin, int M = 4, double posTol = 1e-3,
                                               double energyTol = 1e-4, bool useNet = true, void* stream = nullptr) {
        std::vector<gsph_surrogate_window> w(static_cast<size_t>(nwin));
        chk(gsph_surrogate_advance(s_, pb.get(), nwin, M, posTol, energyTol, useNet ? 1 : 0, w.data(), nullptr,
                                   stream));
        return w;
    }
    void save(const std::string& modelFile) { chk(gsph_surrogate_save(s_, modelFile.c_str())); }
    // the judge-calibrated energy correction (gsph_surrogate_set_energy_correction); resets its estimates
    void energyCorrection(bool on, double gain = 1.0) { chk(gsph_surrogate_set_energy_correction(s_, on ? 1 : 0, gain)); }
    gsph_surrogate* get() { return s_; }

private:
    void chk(int rc) {
        if (rc != GSPH_OK) throw Error(rc, gsph_surrogate_last_error(s_));
    }
    gsph_surrogate* s_ = nullptr;
};

// TextFile reader (src/initialConditions/particleSources/TextFile.h:76-120): non-blank lines are
// particles, values separated by `sep`, the attributes in `mask` in particle_bases order.
inline HostParticleBuffer readTextFile(const std::string& filename, uint32_t mask = kDefaultStoredAttributes,
                                       char sep = '\t') {
    std::ifstream file(filename);
    if (!file.is_open()) throw Error(GSPH_E_INVALID, "Error opening file: " + filename);
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(file, line)) {
        bool blank = true;
        for (char c : line)
            if (!std::isspace(static_cast<unsigned char>(c))) blank = false;
        if (!blank) lines.push_back(line);
    }
    HostParticleBuffer h(lines.size());
    for (size_t i = 0; i < lines.size(); ++i) {
        std::istringstream ls(lines[i]);
        for (int b = 0; b < 11; ++b) {
            if (!(mask >> b & 1u)) continue;
            const int k = attribute_components(b);
            std::vector<float>& a = attribute_data(h, b);
            for (int c = 0; c < k; ++c) {
                std::string tok;
                do {
                    if (!std::getline(ls, tok, sep)) throw Error(GSPH_E_INVALID, "Error parsing input file at line " +
                                                                                     std::to_string(i));
                } while (tok.find_first_not_of(" \t") == std::string::npos);
                // as the reference's TextFile reader: the token as a double, then rounded to float
                // (src/initialConditions/particleSources/TextFile.h:127-129)
                a[k * i + c] = static_cast<float>(std::stod(tok));
            }
        }
    }
    return h;
}

}  // namespace gsph

#endif  // GRASPH2_B200_HPP
