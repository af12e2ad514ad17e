/*
 * ref_driver.cpp -- TEST INFRASTRUCTURE ONLY. Builds GraSPH2's own hot-path code for the host:
 * the job structs and entry points of src/computeDerivatives.h and src/integration.h, and the
 * physics of src/sph/*.h, are #included from the reference tree unchanged, and driven through
 * the reference's own computeDerivatives(pb) and integrate(pb, notFirstStep). What this file adds
 * is the host particle buffer and the two generic launchers those entry points call; they follow
 * the reference's OpenMP host launchers (src/particles/algorithms.h:181-195 for do_for_each,
 * :233-256 and :312-316 for do_for_each_pair / do_for_each_pair_fast).
 *
 * Built by oracle/build_ref.py into oracle/_ref/libref_<variant>_<fp32|fp64>.so, once per physics
 * variant, because the reference's settings are compile-time constants. Used to pin the FP64
 * oracle (oracle/oracle.cpp) and to generate tests/golden/, and as the reference arm of bench.py.
 */
#include <cstdint>
#include <cstddef>
#include <cstring>

#include "settings.h"

/* the host buffer handed to the reference's entry points; it is named DeviceParticleBuffer<>
 * because integrate() static_asserts a DeviceParticleBuffer instantiation (integration.h:222) */
struct ref_particles {
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

template <>
class DeviceParticleBuffer<> {
public:
    ref_particles a;
    int64_t n;
    int64_t i0, i1;        /* targets of the pair passes after the density sum */
    bool density_rows = false;  /* timing samples: the density sum over [i0, i1) too */
    size_t size() const { return static_cast<size_t>(n); }
};
using RefBuffer = DeviceParticleBuffer<>;

template <typename job, typename buf, typename... Ts>
void do_for_each_pair_fast(buf& pb, Ts... args);
template <typename job, typename buf, typename... Ts>
void do_for_each(buf& pb, Ts... args);

#include "computeDerivatives.h"

namespace {

inline f3_t ld3(const f1_t* p, int64_t i) { return f3_t{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline void st3(f1_t* p, int64_t i, const f3_t& v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
inline void ld9(const f1_t* p, int64_t i, m3_t& m) { for (int e = 0; e < 9; ++e) m(e) = p[9 * i + e]; }
inline void st9(f1_t* p, int64_t i, const m3_t& m) { for (int e = 0; e < 9; ++e) p[9 * i + e] = m(e); }

template <typename Tag> struct attr_io;
#define GSPH_ATTR_IO(TAG, FIELD, LOAD, STORE)                                                   \
    template <> struct attr_io<TAG> {                                                           \
        static void load(const ref_particles& b, int64_t i, gsph_particle_record& r) { LOAD; }  \
        static void store(ref_particles& b, int64_t i, const gsph_particle_record& r) { STORE; } \
    };
GSPH_ATTR_IO(POS, pos, r.pos = ld3(b.pos, i), st3(b.pos, i, r.pos))
GSPH_ATTR_IO(MASS, mass, r.mass = b.mass[i], b.mass[i] = r.mass)
GSPH_ATTR_IO(VEL, vel, r.vel = ld3(b.vel, i), st3(b.vel, i, r.vel))
GSPH_ATTR_IO(ACC, acc, r.acc = ld3(b.acc, i), st3(b.acc, i, r.acc))
GSPH_ATTR_IO(BALSARA, balsara, r.balsara = b.balsara[i], b.balsara[i] = r.balsara)
GSPH_ATTR_IO(XVEL, xvel, r.xvel = ld3(b.xvel, i), st3(b.xvel, i, r.xvel))
GSPH_ATTR_IO(DENSITY, density, r.density = b.density[i], b.density[i] = r.density)
GSPH_ATTR_IO(DENSITY_DT, density_dt, r.density_dt = b.density_dt[i], b.density_dt[i] = r.density_dt)
GSPH_ATTR_IO(DSTRESS, dstress, ld9(b.dstress, i, const_cast<gsph_particle_record&>(r).dstress), st9(b.dstress, i, r.dstress))
GSPH_ATTR_IO(DSTRESS_DT, dstress_dt, ld9(b.dstress_dt, i, const_cast<gsph_particle_record&>(r).dstress_dt),
             st9(b.dstress_dt, i, r.dstress_dt))
GSPH_ATTR_IO(MAXVSIG, max_vsig, r.max_vsig = b.maxvsig[i], b.maxvsig[i] = r.max_vsig)
#undef GSPH_ATTR_IO

template <typename P> struct particle_io;
template <typename... A> struct particle_io<Particle<A...>> {
    /* load_helper<Particle<A...>>::load: the listed attributes, value-initialised otherwise */
    static Particle<A...> load(const ref_particles& b, int64_t i) {
        Particle<A...> p{};
        (attr_io<A>::load(b, i, p), ...);
        return p;
    }
    /* storeParticle(i, Particle<A...>): the listed attributes only */
    static void store(ref_particles& b, int64_t i, const Particle<A...>& p) { (attr_io<A>::store(b, i, p), ...); }
};

/* the device-reference view the reference's variable-step kernels take (integration.h:130-217) */
struct RefDeviceView {
    ref_particles* a;
    int64_t n;
    size_t size() const { return static_cast<size_t>(n); }
    template <typename... A> Particle<A...> loadParticle(size_t i) const { return particle_io<Particle<A...>>::load(*a, i); }
    template <typename... A> void storeParticle(size_t i, const Particle<A...>& p) const {
        particle_io<Particle<A...>>::store(*a, i, p);
    }
};

}  // namespace

/* do_for_each_pair on a host buffer, src/particles/algorithms.h:233-256 (do_for_each_pair_fast on
 * a host buffer forwards to it, :312-316). Targets are all particles for the density sum, whose
 * result every later pass reads, and [i0, i1) for the other jobs. */
template <typename job, typename buf, typename... Ts>
void do_for_each_pair_fast(buf& pb, Ts... args) {
    const int64_t n = pb.n;
    const bool all = std::is_same<job, calcDensity>::value && !pb.density_rows;
    const int64_t lo = all ? 0 : pb.i0, hi = all ? n : pb.i1;
#pragma omp parallel for schedule(static)
    for (int64_t i = lo; i < hi; i++) {
        job job_i;
        typename job::pi_type pi{};
        pi = particle_io<typename job::load_type>::load(pb.a, i);
        job_i.do_before(pi, i, args...);
        for (int64_t j = 0; j < n; j++) {
            const auto pj = particle_io<typename job::pj_type>::load(pb.a, j);
            job_i.do_for_each_pair(pi, pj, args...);
        }
        typename job::store_type result = job_i.do_after(pi, args...);
        particle_io<typename job::store_type>::store(pb.a, i, result);
    }
}

/* do_for_each on a host buffer, src/particles/algorithms.h:181-195 */
template <typename job, typename buf, typename... Ts>
void do_for_each(buf& pb, Ts... args) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < pb.n; i++) {
        job job_i;
        typename job::pi_type pi{};
        pi = particle_io<typename job::load_type>::load(pb.a, i);
        typename job::store_type result = job_i.do_for_each(pi, i, args...);
        particle_io<typename job::store_type>::store(pb.a, i, result);
    }
}

extern "C" {

int ref_precision(void) { return static_cast<int>(sizeof(f1_t)); }
const char* ref_variant(void) { return REF_VARIANT_NAME; }

/* computeDerivatives(pb), src/computeDerivatives.h:315-328, then the variable-step reset that
 * calcAcceleration::do_after does when VARIABLE_TIMESTEP_LEAPFROG is set (:306-309) */
int ref_compute_derivatives(int64_t n, ref_particles* s, int64_t i0, int64_t i1) {
    if (!s || n < 0) return -1;
    RefBuffer pb;
    pb.a = *s;
    pb.n = n;
    pb.i0 = i0 < 0 ? 0 : i0;
    pb.i1 = (i1 < 0 || i1 > n) ? n : i1;
    computeDerivatives(pb);
    nextTS = max_timestep;
    return 0;
}

/* Timing sample: every pass of computeDerivatives over target rows [i0, i1) only (the density sum
 * included, so the sample's cost is (i1 - i0) / n of a full evaluation). */
int ref_compute_derivatives_rows(int64_t n, ref_particles* s, int64_t i0, int64_t i1) {
    if (!s || n < 0) return -1;
    RefBuffer pb;
    pb.a = *s;
    pb.n = n;
    pb.i0 = i0 < 0 ? 0 : i0;
    pb.i1 = (i1 < 0 || i1 > n) ? n : i1;
    pb.density_rows = true;
    computeDerivatives(pb);
    return 0;
}

/* integrate(pb, notFirstStep) with FIXED_TIMESTEP_LEAPFROG, src/integration.h:219-224 */
int ref_integrate(int64_t n, int not_first_step, ref_particles* s) {
    if (!s || n < 0) return -1;
    RefBuffer pb;
    pb.a = *s;
    pb.n = n;
    pb.i0 = 0;
    pb.i1 = n;
    integrate(pb, not_first_step != 0);
    return 0;
}

/* integrate(pb, notFirstStep) with VARIABLE_TIMESTEP_LEAPFROG: the dispatch of
 * src/integration.h:225-242 around the reference's own two kernels */
int ref_integrate_variable(int64_t n, int not_first_step, ref_particles* s) {
    if (!s || n < 0) return -1;
    RefDeviceView v{s, n};
    if (not_first_step)
        variableTsLeapfrog_getNewTimestep<INTEG_BS>(v);
    else
        nextTS = initial_timestep;
    variableTsLeapfrog_useNewTimestep(v);
    return 0;
}

double ref_current_timestep(void) { return static_cast<double>(currentTS); }
double ref_next_timestep(void) { return static_cast<double>(nextTS); }
double ref_fixed_timestep(void) { return static_cast<double>(getCurrentTimestep()); }
void ref_set_timestep(double current, double next) {
    currentTS = static_cast<f1_t>(current);
    nextTS = static_cast<f1_t>(next);
}

/* the reference's SPH kernel functions (src/sph/kernel.h:130-136, :169-175) at this build's H */
double ref_w_spline(double r) { return kernel::Wspline(static_cast<f1_t>(r), H, W_prefactor); }
double ref_dw_spline(double r) { return kernel::dWspline(static_cast<f1_t>(r), H, dW_prefactor); }

/* plasticity(), src/sph/models.h:194-205, on one row-major tensor */
void ref_plasticity(double* S9, double Yield) {
    m3_t S;
    for (int e = 0; e < 9; ++e) S(e) = static_cast<f1_t>(S9[e]);
    plasticity(S, static_cast<f1_t>(Yield));
    for (int e = 0; e < 9; ++e) S9[e] = S(e);
}

/* dstress_dt(), src/sph/models.h:250-268 */
void ref_dstress_dt(const double* edot9, const double* rdot9, const double* S9, double shear_mod, double* out9) {
    m3_t E, R, S;
    for (int e = 0; e < 9; ++e) {
        E(e) = static_cast<f1_t>(edot9[e]);
        R(e) = static_cast<f1_t>(rdot9[e]);
        S(e) = static_cast<f1_t>(S9[e]);
    }
    const m3_t out = dstress_dt(E, R, S, static_cast<f1_t>(shear_mod));
    for (int e = 0; e < 9; ++e) out9[e] = out(e);
}

}  // extern "C"
