/*
 * oracle.cpp -- TEST INFRASTRUCTURE ONLY. FP64 CPU restatement of GraSPH2's per-step hot path,
 * used as the checker for the CUDA kernels of grasph2_b200. Nothing in the product links or calls
 * this file; only the tests, the package's smoke check and the CPU-baseline leg of bench.py do.
 *
 * Every function restates the reference's arithmetic with runtime parameters (gsph_params) in
 * place of the reference's compile-time settings. Citations are to the GraSPH2 source tree.
 *
 *   cubic spline W, dW             src/sph/kernel.h:41-87 (prefactors), :130-136, :169-175
 *   EOS liquid / Murnaghan         src/sph/eos.h:88-96
 *   AV, Balsara, plasticity, MC,
 *   artificial stress, strain and
 *   rotation rate, Jaumann dS/dt   src/sph/models.h:158-268
 *   environment acceleration       src/computeDerivatives.h:33-47
 *   calcDensity                    src/computeDerivatives.h:52-91
 *   calcBalsaraDensityDTDStressDT  src/computeDerivatives.h:96-162
 *   calcAcceleration               src/computeDerivatives.h:167-313
 *   computeDerivatives             src/computeDerivatives.h:315-328
 *   fixedTsLeapfrog, plasticity,
 *   box boundary                   src/integration.h:24-125
 *   variable-dt leapfrog           src/integration.h:130-244
 *   host pair / per-particle loops src/particles/algorithms.h:181-195, :233-256
 *
 * Two deliberate generalisations, both reducing to the reference at their reference values:
 * the gravitational softening grav_eps (reference: eps == H, src/computeDerivatives.h:231) and the
 * AV signal-velocity coefficient av_beta (reference: 3, src/sph/models.h:179).
 *
 * Parity pin: this file is checked against the reference's own job structs compiled for the host
 * (oracle/ref_driver.cpp) on every configuration the reference can express, and against golden
 * fixtures generated from that build (tests/golden/).
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>

#include "../include/grasph2_b200.h"

extern "C" {

/* FP64 particle arrays in the reference attribute layout (see gsph_host_particles). */
typedef struct oracle_particles {
    double* pos;        /* 3N */
    double* mass;       /* N  */
    double* vel;        /* 3N */
    double* acc;        /* 3N */
    double* balsara;    /* N  */
    double* xvel;       /* 3N */
    double* density;    /* N  */
    double* density_dt; /* N  */
    double* dstress;    /* 9N, row-major */
    double* dstress_dt; /* 9N */
    double* maxvsig;    /* N  */
} oracle_particles;

/* the variable-step state of src/integration.h:127-128 (device symbols currentTS / nextTS) */
typedef struct oracle_timestep {
    double current;
    double next;
} oracle_timestep;

}

namespace {

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(double s, V3 a) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 load3(const double* p, int64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline void store3(double* p, int64_t i, V3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }

struct M3 {
    double a[3][3];
};
inline M3 mzero() { M3 m; std::memset(&m, 0, sizeof m); return m; }
inline M3 load9(const double* p, int64_t i) { M3 m; std::memcpy(m.a, p + 9 * i, sizeof m.a); return m; }
inline void store9(double* p, int64_t i, const M3& m) { std::memcpy(p + 9 * i, m.a, sizeof m.a); }
inline V3 mul(const M3& m, V3 v) {  /* row-major matrix times column vector */
    return {m.a[0][0] * v.x + m.a[0][1] * v.y + m.a[0][2] * v.z,
            m.a[1][0] * v.x + m.a[1][1] * v.y + m.a[1][2] * v.z,
            m.a[2][0] * v.x + m.a[2][1] * v.y + m.a[2][2] * v.z};
}

inline bool on(const gsph_params& p, uint32_t f) { return (p.flags & f) != 0; }

/* ---- src/sph/kernel.h ---------------------------------------------------------------------- */
/* splinePrefactor<Dim>, kernel.h:44-60 */
double spline_prefactor(int dim, double h) {
    if (dim == 1) return 4.0 / (3.0 * h);
    if (dim == 2) return 40.0 / (7.0 * M_PI * h * h);
    return 8.0 / (M_PI * h * h * h);
}
/* dsplinePrefactor<Dim>, kernel.h:71-87 */
double dspline_prefactor(int dim, double h) {
    if (dim == 1) return 24.0 / (3.0 * h * h);
    if (dim == 2) return 240.0 / (7.0 * M_PI * h * h * h);
    return 48.0 / (M_PI * h * h * h * h);
}
/* Wspline, kernel.h:130-136: support radius h (not 2h) */
inline double w_spline(double r, double h, double f) {
    const double q = r / h;
    if (q > 1.0) return 0.0;
    if (q < 0.5) return f * (6.0 * q * q * q - 6.0 * q * q + 1.0);
    return f * 2.0 * (1.0 - q) * (1.0 - q) * (1.0 - q);
}
/* dWspline, kernel.h:169-175 */
inline double dw_spline(double r, double h, double f) {
    const double q = r / h;
    if (q > 1.0) return 0.0;
    if (q < 0.5) return f * (3.0 * q * q - 2.0 * q);
    return f * -1.0 * (1.0 - q) * (1.0 - q);
}

/* ---- src/sph/eos.h ------------------------------------------------------------------------- */
inline double eos_liquid(double rho, double rho0, double c2) { return c2 * (rho - rho0); }           /* eos.h:88-91 */
inline double eos_murnaghan(double rho, double rho0, double K0, double dK0) {                      /* eos.h:93-96 */
    return K0 / dK0 * (std::pow(rho / rho0, dK0) - 1.0);
}

/* ---- src/sph/models.h ---------------------------------------------------------------------- */
/* artificialViscosity (both overloads), models.h:158-185; av_beta = 3 is the reference */
inline double artificial_viscosity(double* max_vsig, double alpha, double beta, double rho_i, double rho_j,
                                   V3 vij, V3 rij, double r, double ci, double cj, double bi, double bj) {
    const double wij = dot(rij, vij) / r;
    double II = 0.0;
    if (wij < 0.0) {
        const double vsig = ci + cj - beta * wij;
        const double rhoij = (rho_i + rho_j) * 0.5;
        II = -0.25 * (bi + bj) * alpha * wij * vsig / rhoij;
        if (max_vsig) *max_vsig = std::max(*max_vsig, vsig);
    }
    return II;
}
/* balsaraSwitch, models.h:187-192 */
inline double balsara_switch(double divv, V3 curlv, double c, double h) {
    const double absdiv = std::fabs(divv);
    const double abscurl = length(curlv);
    return absdiv / (absdiv + abscurl + 0.0001 * c / h);
}
/* plasticity, models.h:194-205: scales by Y^2/(3 J2) -- no square root, as in the reference */
inline void plasticity(M3& S, double Y) {
    double J2 = 0.0;
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) J2 += S.a[d][e] * S.a[d][e];
    J2 *= 0.5;
    const double f = Y * Y / (3.0 * J2);
    if (f < 1.0)
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 3; ++e) S.a[d][e] *= f;
}
/* mohrCoulombYieldStress, models.h:207-210 */
inline double mohr_coulomb_yield(double tanfr, double pressure, double cohesion) { return tanfr * pressure + cohesion; }
/* artificialStress / artificialPressure, models.h:212-223 */
inline M3 artificial_stress(double mateps, const M3& sor) {
    M3 m;
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) m.a[d][e] = sor.a[d][e] > 0 ? -mateps * sor.a[d][e] : 0.0;
    return m;
}
/* addStrainRateAndRotationRate, models.h:225-248 */
inline void add_strain_rotation(M3& edot, M3& rdot, double mj, double rhoj, V3 vij, V3 g) {
    const double t = -0.5 * mj / rhoj;
    const double v[3] = {vij.x, vij.y, vij.z};
    const double gw[3] = {g.x, g.y, g.z};
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) {
            edot.a[d][e] += t * (v[d] * gw[e] + v[e] * gw[d]);
            rdot.a[d][e] += t * (v[d] * gw[e] - v[e] * gw[d]);
        }
}
/* dstress_dt, models.h:250-268: Hooke deviatoric rate plus the Jaumann rotation terms */
inline M3 dstress_dt(const M3& edot, const M3& rdot, const M3& S, double shear) {
    M3 out;
    const double tr = edot.a[0][0] + edot.a[1][1] + edot.a[2][2];
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) {
            double v = 2.0 * shear * edot.a[d][e];
            if (d == e) v -= 2.0 * shear * tr / 3.0;
            for (int f = 0; f < 3; ++f) v += S.a[d][f] * rdot.a[e][f] + S.a[e][f] * rdot.a[d][f];
            out.a[d][e] = v;
        }
    return out;
}

/* pressure of the selected EOS (src/computeDerivatives.h:200,205) */
inline double pressure(const gsph_params& p, double rho) {
    if (on(p, GSPH_SOLIDS)) return eos_murnaghan(rho, p.rho0, p.bulk, p.dbulk_dp);
    return eos_liquid(rho, p.rho0, p.soundspeed * p.soundspeed);
}
/* sigma/rho^2 as a full tensor; for fluids the scalar -p/rho^2 on the diagonal with zero
 * off-diagonals, which is what the scalar stress_t path of calcAcceleration computes
 * (src/computeDerivatives.h:180-184, :204-208) */
inline M3 sigma_over_rho2(const gsph_params& p, double rho, const M3& S) {
    M3 s = on(p, GSPH_SOLIDS) ? S : mzero();
    const double pr = pressure(p, rho);
    for (int d = 0; d < 3; ++d) s.a[d][d] -= pr;
    const double r2 = rho * rho;
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) s.a[d][e] /= r2;
    return s;
}

/* environmentAcceleration, src/computeDerivatives.h:33-47. The Clohessy-Wiltshire lines add a
 * scalar to an f3_t, which adds it to every component; that is reproduced as written. */
inline V3 environment_acceleration(const gsph_params& p, V3 pos, V3 vel, V3 acc) {
    if (on(p, GSPH_CLOHESSY_WILTSHIRE)) {
        const double n = p.cw_n;
        const double s1 = 3 * n * n * pos.x + 2 * n * vel.y;
        acc = acc + V3{s1, s1, s1};
        const double s2 = -2 * n * vel.x;
        acc = acc + V3{s2, s2, s2};
        const double s3 = -n * n * pos.z;
        acc = acc + V3{s3, s3, s3};
    }
    if (on(p, GSPH_CONSTANT_ACCELERATION)) acc = acc + V3{p.const_acc[0], p.const_acc[1], p.const_acc[2]};
    return acc;
}

/* ---- the three pair jobs ------------------------------------------------------------------- */

/* calcDensity, src/computeDerivatives.h:52-91: rho_i = sum_{0<r^2<=H^2} m_j W(r); self excluded */
void density_pass(const gsph_params& p, int64_t n, oracle_particles& s) {
    const double H = p.H, H2 = H * H, wf = spline_prefactor(p.dimension, H);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const V3 xi = load3(s.pos, i);
        double rho = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const V3 rij = xi - load3(s.pos, j);
            const double r2 = dot(rij, rij);
            if (r2 <= H2 && r2 > 0) rho += s.mass[j] * w_spline(std::sqrt(r2), H, wf);
        }
        if (on(p, GSPH_DEAL_WITH_NO_PARTNERS) && rho < 0.001) rho = p.rho0 * 0.01;  /* :85-88 */
        s.density[i] = rho;
    }
}

/* calcBalsaraDensityDTDStressDT, src/computeDerivatives.h:96-162, for targets [i0, i1) */
void velocity_gradient_pass(const gsph_params& p, int64_t n, oracle_particles& s, int64_t i0, int64_t i1) {
    const double H = p.H, H2 = H * H, dwf = dspline_prefactor(p.dimension, H);
    const bool solids = on(p, GSPH_SOLIDS), bals = on(p, GSPH_BALSARA_SWITCH), integ = on(p, GSPH_INTEGRATE_DENSITY);
#pragma omp parallel for schedule(static)
    for (int64_t i = i0; i < i1; ++i) {
        const V3 xi = load3(s.pos, i), vi = load3(s.vel, i);
        M3 edot = mzero(), rdot = mzero();
        double divv = 0.0;
        V3 curlv{0, 0, 0};
        for (int64_t j = 0; j < n; ++j) {
            const V3 rij = xi - load3(s.pos, j);
            const double r2 = dot(rij, rij);
            if (r2 <= H2 && r2 > 0) {
                const double r = std::sqrt(r2);
                const double dw = dw_spline(r, H, dwf);
                const V3 g = (dw / r) * rij;
                const V3 vij = vi - load3(s.vel, j);
                const double mj = s.mass[j], rhoj = s.density[j];  /* rho_j, as in :132 */
                if (solids) add_strain_rotation(edot, rdot, mj, rhoj, vij, g);
                else if (bals) curlv = curlv + (mj / rhoj) * cross(vij, g);
                if (bals || integ) divv -= (mj / rhoj) * dot(vij, g);
            }
        }
        double bal = 0.0, rho_dt = 0.0;
        M3 sdt = mzero();
        if (solids) {
            sdt = dstress_dt(edot, rdot, load9(s.dstress, i), p.shear);
            curlv = V3{-2 * rdot.a[1][2], -2 * rdot.a[2][0], -2 * rdot.a[0][1]};
        }
        if (integ) rho_dt = -s.density[i] * divv;
        if (bals) bal = balsara_switch(divv, curlv, p.soundspeed, H);
        s.balsara[i] = bal;
        s.density_dt[i] = rho_dt;
        store9(s.dstress_dt, i, sdt);
    }
}

/* calcAcceleration, src/computeDerivatives.h:167-313, for targets [i0, i1) */
void acceleration_pass(const gsph_params& p, int64_t n, oracle_particles& s, int64_t i0, int64_t i1) {
    const double H = p.H, H2 = H * H, eps2 = p.grav_eps * p.grav_eps, G = p.grav_G;
    const double wf = spline_prefactor(p.dimension, H), dwf = dspline_prefactor(p.dimension, H);
    const bool grav = on(p, GSPH_SELF_GRAVITY), sph = on(p, GSPH_SPH), solids = on(p, GSPH_SOLIDS);
    const bool av = on(p, GSPH_ARTIFICIAL_VISCOSITY), bals = on(p, GSPH_BALSARA_SWITCH);
    const bool arts = on(p, GSPH_ARTIFICIAL_STRESS), xsph = on(p, GSPH_XSPH);
    const double c = p.soundspeed;
    const double w_normalsep = arts ? w_spline(p.normalsep, H, wf) : 1.0;

    /* sigma_j / rho_j^2 depends on j alone; evaluate it once per particle */
    std::vector<M3> sor;
    if (sph) {
        sor.resize(n);
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < n; ++j)
            sor[j] = sigma_over_rho2(p, s.density[j], solids ? load9(s.dstress, j) : mzero());
    }

#pragma omp parallel for schedule(static)
    for (int64_t i = i0; i < i1; ++i) {
        const V3 xi = load3(s.pos, i), vi = load3(s.vel, i);
        const double rhoi = sph ? s.density[i] : 0.0;
        const double bi = bals ? s.balsara[i] : 1.0;
        M3 arts_i = mzero();
        if (sph && arts) arts_i = artificial_stress(p.mateps, sor[i]);  /* :210-217 */
        V3 acc{0, 0, 0}, xv{0, 0, 0};
        double max_vsig = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const V3 rij = xi - load3(s.pos, j);
            const double r2 = dot(rij, rij);
            if (!(r2 > 0)) continue;
            const double mj = s.mass[j];
            if (grav) {  /* :229-235 */
                const double inv = 1.0 / std::sqrt(r2 + eps2);
                acc = acc - rij * (G * mj * inv * inv * inv);
            }
            if (sph && r2 <= H2) {  /* :237-295 */
                const double r = std::sqrt(r2);
                const V3 g = (dw_spline(r, H, dwf) / r) * rij;
                M3 st;
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) st.a[d][e] = sor[i].a[d][e] + sor[j].a[d][e];
                const V3 vij = vi - load3(s.vel, j);
                if (arts) {
                    const double f = std::pow(w_spline(r, H, wf) / w_normalsep, p.matexp);
                    const M3 arts_j = artificial_stress(p.mateps, sor[j]);
                    for (int d = 0; d < 3; ++d)
                        for (int e = 0; e < 3; ++e) st.a[d][e] += f * (arts_i.a[d][e] + arts_j.a[d][e]);
                }
                acc = acc + mj * mul(st, g);
                if (av) {
                    const double bj = bals ? s.balsara[j] : 1.0;
                    const double II = artificial_viscosity(bals ? &max_vsig : nullptr, p.av_alpha, p.av_beta, rhoi,
                                                           s.density[j], vij, rij, r, c, c, bi, bj);
                    acc = acc - (mj * II) * g;
                }
                if (xsph) xv = xv + (2 * mj / (rhoi + s.density[j])) * (load3(s.vel, j) - vi) * w_spline(r, H, wf);
            }
        }
        acc = environment_acceleration(p, xi, vi, acc);
        store3(s.acc, i, acc);
        store3(s.xvel, i, xv);
        s.maxvsig[i] = max_vsig;
    }
}

/* per-particle update shared by the fixed and variable leapfrogs (src/integration.h:94-121 and
 * :185-212): kick with kick_dt, drift with dt, density and stress update, plasticity, boundary */
void kick_drift(const gsph_params& p, int64_t n, oracle_particles& s, double kick_dt, double dt) {
    const bool sph = on(p, GSPH_SPH);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        V3 v = load3(s.vel, i) + load3(s.acc, i) * kick_dt;
        V3 x = load3(s.pos, i);
        if (on(p, GSPH_XSPH) && sph) x = x + (v + p.xsph_factor * load3(s.xvel, i)) * dt;
        else x = x + v * dt;
        if (sph) {
            if (on(p, GSPH_INTEGRATE_DENSITY)) {
                double rho = s.density[i] + s.density_dt[i] * dt;
                if (rho < 0.0) rho = 0.0;
                s.density[i] = rho;
            }
            if (on(p, GSPH_SOLIDS)) {
                M3 S = load9(s.dstress, i);
                const M3 Sd = load9(s.dstress_dt, i);
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) S.a[d][e] += Sd.a[d][e] * dt;
                if (on(p, GSPH_PLASTICITY_MC))  /* doPlasticity, integration.h:24-31 */
                    plasticity(S, mohr_coulomb_yield(p.tanfr, eos_murnaghan(s.density[i], p.rho0, p.bulk, p.dbulk_dp),
                                                      p.cohesion));
                else if (on(p, GSPH_PLASTICITY_MIESE))
                    plasticity(S, p.Y);
                store9(s.dstress, i, S);
            }
        }
        if (on(p, GSPH_SIMPLE_BOX_BOUNDARY)) {  /* handleBoundaryConditions, integration.h:33-73 */
            const double m = 1.0 + p.box_reflectiveness;
            double* xc[3] = {&x.x, &x.y, &x.z};
            double* vc[3] = {&v.x, &v.y, &v.z};
            for (int d = 0; d < 3; ++d) {
                if (d == 2 && p.dimension != 3) break;
                if (*xc[d] > p.box_max[d]) { *xc[d] = p.box_max[d]; *vc[d] -= m * *vc[d]; }
                else if (*xc[d] < p.box_min[d]) { *xc[d] = p.box_min[d]; *vc[d] -= m * *vc[d]; }
            }
        }
        store3(s.vel, i, v);
        store3(s.pos, i, x);
    }
}

}  // namespace

extern "C" {

/* computeDerivatives(pb), src/computeDerivatives.h:315-328. The velocity-gradient and
 * acceleration passes are evaluated for targets [i0, i1) only (i1 < 0 means n); the density pass,
 * which every later pass reads for all j, always covers all particles. */
int oracle_compute_derivatives(const gsph_params* p, int64_t n, oracle_particles* s, int64_t i0, int64_t i1,
                               oracle_timestep* ts) {
    if (!p || !s || n < 0) return GSPH_E_INVALID;
    if (i1 < 0 || i1 > n) i1 = n;
    if (i0 < 0) i0 = 0;
    const gsph_params& P = *p;
    if (on(P, GSPH_SPH)) {
        if (!on(P, GSPH_INTEGRATE_DENSITY)) density_pass(P, n, *s);
        if (on(P, GSPH_SOLIDS) || on(P, GSPH_INTEGRATE_DENSITY) || on(P, GSPH_BALSARA_SWITCH))
            velocity_gradient_pass(P, n, *s, i0, i1);
    }
    acceleration_pass(P, n, *s, i0, i1);
    if (on(P, GSPH_VARIABLE_TIMESTEP) && ts) ts->next = P.max_dt;  /* :306-309 */
    return GSPH_OK;
}

/* integrate(pb, notFirstStep), src/integration.h:219-244 */
int oracle_integrate(const gsph_params* p, int64_t n, int not_first_step, oracle_particles* s, oracle_timestep* ts) {
    if (!p || !s || n < 0) return GSPH_E_INVALID;
    const gsph_params& P = *p;
    if (!on(P, GSPH_VARIABLE_TIMESTEP)) {  /* fixedTsLeapfrog, :82-125 */
        const double dt = P.fixed_dt;
        kick_drift(P, n, *s, dt * (not_first_step ? 1.0 : 0.5), dt);
        return GSPH_OK;
    }
    if (!ts) return GSPH_E_INVALID;
    if (not_first_step) {  /* variableTsLeapfrog_getNewTimestep, :130-169 */
        const double dt = ts->current;
        double mindt = P.max_dt;
        for (int64_t i = 0; i < n; ++i) {
            V3 v = load3(s->vel, i) + load3(s->acc, i) * (dt * 0.5);
            store3(s->vel, i, v);
            if (on(P, GSPH_ACCELERATION_CRITERION))
                mindt = std::min(mindt, std::sqrt(P.accel_accuracy * P.H / length(load3(s->acc, i))));
            if (on(P, GSPH_VELOCITY_CRITERION))
                mindt = std::min(mindt, P.velocity_accuracy * P.H / s->maxvsig[i]);
        }
        ts->next = std::min(ts->next, mindt);
    } else {
        ts->next = P.initial_dt;  /* :235-236 */
    }
    /* variableTsLeapfrog_useNewTimestep, :171-217 */
    const double dt = ts->next < P.min_dt ? P.min_dt : ts->next;
    ts->current = dt;
    kick_drift(P, n, *s, dt * 0.5, dt);
    return GSPH_OK;
}

/* Gravity-only accelerations (FP64) of `nt` target particles idx[] against all n sources:
 * a_i = -G sum_{j, r>0} m_j r_ij (r^2+eps^2)^-3/2 (src/computeDerivatives.h:226-235). */
int oracle_gravity_targets(const gsph_params* p, int64_t n, const double* pos, const double* mass, int64_t nt,
                           const int64_t* idx, double* acc_out) {
    if (!p || !pos || !mass || !idx || !acc_out) return GSPH_E_INVALID;
    const double eps2 = p->grav_eps * p->grav_eps, G = p->grav_G;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t i = idx[t];
        const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
        double ax = 0, ay = 0, az = 0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = xi - pos[3 * j], dy = yi - pos[3 * j + 1], dz = zi - pos[3 * j + 2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 > 0)) continue;
            const double inv = 1.0 / std::sqrt(r2 + eps2);
            const double s = G * mass[j] * inv * inv * inv;
            ax -= dx * s; ay -= dy * s; az -= dz * s;
        }
        acc_out[3 * t] = ax; acc_out[3 * t + 1] = ay; acc_out[3 * t + 2] = az;
    }
    return GSPH_OK;
}

/* FP64 diagnostics (no reference counterpart). Velocity used: v + half_kick * a. */
int oracle_diagnostics(const gsph_params* p, int64_t n, const oracle_particles* s, double half_kick, gsph_diag* out) {
    if (!p || !s || !out) return GSPH_E_INVALID;
    const gsph_params& P = *p;
    const double eps2 = P.grav_eps * P.grav_eps;
    double ek = 0, eg = 0, ei = 0, es = 0, px = 0, py = 0, pz = 0, lx = 0, ly = 0, lz = 0, mt = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : ek, eg, ei, es, px, py, pz, lx, ly, lz, mt)
    for (int64_t i = 0; i < n; ++i) {
        const double m = s->mass[i];
        const V3 x = load3(s->pos, i);
        V3 v = load3(s->vel, i);
        if (half_kick != 0.0) v = v + load3(s->acc, i) * half_kick;
        ek += 0.5 * m * dot(v, v);
        px += m * v.x; py += m * v.y; pz += m * v.z;
        const V3 L = cross(x, v);
        lx += m * L.x; ly += m * L.y; lz += m * L.z;
        mt += m;
        if (on(P, GSPH_SELF_GRAVITY)) {
            double phi = 0;
            for (int64_t j = i + 1; j < n; ++j) {
                const V3 d = x - load3(s->pos, j);
                phi += s->mass[j] / std::sqrt(dot(d, d) + eps2);
            }
            eg -= P.grav_G * m * phi;
        }
        if (on(P, GSPH_SPH)) {
            const double rho = s->density[i];
            double u;
            if (on(P, GSPH_SOLIDS)) {
                const double K = P.bulk, nn = P.dbulk_dp, r0 = P.rho0;
                if (std::fabs(nn - 1.0) < 1e-12)
                    u = K / r0 * (std::log(rho / r0) + r0 / rho - 1.0);
                else
                    u = K / nn * ((std::pow(rho, nn - 1.0) - std::pow(r0, nn - 1.0)) / ((nn - 1.0) * std::pow(r0, nn)) +
                                  (1.0 / rho - 1.0 / r0));
                const M3 S = load9(s->dstress, i);
                double ss = 0;
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) ss += S.a[d][e] * S.a[d][e];
                es += m * ss / (4.0 * P.shear * rho);
            } else {
                const double c2 = P.soundspeed * P.soundspeed;
                u = c2 * (std::log(rho / P.rho0) + P.rho0 / rho - 1.0);
            }
            ei += m * u;
        }
    }
    out->e_kin = ek; out->e_grav = eg; out->e_int = ei; out->e_shear = es;
    out->momentum[0] = px; out->momentum[1] = py; out->momentum[2] = pz;
    out->ang_mom[0] = lx; out->ang_mom[1] = ly; out->ang_mom[2] = lz;
    out->mass = mt;
    return GSPH_OK;
}

/* Kernel functions exposed for known-answer tests. */
double oracle_w_spline(int dim, double r, double h) { return w_spline(r, h, spline_prefactor(dim, h)); }
double oracle_dw_spline(int dim, double r, double h) { return dw_spline(r, h, dspline_prefactor(dim, h)); }

/* Plasticity limiter on one row-major 3x3 tensor (KAT). */
void oracle_plasticity(double* S9, double Y) {
    M3 S = load9(S9, 0);
    plasticity(S, Y);
    store9(S9, 0, S);
}

/* Jaumann stress rate for one particle (KAT). */
void oracle_dstress_dt(const double* edot9, const double* rdot9, const double* S9, double shear, double* out9) {
    store9(out9, 0, dstress_dt(load9(edot9, 0), load9(rdot9, 0), load9(S9, 0), shear));
}

int oracle_abi_version(void) { return GSPH_ABI_VERSION; }

}  // extern "C"
