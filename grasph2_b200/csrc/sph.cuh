// sph.cuh -- the per-pair and per-particle physics shared by the all-pairs, culled and ensemble
// kernels: spline kernel, equations of state, j-records sigma/rho^2, the SPH terms of one
// neighbour pair, the environment acceleration, plasticity and the leapfrog update of one particle.
#pragma once

#include "pairs.cuh"

namespace gsph {

// ---- SPH building blocks (src/sph/kernel.h, eos.h, models.h) ---------------------------------
// spline polynomial of Wspline without its prefactor, q in [0,1] (kernel.h:130-136)
__device__ __forceinline__ float w_poly(float q) {
    if (q > 1.0f) return 0.0f;
    if (q < 0.5f) return 6.0f * q * q * q - 6.0f * q * q + 1.0f;
    const float a = 1.0f - q;
    return 2.0f * a * a * a;
}
// polynomial of dWspline without its prefactor (kernel.h:169-175)
__device__ __forceinline__ float dw_poly(float q) {
    if (q > 1.0f) return 0.0f;
    if (q < 0.5f) return 3.0f * q * q - 2.0f * q;
    const float a = 1.0f - q;
    return -a * a;
}
// pressure of the selected EOS (eos.h:88-96; computeDerivatives.h:200,205)
__device__ __forceinline__ float eos_pressure(const DevParams& p, float rho) {
    if (has(p, GSPH_SOLIDS)) return p.bulk / p.dbulk * (powf(rho / p.rho0, p.dbulk) - 1.0f);
    return p.c2 * (rho - p.rho0);
}
// j-record of one particle: sigma/rho^2 in (A, B) with B.z = Balsara value
__device__ __forceinline__ void make_jrecord(const DevParams& p, float rho, float4 sA, float4 sB, float bal,
                                             float4& jA, float4& jB) {
    const float pres = eos_pressure(p, rho);
    if (has(p, GSPH_SOLIDS)) {
        jA = make_float4((sA.x - pres) / (rho * rho), (sA.y - pres) / (rho * rho), (sA.z - pres) / (rho * rho),
                         sA.w / (rho * rho));
        jB = make_float4(sB.x / (rho * rho), sB.y / (rho * rho), bal, 0.0f);
    } else {
        const float s = -pres / (rho * rho);
        jA = make_float4(s, s, s, 0.0f);
        jB = make_float4(0.0f, 0.0f, bal, 0.0f);
    }
}
// artificialStress / artificialPressure (models.h:212-223)
__device__ __forceinline__ float art(float mateps, float s) { return s > 0.0f ? -mateps * s : 0.0f; }

// neighbour test 0 < x <= hi for a non-negative float x, on the bit patterns: one add, one compare
__device__ __forceinline__ bool in_open_closed(float x, uint32_t lo_bits, uint32_t span_bits) {
    return (__float_as_uint(x) - lo_bits - 1u) < span_bits;
}

struct PairAcc {
    float f[F_COUNT];
};

// Per-i state of the SPH pair passes and the run-time switches the pair body reads.
struct ISph {
    float4 pi, vi, jAi, jBi;
    float bi;
    float ai_xx, ai_yy, ai_zz, ai_xy, ai_xz, ai_yz;  // artificial stress of i (computeDerivatives.h:210-217)
    bool bals, av, xsph, arts, curl, divv_on;
    float eps2;           // added to r^2 when gravity shares the squared distance
    uint32_t lo, span;    // neighbour window 0 < r^2 <= H^2 on the bit patterns of r^2 + eps2
};

template <int PASS, bool SOLIDS>
__device__ __forceinline__ ISph load_isph(const DevArrays& a, const DevParams& p, int64_t i, float eps2) {
    constexpr bool DO_A = PASS != PASS_VGRAD;
    ISph s;
    s.pi = a.posm[i];
    s.vi = a.velrho[i];
    s.jAi = make_float4(0, 0, 0, 0);
    s.jBi = make_float4(0, 0, 0, 0);
    if (DO_A) {
        s.jAi = a.jA[i];
        s.jBi = a.jB[i];
    }
    s.bals = has(p, GSPH_BALSARA_SWITCH);
    s.av = has(p, GSPH_ARTIFICIAL_VISCOSITY);
    s.xsph = has(p, GSPH_XSPH);
    s.arts = has(p, GSPH_ARTIFICIAL_STRESS);
    s.curl = !SOLIDS && s.bals;
    s.divv_on = s.bals || has(p, GSPH_INTEGRATE_DENSITY);
    s.bi = s.bals ? s.jBi.z : 1.0f;
    s.ai_xx = art(p.mateps, s.jAi.x); s.ai_yy = art(p.mateps, s.jAi.y); s.ai_zz = art(p.mateps, s.jAi.z);
    s.ai_xy = art(p.mateps, s.jAi.w); s.ai_xz = art(p.mateps, s.jBi.x); s.ai_yz = art(p.mateps, s.jBi.y);
    s.eps2 = eps2;
    s.lo = __float_as_uint(eps2);
    s.span = __float_as_uint(p.H2 + eps2) - s.lo;
    return s;
}

// The SPH terms of one neighbour pair (0 < r <= H): velocity-gradient terms
// (computeDerivatives.h:118-141) and acceleration terms (:237-295). d = x_j - x_i, r2 = |d|^2.
template <int PASS, bool SOLIDS>
__device__ __forceinline__ void sph_neighbour(PairAcc& T, float& maxv, const ISph& I, float mj, float dx, float dy,
                                              float dz, float r2, float4 vj, float4 ja, float4 jb, const DevParams& p) {
    constexpr bool DO_V = PASS != PASS_ACC;
    constexpr bool DO_A = PASS != PASS_VGRAD;
    const float inv_r = rsqrtf(r2);
    const float r = r2 * inv_r;
    const float qq = r * p.inv_h;
    // grad_i W = (dW/r) r_ij with r_ij = -d:  g = -(dW/r) d
    const float gf = -p.dw_pref * dw_poly(qq) * inv_r;
    const float gx = gf * dx, gy = gf * dy, gz = gf * dz;
    const float vx = I.vi.x - vj.x, vy = I.vi.y - vj.y, vz = I.vi.z - vj.z;  // v_ij
    const float rhoj = vj.w;
    if (DO_V) {
        const float mr = mj / rhoj;
        if (SOLIDS) {  // addStrainRateAndRotationRate (models.h:225-248)
            const float t = -0.5f * mr;
            T.f[F_E00] = fmaf(t, vx * gx + vx * gx, T.f[F_E00]);
            T.f[F_E11] = fmaf(t, vy * gy + vy * gy, T.f[F_E11]);
            T.f[F_E22] = fmaf(t, vz * gz + vz * gz, T.f[F_E22]);
            T.f[F_E01] = fmaf(t, vx * gy + vy * gx, T.f[F_E01]);
            T.f[F_E02] = fmaf(t, vx * gz + vz * gx, T.f[F_E02]);
            T.f[F_E12] = fmaf(t, vy * gz + vz * gy, T.f[F_E12]);
            T.f[F_W01] = fmaf(t, vx * gy - vy * gx, T.f[F_W01]);
            T.f[F_W02] = fmaf(t, vx * gz - vz * gx, T.f[F_W02]);
            T.f[F_W12] = fmaf(t, vy * gz - vz * gy, T.f[F_W12]);
        } else if (I.curl) {
            T.f[F_C0] = fmaf(mr, vy * gz - vz * gy, T.f[F_C0]);
            T.f[F_C1] = fmaf(mr, vz * gx - vx * gz, T.f[F_C1]);
            T.f[F_C2] = fmaf(mr, vx * gy - vy * gx, T.f[F_C2]);
        }
        if (I.divv_on) T.f[F_DIVV] = fmaf(-mr, vx * gx + vy * gy + vz * gz, T.f[F_DIVV]);
    }
    if (DO_A) {
        float sxx = I.jAi.x + ja.x, syy = I.jAi.y + ja.y, szz = I.jAi.z + ja.z;
        float sxy = I.jAi.w + ja.w, sxz = I.jBi.x + jb.x, syz = I.jBi.y + jb.y;
        if (I.arts) {
            const float f = powf(p.w_pref * w_poly(qq) * p.inv_w_normalsep, p.matexp);
            sxx += f * (I.ai_xx + art(p.mateps, ja.x));
            syy += f * (I.ai_yy + art(p.mateps, ja.y));
            szz += f * (I.ai_zz + art(p.mateps, ja.z));
            sxy += f * (I.ai_xy + art(p.mateps, ja.w));
            sxz += f * (I.ai_xz + art(p.mateps, jb.x));
            syz += f * (I.ai_yz + art(p.mateps, jb.y));
        }
        T.f[F_AX] = fmaf(mj, sxx * gx + sxy * gy + sxz * gz, T.f[F_AX]);
        T.f[F_AY] = fmaf(mj, sxy * gx + syy * gy + syz * gz, T.f[F_AY]);
        T.f[F_AZ] = fmaf(mj, sxz * gx + syz * gy + szz * gz, T.f[F_AZ]);
        if (I.av) {  // artificialViscosity (models.h:158-185)
            const float w = -(dx * vx + dy * vy + dz * vz) * inv_r;  // r_ij . v_ij / r
            if (w < 0.0f) {
                const float vsig = p.c + p.c - p.beta * w;
                const float rhoij = (I.vi.w + rhoj) * 0.5f;
                const float bj = I.bals ? jb.z : 1.0f;
                const float II = -0.25f * (I.bi + bj) * p.alpha * w * vsig / rhoij;
                const float m2 = -mj * II;
                T.f[F_AX] = fmaf(m2, gx, T.f[F_AX]);
                T.f[F_AY] = fmaf(m2, gy, T.f[F_AY]);
                T.f[F_AZ] = fmaf(m2, gz, T.f[F_AZ]);
                if (I.bals) maxv = fmaxf(maxv, vsig);
            }
        }
        if (I.xsph) {
            const float f = 2.0f * mj / (I.vi.w + rhoj) * (p.w_pref * w_poly(qq));
            T.f[F_XV0] = fmaf(f, -vx, T.f[F_XV0]);
            T.f[F_XV1] = fmaf(f, -vy, T.f[F_XV1]);
            T.f[F_XV2] = fmaf(f, -vz, T.f[F_XV2]);
        }
    }
}

// environmentAcceleration (computeDerivatives.h:33-47); the Clohessy-Wiltshire terms are scalars
// added to all three components, as the reference's f3_t += f1_t does
__device__ __forceinline__ void environment(const DevParams& p, float4 x, float4 v, float& ax, float& ay, float& az) {
    if (has(p, GSPH_CLOHESSY_WILTSHIRE)) {
        const float n = p.cw_n;
        const float s1 = 3 * n * n * x.x + 2 * n * v.y;
        ax += s1; ay += s1; az += s1;
        const float s2 = -2 * n * v.x;
        ax += s2; ay += s2; az += s2;
        const float s3 = -n * n * x.z;
        ax += s3; ay += s3; az += s3;
    }
    if (has(p, GSPH_CONSTANT_ACCELERATION)) {
        ax += p.const_acc[0];
        ay += p.const_acc[1];
        az += p.const_acc[2];
    }
}

// do_after of the SPH passes for particle i: calcBalsaraDensityDTDStressDT (computeDerivatives.h:144-161:
// Jaumann stress rate, drho/dt, Balsara switch) and calcAcceleration (:301-312: G times the gravity
// sum g when `grav`, environment acceleration, max signal velocity, XSPH). val(f) is the summed
// field f of the pair pass.
template <int PASS, bool SOLIDS, typename Val>
__device__ __forceinline__ void sph_finish(const DevArrays& a, const DevParams& p, int64_t i, Val&& val, bool grav,
                                           const float* g) {
    const float4 vi = a.velrho[i];
    if (PASS != PASS_ACC) {  // calcBalsaraDensityDTDStressDT::do_after (:144-161)
        const float divv = val(F_DIVV);
        float c0 = 0, c1 = 0, c2 = 0;
        if (SOLIDS) {
            const float e[6] = {val(F_E00), val(F_E11), val(F_E22), val(F_E01), val(F_E02), val(F_E12)};
            const float w01 = val(F_W01), w02 = val(F_W02), w12 = val(F_W12);
            const float E[3][3] = {{e[0], e[3], e[4]}, {e[3], e[1], e[5]}, {e[4], e[5], e[2]}};
            const float R[3][3] = {{0.0f, w01, w02}, {-w01, 0.0f, w12}, {-w02, -w12, 0.0f}};
            const float4 sa = a.sA[i], sb = a.sB[i];
            const float Sm[3][3] = {{sa.x, sa.w, sb.x}, {sa.w, sa.y, sb.y}, {sb.x, sb.y, sa.z}};
            const float tr = E[0][0] + E[1][1] + E[2][2];
            float D[3][3];
            // dstress_dt (models.h:250-268): Hooke deviatoric rate + Jaumann rotation terms
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int ee = 0; ee < 3; ++ee) {
                    float v = 2.0f * p.shear * E[d][ee];
                    if (d == ee) v -= 2.0f * p.shear * tr / 3.0f;
#pragma unroll
                    for (int f = 0; f < 3; ++f) v += Sm[d][f] * R[ee][f] + Sm[ee][f] * R[d][f];
                    D[d][ee] = v;
                }
            a.dA[i] = make_float4(D[0][0], D[1][1], D[2][2], 0.5f * (D[0][1] + D[1][0]));
            a.dB[i] = make_float4(0.5f * (D[0][2] + D[2][0]), 0.5f * (D[1][2] + D[2][1]), 0.0f, 0.0f);
            c0 = -2.0f * R[1][2];
            c1 = -2.0f * R[2][0];
            c2 = -2.0f * R[0][1];
        } else {
            c0 = val(F_C0);
            c1 = val(F_C1);
            c2 = val(F_C2);
        }
        a.rhodot[i] = has(p, GSPH_INTEGRATE_DENSITY) ? -vi.w * divv : 0.0f;
        float bal = 0.0f;
        if (has(p, GSPH_BALSARA_SWITCH)) {  // balsaraSwitch (models.h:187-192)
            const float absdiv = fabsf(divv);
            const float abscurl = sqrtf(c0 * c0 + c1 * c1 + c2 * c2);
            bal = absdiv / (absdiv + abscurl + p.balsara_floor);
            float4 jb = a.jB[i];
            jb.z = bal;
            a.jB[i] = jb;
            if (a.jrec) a.jrec[4 * i + 3] = jb;
        }
        a.balsara[i] = bal;
    }
    if (PASS != PASS_VGRAD) {  // calcAcceleration::do_after (:301-312)
        float ax = val(F_AX), ay = val(F_AY), az = val(F_AZ);
        if (grav) {
            ax = fmaf(p.G, g[0], ax);
            ay = fmaf(p.G, g[1], ay);
            az = fmaf(p.G, g[2], az);
            if (a.grav) a.grav[i] = make_float4(p.G * g[0], p.G * g[1], p.G * g[2], 0.0f);
        }
        const float4 x = a.posm[i];
        environment(p, x, vi, ax, ay, az);
        a.acc[i] = make_float4(ax, ay, az, val(F_MAXV));
        a.xvel[i] = make_float4(val(F_XV0), val(F_XV1), val(F_XV2), 0.0f);
    }
}

__device__ __forceinline__ float murnaghan(const DevParams& p, float rho) {
    return p.bulk / p.dbulk * (powf(rho / p.rho0, p.dbulk) - 1.0f);
}

// plasticity (src/sph/models.h:194-205) on the six stored components of the symmetric S:
// J2 = 1/2 sum_de S_de^2 counts each off-diagonal twice; S *= Y^2/(3 J2) when that is < 1
__device__ __forceinline__ void plasticity(float4& a, float4& b, float Y) {
    const float J2 = 0.5f * (a.x * a.x + a.y * a.y + a.z * a.z + 2.0f * (a.w * a.w + b.x * b.x + b.y * b.y));
    const float f = Y * Y / (3.0f * J2);
    if (f < 1.0f) {
        a.x *= f; a.y *= f; a.z *= f; a.w *= f;
        b.x *= f; b.y *= f;
    }
}

// the per-particle update shared by fixedTsLeapfrog (integration.h:90-124) and
// variableTsLeapfrog_useNewTimestep (:171-217): kick, drift (FP64 master position), density and
// stress update, plasticity, box boundary
__device__ __forceinline__ void kick_drift(const DevArrays& a, const DevParams& p, int64_t i, float kick_dt, float dt) {
    float4 vr = a.velrho[i];
    const float4 ac = a.acc[i];
    vr.x = fmaf(ac.x, kick_dt, vr.x);
    vr.y = fmaf(ac.y, kick_dt, vr.y);
    vr.z = fmaf(ac.z, kick_dt, vr.z);
    float ux = vr.x, uy = vr.y, uz = vr.z;
    const bool sph = has(p, GSPH_SPH);
    if (sph && has(p, GSPH_XSPH)) {
        const float4 xv = a.xvel[i];
        ux = fmaf(p.xsph, xv.x, ux);
        uy = fmaf(p.xsph, xv.y, uy);
        uz = fmaf(p.xsph, xv.z, uz);
    }
    const int64_t np = a.n_pad;
    double x = a.pos64[i], y = a.pos64[np + i], z = a.pos64[2 * np + i];
    x += static_cast<double>(ux) * static_cast<double>(dt);
    y += static_cast<double>(uy) * static_cast<double>(dt);
    z += static_cast<double>(uz) * static_cast<double>(dt);
    if (sph) {
        if (has(p, GSPH_INTEGRATE_DENSITY)) {
            float rho = fmaf(a.rhodot[i], dt, vr.w);
            if (rho < 0.0f) rho = 0.0f;
            vr.w = rho;
        }
        if (has(p, GSPH_SOLIDS)) {
            float4 sa = a.sA[i], sb = a.sB[i];
            const float4 da = a.dA[i], db = a.dB[i];
            sa.x = fmaf(da.x, dt, sa.x); sa.y = fmaf(da.y, dt, sa.y); sa.z = fmaf(da.z, dt, sa.z);
            sa.w = fmaf(da.w, dt, sa.w); sb.x = fmaf(db.x, dt, sb.x); sb.y = fmaf(db.y, dt, sb.y);
            if (has(p, GSPH_PLASTICITY_MC))  // doPlasticity (integration.h:24-31), updated density
                plasticity(sa, sb, p.tanfr * murnaghan(p, vr.w) + p.cohesion);
            else if (has(p, GSPH_PLASTICITY_MIESE))
                plasticity(sa, sb, p.Y);
            a.sA[i] = sa;
            a.sB[i] = sb;
        }
    }
    if (has(p, GSPH_SIMPLE_BOX_BOUNDARY)) {  // handleBoundaryConditions (integration.h:33-73)
        const float m = 1.0f + p.box_refl;
        double* xc[3] = {&x, &y, &z};
        float* vc[3] = {&vr.x, &vr.y, &vr.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d == 2 && p.dim != 3) break;
            if (*xc[d] > static_cast<double>(p.box_max[d])) {
                *xc[d] = p.box_max[d];
                *vc[d] -= m * *vc[d];
            } else if (*xc[d] < static_cast<double>(p.box_min[d])) {
                *xc[d] = p.box_min[d];
                *vc[d] -= m * *vc[d];
            }
        }
    }
    a.pos64[i] = x;
    a.pos64[np + i] = y;
    a.pos64[2 * np + i] = z;
    const float mass = a.posm[i].w;
    a.posm[i] = make_float4(static_cast<float>(x), static_cast<float>(y), static_cast<float>(z), mass);
    a.velrho[i] = vr;
}


// FP64 per-particle diagnostic terms (every field but the pair potential f[1]): kinetic energy at the
// velocity v + half_kick a, momentum, angular momentum about the origin, mass, internal energy of the
// barotropic EOS and the elastic shear energy S:S / (4 mu rho)
__device__ __forceinline__ void diag_terms(const DevArrays& a, const DevParams& p, int64_t i, double half_kick,
                                           double* f) {
    const int64_t np = a.n_pad;
    const float4 pm = a.posm[i];
    const float4 vr = a.velrho[i];
    const float4 ac = a.acc[i];
    const double mi = pm.w;
    const double xi = a.pos64[i], yi = a.pos64[np + i], zi = a.pos64[2 * np + i];
    const double vx = vr.x + half_kick * ac.x, vy = vr.y + half_kick * ac.y, vz = vr.z + half_kick * ac.z;
    f[0] = 0.5 * mi * (vx * vx + vy * vy + vz * vz);
    f[4] = mi * vx; f[5] = mi * vy; f[6] = mi * vz;
    f[7] = mi * (yi * vz - zi * vy); f[8] = mi * (zi * vx - xi * vz); f[9] = mi * (xi * vy - yi * vx);
    f[10] = mi;
    if (has(p, GSPH_SPH)) {
        const double rho = vr.w, r0 = p.rho0;
        if (has(p, GSPH_SOLIDS)) {
            const double K = p.bulk, nn = p.dbulk;
            double u;
            if (fabs(nn - 1.0) < 1e-12) u = K / r0 * (log(rho / r0) + r0 / rho - 1.0);
            else u = K / nn * ((pow(rho, nn - 1.0) - pow(r0, nn - 1.0)) / ((nn - 1.0) * pow(r0, nn)) + (1.0 / rho - 1.0 / r0));
            f[2] = mi * u;
            const float4 sa = a.sA[i], sb = a.sB[i];
            const double ss = double(sa.x) * sa.x + double(sa.y) * sa.y + double(sa.z) * sa.z +
                              2.0 * (double(sa.w) * sa.w + double(sb.x) * sb.x + double(sb.y) * sb.y);
            f[3] = mi * ss / (4.0 * p.shear * rho);
        } else {
            const double c2 = double(p.c) * p.c;
            f[2] = mi * c2 * (log(rho / r0) + r0 / rho - 1.0);
        }
    }
}

}  // namespace gsph
