// fp64.cu -- the double-precision build of the hot path: GraSPH2's DOUBLE_PRECISION switch
// (settings/precisionSettings.h:16-17, src/types.h:32-43: f1_t = double, m3_t = Mat<double,3,3>).
//
// Same physics and pass sequence as the FP32 kernels, in FP64 throughout, with plain all-pairs
// shared-memory tiles (each thread owns one i and sums every j, so no partial sums): the reference's
// tile loop (src/particles/algorithms.h:270-309) without its remainder bug. B200 runs FP64 at half
// the FP32 rate, so this mode is the accuracy reference for trajectories the FP32 forms are measured
// against (energy drift), and the drop-in for callers of the reference's FP64 build.
#include "fp64.cuh"

namespace gsph {

namespace {

constexpr int kT64 = 128;  // threads per block = j-tile of the FP64 kernels

inline unsigned blocks_for(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

__host__ __device__ __forceinline__ bool has64(const DevParams64& p, uint32_t f) { return (p.flags & f) != 0; }

// ---- src/sph/kernel.h, eos.h, models.h in FP64 ----------------------------------------------------
__device__ __forceinline__ double w_poly64(double q) {  // kernel.h:130-136 without the prefactor
    if (q > 1.0) return 0.0;
    if (q < 0.5) return 6.0 * q * q * q - 6.0 * q * q + 1.0;
    const double a = 1.0 - q;
    return 2.0 * a * a * a;
}
__device__ __forceinline__ double dw_poly64(double q) {  // kernel.h:169-175
    if (q > 1.0) return 0.0;
    if (q < 0.5) return 3.0 * q * q - 2.0 * q;
    const double a = 1.0 - q;
    return -a * a;
}
__device__ __forceinline__ double pressure64(const DevParams64& p, double rho) {  // eos.h:88-96
    if (has64(p, GSPH_SOLIDS)) return p.bulk / p.dbulk * (pow(rho / p.rho0, p.dbulk) - 1.0);
    return p.c * p.c * (rho - p.rho0);
}
__device__ __forceinline__ double art64(double mateps, double s) { return s > 0.0 ? -mateps * s : 0.0; }

__device__ __forceinline__ void jrecord64(const DevParams64& p, double rho, double4 sA, double4 sB, double bal,
                                          double4& jA, double4& jB) {
    const double pres = pressure64(p, rho);
    const double r2 = rho * rho;
    if (has64(p, GSPH_SOLIDS)) {
        jA = make_double4((sA.x - pres) / r2, (sA.y - pres) / r2, (sA.z - pres) / r2, sA.w / r2);
        jB = make_double4(sB.x / r2, sB.y / r2, bal, 0.0);
    } else {
        const double s = -pres / r2;
        jA = make_double4(s, s, s, 0.0);
        jB = make_double4(0.0, 0.0, bal, 0.0);
    }
}

// ---- density ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kT64) k64_density(DevArrays64 a, DevParams64 p) {
    __shared__ double4 tile[kT64];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kT64 + threadIdx.x;
    const double4 pi = a.posm[i];
    double rho = 0.0;
    for (int64_t t0 = 0; t0 < a.n_pad; t0 += kT64) {
        __syncthreads();
        tile[threadIdx.x] = a.posm[t0 + threadIdx.x];
        __syncthreads();
        for (int j = 0; j < kT64; ++j) {
            const double4 q = tile[j];
            const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 <= p.H2 && r2 > 0.0) rho += q.w * w_poly64(sqrt(r2) / p.H);  // computeDerivatives.h:72
        }
    }
    if (i >= a.n) return;
    rho *= p.w_pref;
    if (has64(p, GSPH_DEAL_WITH_NO_PARTNERS) && rho < 0.001) rho = p.rho0 * 0.01;  // :85-88
    double4 vr = a.velrho[i];
    vr.w = rho;
    a.velrho[i] = vr;
    double4 jA, jB;
    jrecord64(p, rho, a.sA[i], a.sB[i], a.balsara[i], jA, jB);
    a.jA[i] = jA;
    a.jB[i] = jB;
}

__global__ void k64_prepare(DevArrays64 a, DevParams64 p) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    double4 jA, jB;
    jrecord64(p, a.velrho[i].w, a.sA[i], a.sB[i], a.balsara[i], jA, jB);
    a.jA[i] = jA;
    a.jB[i] = jB;
}

// ---- velocity gradient / acceleration passes ------------------------------------------------------
// PASS as in pairs.cuh: 0 velocity gradient (calcBalsaraDensityDTDStressDT), 1 acceleration
// (calcAcceleration), 2 both in one sweep.
template <int PASS, bool SOLIDS>
__global__ void __launch_bounds__(kT64) k64_pairs(DevArrays64 a, DevParams64 p) {
    constexpr bool DO_V = PASS != 1;
    constexpr bool DO_A = PASS != 0;
    __shared__ double4 P[kT64], V[kT64], JA[kT64], JB[kT64];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kT64 + threadIdx.x;
    const double4 pi = a.posm[i], vi = a.velrho[i];
    const double4 jAi = a.jA[i], jBi = a.jB[i];
    const bool grav = DO_A && has64(p, GSPH_SELF_GRAVITY);
    const bool sph = has64(p, GSPH_SPH);
    const bool bals = has64(p, GSPH_BALSARA_SWITCH), av = has64(p, GSPH_ARTIFICIAL_VISCOSITY);
    const bool xsph = has64(p, GSPH_XSPH), arts = has64(p, GSPH_ARTIFICIAL_STRESS);
    const bool divv_on = bals || has64(p, GSPH_INTEGRATE_DENSITY);
    const double bi = bals ? jBi.z : 1.0;
    const double ai[6] = {art64(p.mateps, jAi.x), art64(p.mateps, jAi.y), art64(p.mateps, jAi.z),
                          art64(p.mateps, jAi.w), art64(p.mateps, jBi.x), art64(p.mateps, jBi.y)};
    double gx = 0, gy = 0, gz = 0, ax = 0, ay = 0, az = 0, xv0 = 0, xv1 = 0, xv2 = 0, maxv = 0;
    double E[6] = {0, 0, 0, 0, 0, 0}, W[3] = {0, 0, 0}, divv = 0, cu[3] = {0, 0, 0};
    for (int64_t t0 = 0; t0 < a.n_pad; t0 += kT64) {
        __syncthreads();
        P[threadIdx.x] = a.posm[t0 + threadIdx.x];
        V[threadIdx.x] = a.velrho[t0 + threadIdx.x];
        if (DO_A) {
            JA[threadIdx.x] = a.jA[t0 + threadIdx.x];
            JB[threadIdx.x] = a.jB[t0 + threadIdx.x];
        }
        __syncthreads();
        for (int j = 0; j < kT64; ++j) {
            const double4 q = P[j];
            const double rx = pi.x - q.x, ry = pi.y - q.y, rz = pi.z - q.z;  // r_ij
            const double r2 = rx * rx + ry * ry + rz * rz;
            if (!(r2 > 0.0)) continue;
            if (grav) {  // computeDerivatives.h:229-235
                const double inv = 1.0 / sqrt(r2 + p.eps2);
                const double s = q.w * inv * inv * inv;
                gx -= rx * s; gy -= ry * s; gz -= rz * s;
            }
            if (!sph || r2 > p.H2) continue;
            const double r = sqrt(r2);
            const double qq = r / p.H;
            const double dwr = p.dw_pref * dw_poly64(qq) / r;
            const double g0 = dwr * rx, g1 = dwr * ry, g2 = dwr * rz;  // grad_i W
            const double4 vj = V[j];
            const double vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
            const double mj = q.w, rhoj = vj.w;
            if (DO_V) {
                const double mr = mj / rhoj;
                if (SOLIDS) {  // models.h:225-248
                    const double t = -0.5 * mr;
                    E[0] += t * (vx * g0 + vx * g0); E[1] += t * (vy * g1 + vy * g1); E[2] += t * (vz * g2 + vz * g2);
                    E[3] += t * (vx * g1 + vy * g0); E[4] += t * (vx * g2 + vz * g0); E[5] += t * (vy * g2 + vz * g1);
                    W[0] += t * (vx * g1 - vy * g0); W[1] += t * (vx * g2 - vz * g0); W[2] += t * (vy * g2 - vz * g1);
                } else if (bals) {
                    cu[0] += mr * (vy * g2 - vz * g1); cu[1] += mr * (vz * g0 - vx * g2); cu[2] += mr * (vx * g1 - vy * g0);
                }
                if (divv_on) divv -= mr * (vx * g0 + vy * g1 + vz * g2);
            }
            if (DO_A) {
                const double4 ja = JA[j], jb = JB[j];
                double st[6] = {jAi.x + ja.x, jAi.y + ja.y, jAi.z + ja.z, jAi.w + ja.w, jBi.x + jb.x, jBi.y + jb.y};
                if (arts) {
                    const double f = pow(p.w_pref * w_poly64(qq) * p.inv_w_normalsep, p.matexp);
                    const double aj[6] = {art64(p.mateps, ja.x), art64(p.mateps, ja.y), art64(p.mateps, ja.z),
                                          art64(p.mateps, ja.w), art64(p.mateps, jb.x), art64(p.mateps, jb.y)};
                    for (int k = 0; k < 6; ++k) st[k] += f * (ai[k] + aj[k]);
                }
                // (xx, yy, zz, xy, xz, yz) . grad W
                ax += mj * (st[0] * g0 + st[3] * g1 + st[4] * g2);
                ay += mj * (st[3] * g0 + st[1] * g1 + st[5] * g2);
                az += mj * (st[4] * g0 + st[5] * g1 + st[2] * g2);
                if (av) {  // models.h:158-185
                    const double w = (rx * vx + ry * vy + rz * vz) / r;
                    if (w < 0.0) {
                        const double vsig = p.c + p.c - p.beta * w;
                        const double rhoij = (vi.w + rhoj) * 0.5;
                        const double bj = bals ? jb.z : 1.0;
                        const double II = -0.25 * (bi + bj) * p.alpha * w * vsig / rhoij;
                        ax -= mj * II * g0; ay -= mj * II * g1; az -= mj * II * g2;
                        if (bals) maxv = fmax(maxv, vsig);
                    }
                }
                if (xsph) {
                    const double f = 2.0 * mj / (vi.w + rhoj) * (p.w_pref * w_poly64(qq));
                    xv0 -= f * vx; xv1 -= f * vy; xv2 -= f * vz;
                }
            }
        }
    }
    if (i >= a.n) return;
    if (DO_V) {  // calcBalsaraDensityDTDStressDT::do_after (:144-161)
        double c0 = cu[0], c1 = cu[1], c2 = cu[2];
        if (SOLIDS) {
            const double Em[3][3] = {{E[0], E[3], E[4]}, {E[3], E[1], E[5]}, {E[4], E[5], E[2]}};
            const double R[3][3] = {{0.0, W[0], W[1]}, {-W[0], 0.0, W[2]}, {-W[1], -W[2], 0.0}};
            const double4 sa = a.sA[i], sb = a.sB[i];
            const double Sm[3][3] = {{sa.x, sa.w, sb.x}, {sa.w, sa.y, sb.y}, {sb.x, sb.y, sa.z}};
            const double tr = Em[0][0] + Em[1][1] + Em[2][2];
            double D[3][3];
            for (int d = 0; d < 3; ++d)
                for (int e = 0; e < 3; ++e) {  // dstress_dt, models.h:250-268
                    double v = 2.0 * p.shear * Em[d][e];
                    if (d == e) v -= 2.0 * p.shear * tr / 3.0;
                    for (int f = 0; f < 3; ++f) v += Sm[d][f] * R[e][f] + Sm[e][f] * R[d][f];
                    D[d][e] = v;
                }
            a.dA[i] = make_double4(D[0][0], D[1][1], D[2][2], 0.5 * (D[0][1] + D[1][0]));
            a.dB[i] = make_double4(0.5 * (D[0][2] + D[2][0]), 0.5 * (D[1][2] + D[2][1]), 0.0, 0.0);
            c0 = -2.0 * R[1][2];
            c1 = -2.0 * R[2][0];
            c2 = -2.0 * R[0][1];
        }
        a.rhodot[i] = has64(p, GSPH_INTEGRATE_DENSITY) ? -vi.w * divv : 0.0;
        double bal = 0.0;
        if (bals) {  // models.h:187-192
            const double absdiv = fabs(divv);
            bal = absdiv / (absdiv + sqrt(c0 * c0 + c1 * c1 + c2 * c2) + 0.0001 * p.c / p.H);
            double4 jb = a.jB[i];
            jb.z = bal;
            a.jB[i] = jb;
        }
        a.balsara[i] = bal;
    }
    if (DO_A) {  // calcAcceleration::do_after (:301-312), environmentAcceleration (:33-47)
        ax += p.G * gx;
        ay += p.G * gy;
        az += p.G * gz;
        if (has64(p, GSPH_CLOHESSY_WILTSHIRE)) {
            const double n = p.cw_n;
            const double s1 = 3 * n * n * pi.x + 2 * n * vi.y, s2 = -2 * n * vi.x, s3 = -n * n * pi.z;
            ax += s1 + s2 + s3; ay += s1 + s2 + s3; az += s1 + s2 + s3;
        }
        if (has64(p, GSPH_CONSTANT_ACCELERATION)) {
            ax += p.const_acc[0]; ay += p.const_acc[1]; az += p.const_acc[2];
        }
        a.acc[i] = make_double4(ax, ay, az, maxv);
        a.xvel[i] = make_double4(xv0, xv1, xv2, 0.0);
        if (has64(p, GSPH_VARIABLE_TIMESTEP) && i == 0) a.dt_state[1] = p.max_dt;  // :306-309
    }
}

// ---- leapfrog (src/integration.h) ---------------------------------------------------------------------
__device__ __forceinline__ void plasticity64(double4& a, double4& b, double Y) {  // models.h:194-205
    const double J2 = 0.5 * (a.x * a.x + a.y * a.y + a.z * a.z + 2.0 * (a.w * a.w + b.x * b.x + b.y * b.y));
    const double f = Y * Y / (3.0 * J2);
    if (f < 1.0) {
        a.x *= f; a.y *= f; a.z *= f; a.w *= f;
        b.x *= f; b.y *= f;
    }
}

__device__ __forceinline__ void kick_drift64(const DevArrays64& a, const DevParams64& p, int64_t i, double kick_dt,
                                             double dt) {
    double4 vr = a.velrho[i];
    const double4 ac = a.acc[i];
    vr.x += ac.x * kick_dt; vr.y += ac.y * kick_dt; vr.z += ac.z * kick_dt;
    double4 x = a.posm[i];
    const bool sph = has64(p, GSPH_SPH);
    double ux = vr.x, uy = vr.y, uz = vr.z;
    if (sph && has64(p, GSPH_XSPH)) {
        const double4 xv = a.xvel[i];
        ux += p.xsph * xv.x; uy += p.xsph * xv.y; uz += p.xsph * xv.z;
    }
    x.x += ux * dt; x.y += uy * dt; x.z += uz * dt;
    if (sph) {
        if (has64(p, GSPH_INTEGRATE_DENSITY)) {
            double rho = vr.w + a.rhodot[i] * dt;
            if (rho < 0.0) rho = 0.0;
            vr.w = rho;
        }
        if (has64(p, GSPH_SOLIDS)) {
            double4 sa = a.sA[i], sb = a.sB[i];
            const double4 da = a.dA[i], db = a.dB[i];
            sa.x += da.x * dt; sa.y += da.y * dt; sa.z += da.z * dt; sa.w += da.w * dt;
            sb.x += db.x * dt; sb.y += db.y * dt;
            if (has64(p, GSPH_PLASTICITY_MC))
                plasticity64(sa, sb, p.tanfr * (p.bulk / p.dbulk * (pow(vr.w / p.rho0, p.dbulk) - 1.0)) + p.cohesion);
            else if (has64(p, GSPH_PLASTICITY_MIESE))
                plasticity64(sa, sb, p.Y);
            a.sA[i] = sa;
            a.sB[i] = sb;
        }
    }
    if (has64(p, GSPH_SIMPLE_BOX_BOUNDARY)) {
        const double m = 1.0 + p.box_refl;
        double* xc[3] = {&x.x, &x.y, &x.z};
        double* vc[3] = {&vr.x, &vr.y, &vr.z};
        for (int d = 0; d < 3; ++d) {
            if (d == 2 && p.dim != 3) break;
            if (*xc[d] > p.box_max[d]) { *xc[d] = p.box_max[d]; *vc[d] -= m * *vc[d]; }
            else if (*xc[d] < p.box_min[d]) { *xc[d] = p.box_min[d]; *vc[d] -= m * *vc[d]; }
        }
    }
    a.posm[i] = x;
    a.velrho[i] = vr;
}

__global__ void k64_leapfrog_fixed(DevArrays64 a, DevParams64 p, double kick_dt) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < a.n) kick_drift64(a, p, i, kick_dt, p.fixed_dt);
}

// variable step (integration.h:130-217); dt_state holds positive doubles, min-reduced as int64
__global__ void k64_dt_criteria(DevArrays64 a, DevParams64 p) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const double dt = a.dt_state[0];
    double mindt = p.max_dt;
    if (i < a.n) {
        double4 vr = a.velrho[i];
        const double4 ac = a.acc[i];
        vr.x += ac.x * dt * 0.5; vr.y += ac.y * dt * 0.5; vr.z += ac.z * dt * 0.5;
        a.velrho[i] = vr;
        if (has64(p, GSPH_ACCELERATION_CRITERION))
            mindt = fmin(mindt, sqrt(p.accel_acc * p.H / sqrt(ac.x * ac.x + ac.y * ac.y + ac.z * ac.z)));
        if (has64(p, GSPH_VELOCITY_CRITERION)) mindt = fmin(mindt, p.vel_acc * p.H / ac.w);
    }
    for (int o = 16; o > 0; o >>= 1) mindt = fmin(mindt, __shfl_xor_sync(0xffffffffu, mindt, o));
    if ((threadIdx.x & 31) == 0)
        atomicMin(reinterpret_cast<unsigned long long*>(a.dt_state + 1),
                  static_cast<unsigned long long>(__double_as_longlong(mindt)));
}
__global__ void k64_dt_first(DevArrays64 a, DevParams64 p) {
    if (threadIdx.x == 0 && blockIdx.x == 0) a.dt_state[1] = p.initial_dt;
}
__global__ void k64_leapfrog_variable(DevArrays64 a, DevParams64 p) {
    const double nxt = a.dt_state[1];
    const double dt = nxt < p.min_dt ? p.min_dt : nxt;
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < a.n) kick_drift64(a, p, i, dt * 0.5, dt);
}
__global__ void k64_dt_commit(DevArrays64 a, DevParams64 p) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const double nxt = a.dt_state[1];
        a.dt_state[0] = nxt < p.min_dt ? p.min_dt : nxt;
    }
}

// ---- transfers: caller's float attributes (and FP64 positions) <-> device doubles --------------------
__global__ void k64_pack(DevArrays64 a, int attr, const float* __restrict__ src) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    switch (attr) {
        case 0: { double4 q = a.posm[i]; q.x = src[3 * i]; q.y = src[3 * i + 1]; q.z = src[3 * i + 2]; a.posm[i] = q; break; }
        case 1: { double4 q = a.posm[i]; q.w = src[i]; a.posm[i] = q; break; }
        case 2: { double4 q = a.velrho[i]; q.x = src[3 * i]; q.y = src[3 * i + 1]; q.z = src[3 * i + 2]; a.velrho[i] = q; break; }
        case 3: { double4 q = a.acc[i]; q.x = src[3 * i]; q.y = src[3 * i + 1]; q.z = src[3 * i + 2]; a.acc[i] = q; break; }
        case 4: a.balsara[i] = src[i]; break;
        case 5: a.xvel[i] = make_double4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0); break;
        case 6: { double4 q = a.velrho[i]; q.w = src[i]; a.velrho[i] = q; break; }
        case 7: a.rhodot[i] = src[i]; break;
        case 8:
        case 9: {
            const float* m = src + 9 * i;
            const double4 A = make_double4(m[0], m[4], m[8], 0.5 * (double(m[1]) + m[3]));
            const double4 B = make_double4(0.5 * (double(m[2]) + m[6]), 0.5 * (double(m[5]) + m[7]), 0.0, 0.0);
            if (attr == 8) { a.sA[i] = A; a.sB[i] = B; }
            else { a.dA[i] = A; a.dB[i] = B; }
            break;
        }
        case 10: { double4 q = a.acc[i]; q.w = src[i]; a.acc[i] = q; break; }
        default: break;
    }
}

__global__ void k64_unpack(DevArrays64 a, int attr, float* __restrict__ dst) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    auto f = [](double v) { return static_cast<float>(v); };
    switch (attr) {
        case 0: { const double4 q = a.posm[i]; dst[3 * i] = f(q.x); dst[3 * i + 1] = f(q.y); dst[3 * i + 2] = f(q.z); break; }
        case 1: dst[i] = f(a.posm[i].w); break;
        case 2: { const double4 q = a.velrho[i]; dst[3 * i] = f(q.x); dst[3 * i + 1] = f(q.y); dst[3 * i + 2] = f(q.z); break; }
        case 3: { const double4 q = a.acc[i]; dst[3 * i] = f(q.x); dst[3 * i + 1] = f(q.y); dst[3 * i + 2] = f(q.z); break; }
        case 4: dst[i] = f(a.balsara[i]); break;
        case 5: { const double4 q = a.xvel[i]; dst[3 * i] = f(q.x); dst[3 * i + 1] = f(q.y); dst[3 * i + 2] = f(q.z); break; }
        case 6: dst[i] = f(a.velrho[i].w); break;
        case 7: dst[i] = f(a.rhodot[i]); break;
        case 8:
        case 9: {
            const double4 A = (attr == 8) ? a.sA[i] : a.dA[i];
            const double4 B = (attr == 8) ? a.sB[i] : a.dB[i];
            float* m = dst + 9 * i;
            m[0] = f(A.x); m[1] = f(A.w); m[2] = f(B.x);
            m[3] = f(A.w); m[4] = f(A.y); m[5] = f(B.y);
            m[6] = f(B.x); m[7] = f(B.y); m[8] = f(A.z);
            break;
        }
        case 10: dst[i] = f(a.acc[i].w); break;
        default: break;
    }
}

// `acc64`: caller-side double output of one attribute (3 or 1 components) -- the FP64 download
__global__ void k64_unpack_d(DevArrays64 a, int attr, double* __restrict__ dst) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    double4 q;
    switch (attr) {
        case 0: q = a.posm[i]; break;
        case 2: q = a.velrho[i]; break;
        case 3: q = a.acc[i]; break;
        default: q = make_double4(a.velrho[i].w, 0, 0, 0);  // density
    }
    if (attr == 6) {
        dst[i] = q.x;
    } else {
        dst[3 * i] = q.x; dst[3 * i + 1] = q.y; dst[3 * i + 2] = q.z;
    }
}

// double host layout <-> device doubles, every attribute (the DOUBLE_PRECISION host buffers)
__global__ void k64_pack_f64(DevArrays64 a, int attr, const double* __restrict__ src) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    switch (attr) {
        case 0: { double4 q = a.posm[i]; q.x = src[3 * i]; q.y = src[3 * i + 1]; q.z = src[3 * i + 2]; a.posm[i] = q; break; }
        case 1: { double4 q = a.posm[i]; q.w = src[i]; a.posm[i] = q; break; }
        case 2: { double4 q = a.velrho[i]; q.x = src[3 * i]; q.y = src[3 * i + 1]; q.z = src[3 * i + 2]; a.velrho[i] = q; break; }
        case 3: { double4 q = a.acc[i]; q.x = src[3 * i]; q.y = src[3 * i + 1]; q.z = src[3 * i + 2]; a.acc[i] = q; break; }
        case 4: a.balsara[i] = src[i]; break;
        case 5: a.xvel[i] = make_double4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0); break;
        case 6: { double4 q = a.velrho[i]; q.w = src[i]; a.velrho[i] = q; break; }
        case 7: a.rhodot[i] = src[i]; break;
        case 8:
        case 9: {
            const double* m = src + 9 * i;
            const double4 A = make_double4(m[0], m[4], m[8], 0.5 * (m[1] + m[3]));
            const double4 B = make_double4(0.5 * (m[2] + m[6]), 0.5 * (m[5] + m[7]), 0.0, 0.0);
            if (attr == 8) { a.sA[i] = A; a.sB[i] = B; }
            else { a.dA[i] = A; a.dB[i] = B; }
            break;
        }
        case 10: { double4 q = a.acc[i]; q.w = src[i]; a.acc[i] = q; break; }
        default: break;
    }
}

__global__ void k64_unpack_f64(DevArrays64 a, int attr, double* __restrict__ dst) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    switch (attr) {
        case 0: { const double4 q = a.posm[i]; dst[3 * i] = q.x; dst[3 * i + 1] = q.y; dst[3 * i + 2] = q.z; break; }
        case 1: dst[i] = a.posm[i].w; break;
        case 2: { const double4 q = a.velrho[i]; dst[3 * i] = q.x; dst[3 * i + 1] = q.y; dst[3 * i + 2] = q.z; break; }
        case 3: { const double4 q = a.acc[i]; dst[3 * i] = q.x; dst[3 * i + 1] = q.y; dst[3 * i + 2] = q.z; break; }
        case 4: dst[i] = a.balsara[i]; break;
        case 5: { const double4 q = a.xvel[i]; dst[3 * i] = q.x; dst[3 * i + 1] = q.y; dst[3 * i + 2] = q.z; break; }
        case 6: dst[i] = a.velrho[i].w; break;
        case 7: dst[i] = a.rhodot[i]; break;
        case 8:
        case 9: {
            const double4 A = (attr == 8) ? a.sA[i] : a.dA[i];
            const double4 B = (attr == 8) ? a.sB[i] : a.dB[i];
            double* m = dst + 9 * i;
            m[0] = A.x; m[1] = A.w; m[2] = B.x;
            m[3] = A.w; m[4] = A.y; m[5] = B.y;
            m[6] = B.x; m[7] = B.y; m[8] = A.z;
            break;
        }
        case 10: dst[i] = a.acc[i].w; break;
        default: break;
    }
}

__global__ void k_narrow(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<float>(in[i]);
}
__global__ void k_widen(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

__global__ void k64_pack_pos(DevArrays64 a, const double* __restrict__ src) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    double4 q = a.posm[i];
    q.x = src[3 * i]; q.y = src[3 * i + 1]; q.z = src[3 * i + 2];
    a.posm[i] = q;
}

__global__ void k64_init(DevArrays64 a) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n_pad) return;
    const double4 z = make_double4(0, 0, 0, 0);
    a.posm[i] = (i < a.n) ? z : make_double4(1e18, 1e18, 1e18, 0.0);
    a.velrho[i] = (i < a.n) ? z : make_double4(0, 0, 0, 1.0);
    a.acc[i] = z; a.xvel[i] = z; a.sA[i] = z; a.sB[i] = z; a.dA[i] = z; a.dB[i] = z; a.jA[i] = z; a.jB[i] = z;
    a.rhodot[i] = 0.0;
    a.balsara[i] = 0.0;
}

// ---- FP64 diagnostics (same quantities as the FP32 path) ---------------------------------------------
constexpr int kDiag64 = 12;
__global__ void __launch_bounds__(kT64) k64_diag(DevArrays64 a, DevParams64 p, double half_kick, double* blocks) {
    __shared__ double4 tile[kT64];
    __shared__ double red[kT64 / 32][kDiag64];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kT64 + threadIdx.x;
    double f[kDiag64] = {};
    const double4 x = a.posm[i];
    if (i < a.n) {
        const double4 vr = a.velrho[i], ac = a.acc[i];
        const double m = x.w;
        const double vx = vr.x + half_kick * ac.x, vy = vr.y + half_kick * ac.y, vz = vr.z + half_kick * ac.z;
        f[0] = 0.5 * m * (vx * vx + vy * vy + vz * vz);
        f[4] = m * vx; f[5] = m * vy; f[6] = m * vz;
        f[7] = m * (x.y * vz - x.z * vy); f[8] = m * (x.z * vx - x.x * vz); f[9] = m * (x.x * vy - x.y * vx);
        f[10] = m;
        if (has64(p, GSPH_SPH)) {
            const double rho = vr.w, r0 = p.rho0;
            if (has64(p, GSPH_SOLIDS)) {
                const double K = p.bulk, nn = p.dbulk;
                f[2] = m * ((fabs(nn - 1.0) < 1e-12)
                                ? K / r0 * (log(rho / r0) + r0 / rho - 1.0)
                                : K / nn * ((pow(rho, nn - 1.0) - pow(r0, nn - 1.0)) / ((nn - 1.0) * pow(r0, nn)) +
                                            (1.0 / rho - 1.0 / r0)));
                const double4 sa = a.sA[i], sb = a.sB[i];
                const double ss = sa.x * sa.x + sa.y * sa.y + sa.z * sa.z + 2.0 * (sa.w * sa.w + sb.x * sb.x + sb.y * sb.y);
                f[3] = m * ss / (4.0 * p.shear * rho);
            } else {
                f[2] = m * p.c * p.c * (log(rho / r0) + r0 / rho - 1.0);
            }
        }
    }
    if (has64(p, GSPH_SELF_GRAVITY)) {  // -G m_i sum_{j > i} m_j / sqrt(r^2 + eps^2)
        double phi = 0.0;
        for (int64_t t0 = static_cast<int64_t>(blockIdx.x) * kT64; t0 < a.n_pad; t0 += kT64) {
            __syncthreads();
            tile[threadIdx.x] = a.posm[t0 + threadIdx.x];
            __syncthreads();
            for (int jj = 0; jj < kT64; ++jj) {
                if (t0 + jj <= i) continue;
                const double4 q = tile[jj];
                const double dx = q.x - x.x, dy = q.y - x.y, dz = q.z - x.z;
                phi += q.w / sqrt(dx * dx + dy * dy + dz * dz + p.eps2);
            }
        }
        if (i < a.n) f[1] = -p.G * x.w * phi;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < kDiag64; ++k) {
        double v = f[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < kDiag64) {
        double s = 0.0;
        for (int w = 0; w < kT64 / 32; ++w) s += red[w][threadIdx.x];
        blocks[static_cast<int64_t>(blockIdx.x) * kDiag64 + threadIdx.x] = s;
    }
}
__global__ void k64_diag_reduce(const double* blocks, int nblocks, double* out) {
    const int k = threadIdx.x;
    if (k >= kDiag64) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += blocks[static_cast<int64_t>(b) * kDiag64 + k];
    out[k] = s;
}

}  // namespace

DevParams64 make_dev_params64(const gsph_params& p, double w_pref, double dw_pref, double inv_w_normalsep) {
    DevParams64 d{};
    d.flags = p.flags;
    d.dim = p.dimension;
    d.H = p.H;
    d.H2 = p.H * p.H;
    d.eps2 = p.grav_eps * p.grav_eps;
    d.G = p.grav_G;
    d.w_pref = w_pref;
    d.dw_pref = dw_pref;
    d.rho0 = p.rho0;
    d.bulk = p.bulk;
    d.dbulk = p.dbulk_dp;
    d.c = p.soundspeed;
    d.shear = p.shear;
    d.Y = p.Y;
    d.tanfr = p.tanfr;
    d.cohesion = p.cohesion;
    d.alpha = p.av_alpha;
    d.beta = p.av_beta;
    d.mateps = p.mateps;
    d.matexp = p.matexp;
    d.inv_w_normalsep = inv_w_normalsep;
    d.xsph = p.xsph_factor;
    d.fixed_dt = p.fixed_dt;
    d.initial_dt = p.initial_dt;
    d.min_dt = p.min_dt;
    d.max_dt = p.max_dt;
    d.accel_acc = p.accel_accuracy;
    d.vel_acc = p.velocity_accuracy;
    d.cw_n = p.cw_n;
    for (int k = 0; k < 3; ++k) {
        d.const_acc[k] = p.const_acc[k];
        d.box_min[k] = p.box_min[k];
        d.box_max[k] = p.box_max[k];
    }
    d.box_refl = p.box_reflectiveness;
    return d;
}

cudaError_t launch64_init(const DevArrays64& a, cudaStream_t s) {
    k64_init<<<blocks_for(a.n_pad, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch64_derivatives(const DevArrays64& a, const DevParams64& p, cudaStream_t s, int& launches) {
    const unsigned nb = static_cast<unsigned>(a.n_pad / kT64);
    const bool sph = has64(p, GSPH_SPH);
    if (sph) {
        if (!has64(p, GSPH_INTEGRATE_DENSITY)) k64_density<<<nb, kT64, 0, s>>>(a, p);
        else k64_prepare<<<blocks_for(a.n, 256), 256, 0, s>>>(a, p);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ++launches;
    }
    const bool solids = has64(p, GSPH_SOLIDS);
    const bool vgrad = sph && (solids || has64(p, GSPH_INTEGRATE_DENSITY) || has64(p, GSPH_BALSARA_SWITCH));
    if (vgrad && has64(p, GSPH_BALSARA_SWITCH)) {
        if (solids) k64_pairs<0, true><<<nb, kT64, 0, s>>>(a, p);
        else k64_pairs<0, false><<<nb, kT64, 0, s>>>(a, p);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (solids) k64_pairs<1, true><<<nb, kT64, 0, s>>>(a, p);
        else k64_pairs<1, false><<<nb, kT64, 0, s>>>(a, p);
        launches += 2;
    } else if (vgrad) {
        if (solids) k64_pairs<2, true><<<nb, kT64, 0, s>>>(a, p);
        else k64_pairs<2, false><<<nb, kT64, 0, s>>>(a, p);
        ++launches;
    } else {
        if (solids) k64_pairs<1, true><<<nb, kT64, 0, s>>>(a, p);
        else k64_pairs<1, false><<<nb, kT64, 0, s>>>(a, p);
        ++launches;
    }
    return cudaGetLastError();
}

cudaError_t launch64_leapfrog(const DevArrays64& a, const DevParams64& p, int not_first_step, cudaStream_t s,
                              int& launches) {
    const unsigned nb = blocks_for(a.n, 256);
    if (!has64(p, GSPH_VARIABLE_TIMESTEP)) {
        k64_leapfrog_fixed<<<nb, 256, 0, s>>>(a, p, p.fixed_dt * (not_first_step ? 1.0 : 0.5));
        ++launches;
        return cudaGetLastError();
    }
    if (not_first_step) k64_dt_criteria<<<nb, 256, 0, s>>>(a, p);
    else k64_dt_first<<<1, 32, 0, s>>>(a, p);
    k64_leapfrog_variable<<<nb, 256, 0, s>>>(a, p);
    k64_dt_commit<<<1, 32, 0, s>>>(a, p);
    launches += 3;
    return cudaGetLastError();
}

cudaError_t launch64_pack(const DevArrays64& a, int attr, const float* src, cudaStream_t s) {
    k64_pack<<<blocks_for(a.n, 256), 256, 0, s>>>(a, attr, src);
    return cudaGetLastError();
}
cudaError_t launch64_unpack(const DevArrays64& a, int attr, float* dst, cudaStream_t s) {
    k64_unpack<<<blocks_for(a.n, 256), 256, 0, s>>>(a, attr, dst);
    return cudaGetLastError();
}
cudaError_t launch64_unpack_d(const DevArrays64& a, int attr, double* dst, cudaStream_t s) {
    k64_unpack_d<<<blocks_for(a.n, 256), 256, 0, s>>>(a, attr, dst);
    return cudaGetLastError();
}
cudaError_t launch64_pack_f64(const DevArrays64& a, int attr, const double* src, cudaStream_t s) {
    k64_pack_f64<<<blocks_for(a.n, 256), 256, 0, s>>>(a, attr, src);
    return cudaGetLastError();
}
cudaError_t launch64_unpack_f64(const DevArrays64& a, int attr, double* dst, cudaStream_t s) {
    k64_unpack_f64<<<blocks_for(a.n, 256), 256, 0, s>>>(a, attr, dst);
    return cudaGetLastError();
}
cudaError_t launch_narrow(const double* in, float* out, int64_t n, cudaStream_t s) {
    k_narrow<<<blocks_for(n, 256), 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}
cudaError_t launch_widen(const float* in, double* out, int64_t n, cudaStream_t s) {
    k_widen<<<blocks_for(n, 256), 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}
cudaError_t launch64_pack_pos(const DevArrays64& a, const double* src, cudaStream_t s) {
    k64_pack_pos<<<blocks_for(a.n, 256), 256, 0, s>>>(a, src);
    return cudaGetLastError();
}
size_t diag64_scratch_doubles(int64_t n_pad) { return static_cast<size_t>(n_pad / kT64) * kDiag64 + kDiag64; }
cudaError_t launch64_diagnostics(const DevArrays64& a, const DevParams64& p, double half_kick, double* scratch,
                                 double* out, cudaStream_t s) {
    const int nb = static_cast<int>(a.n_pad / kT64);
    k64_diag<<<nb, kT64, 0, s>>>(a, p, half_kick, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k64_diag_reduce<<<1, 32, 0, s>>>(scratch, nb, out);
    return cudaGetLastError();
}

}  // namespace gsph
