// ics.cu -- initial conditions generated on the device: uniform spheres, Plummer spheres, the
// particle-source modifiers (move, rotate, positional noise, angular / linear / random velocity,
// constant attributes) and the centre-of-mass correction (the reference's particle sources,
// src/initialConditions/particleSources/UniformSphere.cu and PlummerSphere.cu, ParticleSource.h, and
// InitGenerator.h:113-152), so large inputs need no host generation or transfer.
//
// Random numbers are counter-based: value k of particle i under seed s is
//     u = (splitmix64(splitmix64(s + k) + i) >> 11) * 2^-53        (Steele, Lea & Flood 2014)
// so every particle's draws are independent of the launch shape and a host restatement reproduces
// them exactly.
#include <cmath>
#include <string>

#include "common.cuh"

void set_global_error(const std::string& msg);  // capi.cu

namespace {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ double uniform(uint64_t seed, uint64_t k, uint64_t i) {
    return static_cast<double>(splitmix64(splitmix64(seed + k) + i) >> 11) * (1.0 / 9007199254740992.0);
}

constexpr double kPi = 3.14159265358979323846;

// isotropic unit vector from draws k, k+1
__device__ __forceinline__ void direction(uint64_t seed, uint64_t k, uint64_t i, double* d) {
    const double ct = 2.0 * uniform(seed, k, i) - 1.0;
    const double ph = 2.0 * kPi * uniform(seed, k + 1, i);
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    d[0] = st * cos(ph);
    d[1] = st * sin(ph);
    d[2] = ct;
}

// uniform in a sphere of radius R (inverse CDF r = R u^(1/3)); rigid rotation v = omega x x;
// equal masses total_mass / n; density rho0
__global__ void k_uniform_sphere(int64_t n, double R, double mass, double rho0, double wx, double wy, double wz,
                                 uint64_t seed, float* pos, float* vel, float* m, float* rho) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d[3];
    direction(seed, 1, i, d);
    const double r = R * cbrt(uniform(seed, 0, i));
    const double x = r * d[0], y = r * d[1], z = r * d[2];
    pos[3 * i] = static_cast<float>(x);
    pos[3 * i + 1] = static_cast<float>(y);
    pos[3 * i + 2] = static_cast<float>(z);
    if (vel) {
        vel[3 * i] = static_cast<float>(wy * z - wz * y);
        vel[3 * i + 1] = static_cast<float>(wz * x - wx * z);
        vel[3 * i + 2] = static_cast<float>(wx * y - wy * x);
    }
    if (m) m[i] = static_cast<float>(mass);
    if (rho) rho[i] = static_cast<float>(rho0);
}

// Plummer sphere (Aarseth, Henon & Wielen 1974): r = a / sqrt(u^(-2/3) - 1); speed q * v_esc with q
// drawn by rejection from g(q) = q^2 (1 - q^2)^(7/2) (bounded number of tries; the last draw is kept)
__global__ void k_plummer(int64_t n, double a, double M, double G, uint64_t seed, float* pos, float* vel, float* m) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double u = fmin(fmax(uniform(seed, 0, i), 1e-300), 1.0 - 1e-16);
    const double r = a / sqrt(pow(u, -2.0 / 3.0) - 1.0);
    double d[3];
    direction(seed, 1, i, d);
    pos[3 * i] = static_cast<float>(r * d[0]);
    pos[3 * i + 1] = static_cast<float>(r * d[1]);
    pos[3 * i + 2] = static_cast<float>(r * d[2]);
    double q = 0.0;
    for (int t = 0; t < 1000; ++t) {
        const double x = uniform(seed, 3 + 2 * t, i), y = 0.1 * uniform(seed, 4 + 2 * t, i);
        q = x;
        if (y <= x * x * pow(1.0 - x * x, 3.5)) break;
    }
    const double speed = q * sqrt(2.0 * G * M / sqrt(r * r + a * a));
    double e[3];
    direction(seed, 2003, i, e);
    vel[3 * i] = static_cast<float>(speed * e[0]);
    vel[3 * i + 1] = static_cast<float>(speed * e[1]);
    vel[3 * i + 2] = static_cast<float>(speed * e[2]);
    if (m) m[i] = static_cast<float>(M / static_cast<double>(n));
}

// mass-weighted sums of position and velocity (FP64, block partials then one block; fixed order)
__global__ void k_com_partial(int64_t n, const float* pos, const float* vel, const float* m, double* part) {
    __shared__ double sh[7][256];
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double mi = m[i];
        s[0] += mi;
        for (int c = 0; c < 3; ++c) {
            s[1 + c] += mi * pos[3 * i + c];
            if (vel) s[4 + c] += mi * vel[3 * i + c];
        }
    }
    for (int k = 0; k < 7; ++k) sh[k][threadIdx.x] = s[k];
    __syncthreads();
    if (threadIdx.x < 7) {
        double t = 0.0;
        for (int j = 0; j < static_cast<int>(blockDim.x); ++j) t += sh[threadIdx.x][j];
        part[blockIdx.x * 7 + threadIdx.x] = t;
    }
}

// shift by (target - mean): the targets are zero for gsph_ic_com_correct; a NULL target leaves that field
struct ComTarget {
    double com[3], vcom[3];
    int set_com, set_vcom;
};
__global__ void k_com_apply(int64_t n, float* pos, float* vel, const double* part, int nparts, ComTarget t) {
    __shared__ double c[7];
    if (threadIdx.x < 7) {
        double s = 0.0;
        for (int b = 0; b < nparts; ++b) s += part[b * 7 + threadIdx.x];
        c[threadIdx.x] = s;
    }
    __syncthreads();
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n || c[0] == 0.0) return;
    for (int k = 0; k < 3; ++k) {
        if (t.set_com) pos[3 * i + k] = static_cast<float>(pos[3 * i + k] + (t.com[k] - c[1 + k] / c[0]));
        if (vel && t.set_vcom) vel[3 * i + k] = static_cast<float>(vel[3 * i + k] + (t.vcom[k] - c[4 + k] / c[0]));
    }
}

// the modifier list of a particle source, applied per particle in order (arithmetic in FP64, stored FP32)
struct IcOps {
    int n;
    gsph_ic_op op[GSPH_IC_MAX_OPS];
};
struct IcArrays {
    float* a[11];  // gsph_host_particles in attribute-bit order
};
__global__ void k_ic_modify(int64_t n, IcOps ops, IcArrays arr) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* pos = arr.a[0];
    float* vel = arr.a[2];
    double x[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    if (pos)
        for (int c = 0; c < 3; ++c) x[c] = pos[3 * i + c];
    if (vel)
        for (int c = 0; c < 3; ++c) v[c] = vel[3 * i + c];
    for (int k = 0; k < ops.n; ++k) {
        const gsph_ic_op& o = ops.op[k];
        switch (o.kind) {
            case GSPH_IC_MOVE:
                for (int c = 0; c < 3; ++c) x[c] += o.v[c];
                break;
            case GSPH_IC_ROTATE: {  // v[0..8]: the rotation matrix, row-major (built on the host)
                double y[3], w[3];
                for (int r = 0; r < 3; ++r) {
                    y[r] = o.v[3 * r] * x[0] + o.v[3 * r + 1] * x[1] + o.v[3 * r + 2] * x[2];
                    w[r] = o.v[3 * r] * v[0] + o.v[3 * r + 1] * v[1] + o.v[3 * r + 2] * v[2];
                }
                for (int c = 0; c < 3; ++c) {
                    x[c] = y[c];
                    v[c] = w[c];
                }
                break;
            }
            case GSPH_IC_POS_NOISE:
                for (int c = 0; c < 3; ++c) x[c] += o.v[0] * (2.0 * uniform(o.seed, c, i) - 1.0);
                break;
            case GSPH_IC_ANGULAR_VEL:
                v[0] += o.v[1] * x[2] - o.v[2] * x[1];
                v[1] += o.v[2] * x[0] - o.v[0] * x[2];
                v[2] += o.v[0] * x[1] - o.v[1] * x[0];
                break;
            case GSPH_IC_LINEAR_VEL:
                for (int c = 0; c < 3; ++c) v[c] += o.v[c];
                break;
            case GSPH_IC_RANDOM_VEL:
                for (int c = 0; c < 3; ++c) v[c] += o.v[0] * (2.0 * uniform(o.seed, c, i) - 1.0);
                break;
            case GSPH_IC_SET_CONSTANT: {
                const int b = __ffs(static_cast<int>(o.attr)) - 1;
                const int kc = (b == 8 || b == 9) ? 9 : ((b == 0 || b == 2 || b == 3 || b == 5) ? 3 : 1);
                if (b == 0)
                    for (int c = 0; c < 3; ++c) x[c] = o.v[c];
                else if (b == 2)
                    for (int c = 0; c < 3; ++c) v[c] = o.v[c];
                else
                    for (int c = 0; c < kc; ++c) arr.a[b][kc * i + c] = static_cast<float>(o.v[c]);
                break;
            }
            default:
                break;
        }
    }
    if (pos)
        for (int c = 0; c < 3; ++c) pos[3 * i + c] = static_cast<float>(x[c]);
    if (vel)
        for (int c = 0; c < 3; ++c) vel[3 * i + c] = static_cast<float>(v[c]);
}

inline unsigned blocks_for(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

int ic_fail(cudaError_t e, const char* what) {
    set_global_error(std::string(what) + ": " + cudaGetErrorString(e));
    return GSPH_E_CUDA;
}

}  // namespace

extern "C" {

int gsph_ic_uniform_sphere(int64_t n, double radius, double total_mass, double rho0, const double* omega,
                           uint64_t seed, float* pos, float* vel, float* mass, float* density, void* stream) {
    if (n < 1 || !pos || !(radius > 0)) {
        set_global_error("gsph_ic_uniform_sphere: n >= 1, radius > 0 and pos are required");
        return GSPH_E_INVALID;
    }
    const double w[3] = {omega ? omega[0] : 0.0, omega ? omega[1] : 0.0, omega ? omega[2] : 0.0};
    k_uniform_sphere<<<blocks_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        n, radius, total_mass / static_cast<double>(n), rho0, w[0], w[1], w[2], seed, pos, vel, mass, density);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GSPH_OK : ic_fail(e, "gsph_ic_uniform_sphere");
}

int gsph_ic_plummer(int64_t n, double a, double total_mass, double G, uint64_t seed, float* pos, float* vel,
                    float* mass, void* stream) {
    if (n < 1 || !pos || !vel || !(a > 0)) {
        set_global_error("gsph_ic_plummer: n >= 1, a > 0, pos and vel are required");
        return GSPH_E_INVALID;
    }
    k_plummer<<<blocks_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, a, total_mass, G, seed, pos,
                                                                                      vel, mass);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GSPH_OK : ic_fail(e, "gsph_ic_plummer");
}

// subtract the mass-weighted mean position and velocity (vel may be NULL); scratch is 7 * 256 doubles
int gsph_ic_com_correct(int64_t n, float* pos, float* vel, const float* mass, double* scratch, void* stream) {
    if (n < 1 || !pos || !mass || !scratch) {
        set_global_error("gsph_ic_com_correct: n >= 1, pos, mass and scratch are required");
        return GSPH_E_INVALID;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int parts = 256;
    k_com_partial<<<parts, 256, 0, s>>>(n, pos, vel, mass, scratch);
    k_com_apply<<<blocks_for(n, 256), 256, 0, s>>>(n, pos, vel, scratch, parts, ComTarget{{0, 0, 0}, {0, 0, 0}, 1, 1});
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GSPH_OK : ic_fail(e, "gsph_ic_com_correct");
}

int gsph_ic_com_set(int64_t n, float* pos, float* vel, const float* mass, const double* com, const double* vcom,
                    double* scratch, void* stream) {
    if (n < 1 || !pos || !mass || !scratch || (vcom && !vel)) {
        set_global_error("gsph_ic_com_set: n >= 1, pos, mass and scratch are required (and vel with vcom)");
        return GSPH_E_INVALID;
    }
    ComTarget t{};
    t.set_com = com != nullptr;
    t.set_vcom = vcom != nullptr;
    for (int c = 0; c < 3; ++c) {
        t.com[c] = com ? com[c] : 0.0;
        t.vcom[c] = vcom ? vcom[c] : 0.0;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int parts = 256;
    k_com_partial<<<parts, 256, 0, s>>>(n, pos, vel, mass, scratch);
    k_com_apply<<<blocks_for(n, 256), 256, 0, s>>>(n, pos, vel, scratch, parts, t);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GSPH_OK : ic_fail(e, "gsph_ic_com_set");
}

int gsph_ic_modify(int64_t n, const gsph_ic_op* ops, int32_t nops, const gsph_host_particles* dev, double* desired_com,
                   double* desired_vcom, void* stream) {
    if (n < 1 || !dev || nops < 0 || nops > GSPH_IC_MAX_OPS || (nops > 0 && !ops)) {
        set_global_error("gsph_ic_modify: n >= 1, dev and 0 <= nops <= GSPH_IC_MAX_OPS ops are required");
        return GSPH_E_INVALID;
    }
    IcArrays arr;
    float* const src[11] = {dev->pos, dev->mass, dev->vel, dev->acc, dev->balsara, dev->xvel,
                            dev->density, dev->density_dt, dev->dstress, dev->dstress_dt, dev->maxvsig};
    for (int b = 0; b < 11; ++b) arr.a[b] = src[b];
    IcOps list{};
    list.n = nops;
    double com[3] = {0, 0, 0}, vcom[3] = {0, 0, 0};
    for (int c = 0; c < 3; ++c) {
        com[c] = desired_com ? desired_com[c] : 0.0;
        vcom[c] = desired_vcom ? desired_vcom[c] : 0.0;
    }
    for (int k = 0; k < nops; ++k) {
        gsph_ic_op o = ops[k];
        const bool needs_pos = o.kind == GSPH_IC_MOVE || o.kind == GSPH_IC_ROTATE || o.kind == GSPH_IC_POS_NOISE ||
                               o.kind == GSPH_IC_ANGULAR_VEL;
        const bool needs_vel = o.kind == GSPH_IC_ROTATE || o.kind == GSPH_IC_ANGULAR_VEL ||
                               o.kind == GSPH_IC_LINEAR_VEL || o.kind == GSPH_IC_RANDOM_VEL;
        if (o.kind < GSPH_IC_MOVE || o.kind > GSPH_IC_SET_CONSTANT) {
            set_global_error("gsph_ic_modify: unknown op kind " + std::to_string(o.kind));
            return GSPH_E_INVALID;
        }
        if ((needs_pos && !dev->pos) || (needs_vel && !dev->vel)) {
            set_global_error("gsph_ic_modify: op " + std::to_string(k) + " needs the pos / vel arrays");
            return GSPH_E_INVALID;
        }
        if (o.kind == GSPH_IC_SET_CONSTANT) {
            const uint32_t a = o.attr;
            if (a == 0 || (a & (a - 1)) || a > GSPH_MAXVSIG || !src[__builtin_ctz(a)]) {
                set_global_error("gsph_ic_modify: setConstant needs one attribute bit whose array is given");
                return GSPH_E_INVALID;
            }
        }
        if (o.kind == GSPH_IC_ROTATE) {  // R = c I + (1 - c) a a^T + s [a]x, a the unit axis
            const double ax = o.v[0], ay = o.v[1], az = o.v[2], ang = o.v[3];
            const double l = std::sqrt(ax * ax + ay * ay + az * az);
            if (!(l > 0.0)) {
                set_global_error("gsph_ic_modify: rotate needs a nonzero axis");
                return GSPH_E_INVALID;
            }
            const double u[3] = {ax / l, ay / l, az / l}, c = std::cos(ang), sn = std::sin(ang);
            const double K[9] = {0, -u[2], u[1], u[2], 0, -u[0], -u[1], u[0], 0};
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) o.v[3 * r + q] = (r == q ? c : 0.0) + (1.0 - c) * u[r] * u[q] + sn * K[3 * r + q];
            double y[3], w[3];
            for (int r = 0; r < 3; ++r) {
                y[r] = o.v[3 * r] * com[0] + o.v[3 * r + 1] * com[1] + o.v[3 * r + 2] * com[2];
                w[r] = o.v[3 * r] * vcom[0] + o.v[3 * r + 1] * vcom[1] + o.v[3 * r + 2] * vcom[2];
            }
            for (int r = 0; r < 3; ++r) {
                com[r] = y[r];
                vcom[r] = w[r];
            }
        } else if (o.kind == GSPH_IC_MOVE) {
            for (int c = 0; c < 3; ++c) com[c] += o.v[c];
        } else if (o.kind == GSPH_IC_ANGULAR_VEL) {
            vcom[0] += o.v[1] * com[2] - o.v[2] * com[1];
            vcom[1] += o.v[2] * com[0] - o.v[0] * com[2];
            vcom[2] += o.v[0] * com[1] - o.v[1] * com[0];
        } else if (o.kind == GSPH_IC_LINEAR_VEL) {
            for (int c = 0; c < 3; ++c) vcom[c] += o.v[c];
        }
        list.op[k] = o;
    }
    if (nops > 0) {
        k_ic_modify<<<blocks_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, list, arr);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return ic_fail(e, "gsph_ic_modify");
    }
    for (int c = 0; c < 3; ++c) {
        if (desired_com) desired_com[c] = com[c];
        if (desired_vcom) desired_vcom[c] = vcom[c];
    }
    return GSPH_OK;
}

}  // extern "C"
