// ics.cu -- initial conditions generated on the device: uniform spheres, Plummer spheres and the
// centre-of-mass correction (the reference's particle sources, src/initialConditions/particleSources/
// UniformSphere.cu and PlummerSphere.cu, and InitGenerator.h:113-152), so large inputs need no host
// generation or transfer.
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

__global__ void k_com_apply(int64_t n, float* pos, float* vel, const double* part, int nparts) {
    __shared__ double c[7];
    if (threadIdx.x < 7) {
        double t = 0.0;
        for (int b = 0; b < nparts; ++b) t += part[b * 7 + threadIdx.x];
        c[threadIdx.x] = t;
    }
    __syncthreads();
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n || c[0] == 0.0) return;
    for (int k = 0; k < 3; ++k) {
        pos[3 * i + k] = static_cast<float>(pos[3 * i + k] - c[1 + k] / c[0]);
        if (vel) vel[3 * i + k] = static_cast<float>(vel[3 * i + k] - c[4 + k] / c[0]);
    }
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
    k_com_apply<<<blocks_for(n, 256), 256, 0, s>>>(n, pos, vel, scratch, parts);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GSPH_OK : ic_fail(e, "gsph_ic_com_correct");
}

}  // extern "C"
