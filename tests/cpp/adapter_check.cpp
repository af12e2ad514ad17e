// C++ caller of the library through include/grasph2_b200.hpp: the reference's main-loop shape
// (src/main.cu:228-273) on a small rotating solid sphere, with a tsv snapshot round trip.
// Prints "ADAPTER OK" and exits 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <random>

#include "grasph2_b200.hpp"

int main(int argc, char** argv) {
    const std::string tmp = argc > 1 ? argv[1] : "/tmp";
    gsph_params p;
    gsph_params_reference_defaults(&p);  // settings/settings.h as shipped
    p.H = 0.3;
    p.grav_eps = 0.3;
    p.rho0 = 1.0;
    p.bulk = 10.0;
    p.soundspeed = std::sqrt(10.0);
    p.shear = 5.0;
    const int n = 2000;
    gsph::HostParticleBuffer hpb(n);
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    for (int i = 0; i < n; ++i) {
        float x, y, z;
        do { x = u(rng); y = u(rng); z = u(rng); } while (x * x + y * y + z * z > 1.f);
        hpb.pos[3 * i] = x; hpb.pos[3 * i + 1] = y; hpb.pos[3 * i + 2] = z;
        hpb.vel[3 * i] = -0.3f * y; hpb.vel[3 * i + 1] = 0.3f * x;
        hpb.mass[i] = 1.0f / n;
        hpb.density[i] = 1.0f;
    }
    gsph::DeviceParticleBuffer pb(p, n);
    pb = hpb;
    double t = 0.0;
    for (int s = 0; s < 5; ++s) {
        gsph::computeDerivatives(pb);
        gsph::integrate(pb, true);
        t += gsph::getCurrentTimestep(pb);
    }
    gsph::HostParticleBuffer out;
    pb.download(out);
    double fx = 0, fy = 0, fz = 0, fa = 0;
    for (int i = 0; i < n; ++i) {
        fx += out.mass[i] * out.acc[3 * i]; fy += out.mass[i] * out.acc[3 * i + 1]; fz += out.mass[i] * out.acc[3 * i + 2];
        fa += out.mass[i] * (std::fabs(out.acc[3 * i]) + std::fabs(out.acc[3 * i + 1]) + std::fabs(out.acc[3 * i + 2]));
    }
    if (!(std::fabs(fx) + std::fabs(fy) + std::fabs(fz) < 1e-4 * fa) || !(t > 0)) {
        std::printf("momentum check failed: %g %g %g vs %g, t=%g\n", fx, fy, fz, fa, t);
        return 1;
    }
    const std::string fn = gsph::snapshotFileName(tmp + "/", "graSPH2_", "test", static_cast<float>(t));
    gsph::printTextFile(out, fn);
    gsph::HostParticleBuffer back = gsph::readTextFile(fn);
    if (back.size() != out.size()) { std::printf("tsv size mismatch\n"); return 1; }
    for (size_t i = 0; i < 3 * back.size(); ++i)
        if (std::fabs(back.pos[i] - out.pos[i]) > 1e-6f * (1.f + std::fabs(out.pos[i]))) {
            std::printf("tsv value mismatch at %zu\n", i);
            return 1;
        }
    try {
        gsph::integrate(pb, true);
        gsph_host_particles bad{};
        gsph::check(gsph_upload(pb.get(), GSPH_POS, &bad, nullptr), pb.get());
        std::printf("expected an error\n");
        return 1;
    } catch (const gsph::Error& e) {
        if (e.code() != GSPH_E_INVALID) return 1;
    }
    {  // the same physics as an ensemble of three simulations of uneven sizes
        gsph_params q = p;
        q.flags &= ~(GSPH_VARIABLE_TIMESTEP | GSPH_BALSARA_SWITCH);
        std::vector<int64_t> counts = {300, 77, 512};
        gsph::Ensemble ens(q, counts);
        gsph::HostParticleBuffer h(static_cast<size_t>(ens.size()));
        for (size_t i = 0; i < h.size(); ++i) {
            const double u = std::fmod(0.6180339887 * (i + 1), 1.0), w = std::fmod(0.7548776662 * (i + 1), 1.0),
                         z = std::fmod(0.5698402910 * (i + 1), 1.0);
            h.pos[3 * i] = static_cast<float>(u - 0.5);
            h.pos[3 * i + 1] = static_cast<float>(w - 0.5);
            h.pos[3 * i + 2] = static_cast<float>(z - 0.5);
            h.mass[i] = 1.0f / 300.0f;
            h.density[i] = static_cast<float>(q.rho0);
        }
        ens.upload(h, GSPH_POS | GSPH_MASS | GSPH_VEL | GSPH_DENSITY | GSPH_DSTRESS);
        ens.autotune(1);
        ens.step(3);
        ens.download(h);
        const std::vector<gsph_diag> d = ens.diagnostics();
        if (d.size() != counts.size() || !(d[2].mass > 0)) {
            std::printf("ensemble check failed\n");
            return 1;
        }
    }
    {  // asynchronous snapshots while stepping
        gsph::SnapshotWriter w(pb, gsph::kDefaultStoredAttributes, 2);
        for (int k = 0; k < 3; ++k) {
            gsph::integrate(pb, true);
            gsph::computeDerivatives(pb);
            w.write(gsph::snapshotFileName(tmp + "/", "async_", "test", static_cast<float>(k)));
        }
        if (w.flush() != 3) {
            std::printf("writer count mismatch\n");
            return 1;
        }
        gsph::HostParticleBuffer last = gsph::readTextFile(gsph::snapshotFileName(tmp + "/", "async_", "test", 2.0f));
        if (last.size() != out.size()) {
            std::printf("async snapshot size mismatch\n");
            return 1;
        }
    }
    if (argc > 2) {  // the learned surrogate from a model file: one judged window, then a save/load round trip
        gsph_params q = p;
        q.flags &= ~(GSPH_VARIABLE_TIMESTEP | GSPH_BALSARA_SWITCH);
        gsph::DeviceParticleBuffer sb(q, n);
        sb = hpb;
        gsph::Surrogate sur(argv[2]);
        sur.energyCorrection(true);
        const std::vector<gsph_surrogate_window> w = sur.advance(sb, 1, 2);
        if (w.size() != 1 || !(w[0].pos_error >= 0) || !(w[0].energy_error >= 0)) {
            std::printf("surrogate window failed\n");
            return 1;
        }
        sur.save(tmp + "/model.gsur");
        gsph::Surrogate back2(tmp + "/model.gsur");
        if (back2.substeps() != sur.substeps()) {
            std::printf("surrogate file round trip failed\n");
            return 1;
        }
    }
    {  // per-particle host access with the reference's names
        gsph::Particle q = out.loadParticle(5);
        q.pos = q.pos + gsph::f3_t{1.0f, 0.0f, 0.0f};
        q.dstress(0, 1) = 0.25f;
        out.storeParticle(5, q, GSPH_POS | GSPH_DSTRESS);
        if (out.pos[15] != q.pos.x || out.dstress[9 * 5 + 1] != 0.25f) {
            std::printf("particle access mismatch\n");
            return 1;
        }
    }
    std::printf("ADAPTER OK t=%.6f file=%s\n", t, fn.c_str());
    return 0;
}
