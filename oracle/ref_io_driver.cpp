/*
 * ref_io_driver.cpp -- TEST INFRASTRUCTURE ONLY. GraSPH2's own tsv snapshot writer,
 * ResultStorageManager::printTextFile and its attributePrinter (src/ResultStorageManager.cu:102-186),
 * and its tsv particle source ps::TextFile (src/initialConditions/particleSources/TextFile.h:43-170),
 * compiled unchanged for the host against oracle/ref_shim/ref_io.h, so the tests can compare the
 * library's snapshot files with the reference's byte for byte and its reader with the reference's
 * value for value. Built by oracle/build_ref.py into oracle/_ref/libref_io.so.
 */
#include <algorithm>
#include <cctype>
#include <cstring>

#include "ref_io.h"
#include "ResultStorageManager.cu"
#include "initialConditions/particleSources/TextFile.h"

extern "C" {

/* Write n particles (host layout: pos[3n], mass[n], vel[3n], density[n]) at simulation time `time`
 * through the reference's printTextFile into directory `dir` (with its trailing '/') with file-name
 * prefix `prefix` and start-time stamp `start_time`. 0 on success. */
int refio_print_text(const char* dir, const char* prefix, const char* start_time, int64_t n, const float* pos,
                     const float* mass, const float* vel, const float* density, double time) {
    try {
        mpu::gsph_start_time() = start_time;
        HostDiscPT data(static_cast<size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            gsph_disc_particle& q = data.p[static_cast<size_t>(i)];
            q.pos = f3_t{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
            q.mass = mass[i];
            q.vel = f3_t{vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
            q.density = density[i];
        }
        ResultStorageManager rsm(dir, prefix, 2);
        rsm.printTextFile(data, static_cast<f1_t>(time));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

/* Read a tsv file through the reference's TextFile source (POS, MASS, VEL, DENSITY per line):
 * n_out = the number of non-blank lines; the arrays (capacity `cap` particles) receive the values. */
int refio_read_text(const char* filename, int64_t cap, int64_t* n_out, float* pos, float* mass, float* vel,
                    float* density) {
    try {
        ps::TextFile<gsph_disc_particle> src(filename);
        const int64_t n = static_cast<int64_t>(src.getNumParticles());
        if (n_out) *n_out = n;
        for (int64_t i = 0; i < n && i < cap; ++i) {
            const gsph_disc_particle q = src.particle(static_cast<size_t>(i));
            pos[3 * i] = q.pos.x; pos[3 * i + 1] = q.pos.y; pos[3 * i + 2] = q.pos.z;
            mass[i] = q.mass;
            vel[3 * i] = q.vel.x; vel[3 * i + 1] = q.vel.y; vel[3 * i + 2] = q.vel.z;
            density[i] = q.density;
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
