/*
 * TEST INFRASTRUCTURE ONLY. Declarations that let GraSPH2's own result writer,
 * src/ResultStorageManager.cu, and its tsv particle source,
 * src/initialConditions/particleSources/TextFile.h, compile unchanged for the host
 * (oracle/ref_io_driver.cpp): the class ResultStorageManager declared with the members that file
 * defines and uses (the reference's declaration, src/ResultStorageManager.h:51-120, pulls in the full
 * particle engine), a ParticleSource base with the members TextFile uses
 * (src/initialConditions/ParticleSource.h:53-88), a particle and host buffer standing in for
 * HostDiscPT (settings/outputSettings.h:26: POSM, VEL, DENSITY, so a particle holds POS, MASS, VEL,
 * DENSITY in that order), and the mpUtils logging / assertion / timestamp helpers they call. Defines
 * the reference headers' include guards so their own #includes resolve to this.
 */
#ifndef GSPH_REF_IO_H
#define GSPH_REF_IO_H
#define GRASPH2_RESULTSTORAGEMANAGER_H
#define GRASPH2_PARTICLEGENERATOR_H

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <limits>
#include <memory>
#include <mutex>
#include <queue>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "settings.h"

/* mpUtils' logging and assertion helpers, as the writer calls them */
struct gsph_null_log {
    template <typename T>
    gsph_null_log& operator<<(const T&) { return *this; }
};
#define logERROR(module) gsph_null_log()
#define logDEBUG(module) gsph_null_log()
#define logINFO(module) gsph_null_log()
#define logFlush()
#define assert_critical(cond, module, msg) { if (!(cond)) throw std::runtime_error(msg); }
inline int cudaGetLastError() { return 0; }
#define assert_cuda(x) (void)(x)
namespace mpu {
/* the simulation's start time in the file name; the checker sets it so that names are reproducible */
inline std::string& gsph_start_time() {
    static std::string s = "2000-01-01_00-00";
    return s;
}
inline std::string timestamp(const char*) { return gsph_start_time(); }
}  // namespace mpu

/* one stored particle: POS, MASS, VEL, DENSITY; doForEachAttribute takes the functor by value, as
 * Particle::doForEachAttribute does (src/particles/Particle.h:108-113) */
struct gsph_disc_particle {
    f3_t pos;
    f1_t mass;
    f3_t vel;
    f1_t density;
    template <typename F>
    void doForEachAttribute(F f) {
        f(pos);
        f(mass);
        f(vel);
        f(density);
    }
};
class HostDiscPT {
public:
    using deviceType = HostDiscPT;
    HostDiscPT() = default;
    explicit HostDiscPT(size_t n) : p(n) {}
    size_t size() const { return p.size(); }
    void pinMemory() {}
    gsph_disc_particle loadParticle(size_t i) const { return p[i]; }
    std::vector<gsph_disc_particle> p;
};

/* the particle-source base: TextFile sets m_numberOfParticles and overrides generateParticle */
template <typename particleType, typename Derived>
class ParticleSource {
public:
    virtual ~ParticleSource() = default;
    size_t getNumParticles() const { return m_numberOfParticles; }
    particleType particle(size_t id) { return generateParticle(id); }

protected:
    size_t m_numberOfParticles{0};

private:
    virtual particleType generateParticle(size_t id) = 0;
};

class ResultStorageManager {
public:
    ResultStorageManager(std::string directory, std::string prefix, int maxJobs);
    ~ResultStorageManager();
    void printTextFile(HostDiscPT& data, f1_t time);

private:
    const std::string m_directory;
    const std::string m_prefix;
    const std::string m_startTime;
    const int m_maxQueue;
    using hdcQueueType = std::pair<std::unique_ptr<HostDiscPT>, f1_t>;
    using ddcQueueType = std::pair<std::unique_ptr<HostDiscPT::deviceType>, f1_t>;
    std::queue<hdcQueueType> m_hostDiskCopy;
    std::queue<ddcQueueType> m_deviceDiskCopy;
    std::mutex m_queueMutex;
    std::mutex m_workerMutex;
    std::condition_variable m_workSignal;
    bool m_terminateWorker;
    std::atomic_int m_numberJobs;
    std::thread m_workerThread;
    void worker();
    void printFile(HostDiscPT& data, f1_t time);
    struct attributePrinter {
    public:
        template <typename T>
        void operator()(T v);
        explicit attributePrinter(std::ostream& s);
        ~attributePrinter();

    private:
        std::ostream& m_stream;
    };
};

#endif
