/*
 * TEST INFRASTRUCTURE ONLY. CUDA stand-in for GraSPH2's particle engine (src/particles/), whose real
 * headers depend on mpUtils' template-metaprogramming library and on OpenGL interop
 * (Device_base.h includes cuda_gl_interop.h). It supplies the types that the reference's own device
 * launchers and kernels use -- Particle<...>, the attribute tags, merge_particles_t, load_helper,
 * SharedParticles with the SHARED_* shared-memory bases, DeviceParticleBuffer and its device
 * reference -- and then includes the reference's src/particles/algorithms.h itself, so the tile
 * kernel do_for_each_pair_fast_impl and the per-particle kernel do_for_each_impl
 * (algorithms.h:164-177, :270-309) are GraSPH2's own code.
 *
 * Memory layout follows the reference's device buffers (settings/settings.h:184 with
 * particle_buffer_impl.h): POSM, VEL, ACC, XVEL as f4_t; BALSARA, DENSITY, DENSITY_DT, MAXVSIG as
 * f1_t; DSTRESS, DSTRESS_DT as m3_t. A Particle<A...> is one flat record of every attribute that
 * remembers its list A..., so loads and stores touch exactly the listed attributes, as the
 * reference's do.
 */
#ifndef MPUTILS_PARTICLES_H
#define MPUTILS_PARTICLES_H

#include <cstddef>
#include <cstdint>
#include <tuple>
#include <type_traits>

#include "types.h"

struct particle_attrib {};

#define GSPH_SHIM_ATTR(NAME)          \
    struct NAME : particle_attrib {}; \
    struct r##NAME : particle_attrib {};
GSPH_SHIM_ATTR(POS)
GSPH_SHIM_ATTR(MASS)
GSPH_SHIM_ATTR(VEL)
GSPH_SHIM_ATTR(ACC)
GSPH_SHIM_ATTR(BALSARA)
GSPH_SHIM_ATTR(XVEL)
GSPH_SHIM_ATTR(DENSITY)
GSPH_SHIM_ATTR(DENSITY_DT)
GSPH_SHIM_ATTR(DSTRESS)
GSPH_SHIM_ATTR(DSTRESS_DT)
GSPH_SHIM_ATTR(MAXVSIG)
#undef GSPH_SHIM_ATTR

/* every attribute of particle_bases (src/particles/partice_attributes.h:91-106) */
struct gsph_particle_record {
    f3_t pos{0, 0, 0};
    f1_t mass{0};
    f3_t vel{0, 0, 0};
    f3_t acc{0, 0, 0};
    f1_t balsara{0};
    f3_t xvel{0, 0, 0};
    f1_t density{0};
    f1_t density_dt{0};
    m3_t dstress{0};
    m3_t dstress_dt{0};
    f1_t max_vsig{0};
};

template <typename... A>
struct Particle : gsph_particle_record {
    using attributes = std::tuple<A...>;
    __host__ __device__ Particle() {}
    template <typename... B>
    __host__ __device__ Particle(const Particle<B...>& o) : gsph_particle_record(static_cast<const gsph_particle_record&>(o)) {}
};

/* the two reference-binding forms used by src/integration.h:24 and :33 */
template <>
struct Particle<DENSITY, rDSTRESS> {
    f1_t density;
    m3_t& dstress;
    template <typename... B>
    __host__ __device__ Particle(Particle<B...>& o) : density(o.density), dstress(o.dstress) {}
};
template <>
struct Particle<rPOS, rVEL> {
    f3_t& pos;
    f3_t& vel;
    template <typename... B>
    __host__ __device__ Particle(Particle<B...>& o) : pos(o.pos), vel(o.vel) {}
};

template <typename... P>
struct gsph_merge;
template <typename... A>
struct gsph_merge<Particle<A...>> {
    using type = Particle<A...>;
};
template <typename... A, typename... B, typename... R>
struct gsph_merge<Particle<A...>, Particle<B...>, R...> {
    using type = typename gsph_merge<Particle<A..., B...>, R...>::type;
};
template <typename... P>
using merge_particles_t = typename gsph_merge<P...>::type;

/* ---- device storage of one attribute (the reference's DEVICE_REFERENCE bases) ---------------- */
struct gsph_dev_arrays {
    f4_t* posm;
    f4_t* vel;
    f4_t* acc;
    f4_t* xvel;
    f1_t* balsara;
    f1_t* density;
    f1_t* density_dt;
    f1_t* maxvsig;
    m3_t* dstress;
    m3_t* dstress_dt;
};

template <typename Tag>
struct gsph_attr;
#define GSPH_ATTR(TAG, LOAD, STORE)                                                                        \
    template <>                                                                                              \
    struct gsph_attr<TAG> {                                                                                  \
        __host__ __device__ static void load(const gsph_dev_arrays& a, size_t i, gsph_particle_record& r) { \
            LOAD;                                                                                            \
        }                                                                                                    \
        __host__ __device__ static void store(const gsph_dev_arrays& a, size_t i, const gsph_particle_record& r) { \
            STORE;                                                                                           \
        }                                                                                                    \
    };
/* POS and MASS share the POSM float4 (posm_impl, particle_buffer_impl.h) */
GSPH_ATTR(POS, (r.pos = f3_t{a.posm[i].x, a.posm[i].y, a.posm[i].z}),
          (a.posm[i].x = r.pos.x, a.posm[i].y = r.pos.y, a.posm[i].z = r.pos.z))
GSPH_ATTR(MASS, (r.mass = a.posm[i].w), (a.posm[i].w = r.mass))
GSPH_ATTR(VEL, (r.vel = f3_t{a.vel[i].x, a.vel[i].y, a.vel[i].z}), (a.vel[i] = f4_t{r.vel.x, r.vel.y, r.vel.z, 0}))
GSPH_ATTR(ACC, (r.acc = f3_t{a.acc[i].x, a.acc[i].y, a.acc[i].z}), (a.acc[i] = f4_t{r.acc.x, r.acc.y, r.acc.z, 0}))
GSPH_ATTR(XVEL, (r.xvel = f3_t{a.xvel[i].x, a.xvel[i].y, a.xvel[i].z}),
          (a.xvel[i] = f4_t{r.xvel.x, r.xvel.y, r.xvel.z, 0}))
GSPH_ATTR(BALSARA, (r.balsara = a.balsara[i]), (a.balsara[i] = r.balsara))
GSPH_ATTR(DENSITY, (r.density = a.density[i]), (a.density[i] = r.density))
GSPH_ATTR(DENSITY_DT, (r.density_dt = a.density_dt[i]), (a.density_dt[i] = r.density_dt))
GSPH_ATTR(MAXVSIG, (r.max_vsig = a.maxvsig[i]), (a.maxvsig[i] = r.max_vsig))
GSPH_ATTR(DSTRESS, (r.dstress = a.dstress[i]), (a.dstress[i] = r.dstress))
GSPH_ATTR(DSTRESS_DT, (r.dstress_dt = a.dstress_dt[i]), (a.dstress_dt[i] = r.dstress_dt))
#undef GSPH_ATTR

/* the non-owning view passed by value to kernels (DeviceParticleReference,
 * src/particles/DeviceParticleBuffer.h:218-221) */
template <typename... Args>
class DeviceParticleReference {
public:
    gsph_dev_arrays a;
    size_t n;
    __host__ __device__ size_t size() const { return n; }
    template <typename... A>
    __device__ Particle<A...> loadParticle(size_t i) const {
        Particle<A...> p{};
        int t[] = {0, (gsph_attr<A>::load(a, i, p), 1)...};
        (void)t;
        return p;
    }
    template <typename... A>
    __device__ void storeParticle(size_t i, const Particle<A...>& p) const {
        int t[] = {0, (gsph_attr<A>::store(a, i, p), 1)...};
        (void)t;
    }
};

/* the owning device buffer (DeviceParticleBuffer, src/particles/Device_base.h:126-145): one
 * cudaMalloc array per attribute */
template <typename... Args>
class DeviceParticleBuffer {
public:
    DeviceParticleReference<> ref{};
    explicit DeviceParticleBuffer(size_t n) {
        ref.n = n;
        auto al = [&](auto*& p, size_t bytes) { assert_cuda(cudaMalloc(reinterpret_cast<void**>(&p), bytes ? bytes : 16)); };
        al(ref.a.posm, n * sizeof(f4_t));
        al(ref.a.vel, n * sizeof(f4_t));
        al(ref.a.acc, n * sizeof(f4_t));
        al(ref.a.xvel, n * sizeof(f4_t));
        al(ref.a.balsara, n * sizeof(f1_t));
        al(ref.a.density, n * sizeof(f1_t));
        al(ref.a.density_dt, n * sizeof(f1_t));
        al(ref.a.maxvsig, n * sizeof(f1_t));
        al(ref.a.dstress, n * sizeof(m3_t));
        al(ref.a.dstress_dt, n * sizeof(m3_t));
    }
    ~DeviceParticleBuffer() {
        void* ps[] = {ref.a.posm, ref.a.vel, ref.a.acc, ref.a.xvel, ref.a.balsara, ref.a.density, ref.a.density_dt,
                      ref.a.maxvsig, ref.a.dstress, ref.a.dstress_dt};
        for (void* p : ps)
            if (p) cudaFree(p);
    }
    DeviceParticleBuffer(const DeviceParticleBuffer&) = delete;
    DeviceParticleBuffer& operator=(const DeviceParticleBuffer&) = delete;
    size_t size() const { return ref.n; }
    DeviceParticleReference<> getDeviceReference() const { return ref; }
};
template <typename... Args>
class HostParticleBuffer;

template <typename P, typename buffer>
struct load_helper;
template <typename... A, typename buffer>
struct load_helper<Particle<A...>, buffer> {
    __host__ __device__ static auto load(const buffer& pb, size_t i) { return pb.template loadParticle<A...>(i); }
};

/* ---- shared memory (SHARED_BASE, src/particles/Shared_base.h:39-64) ------------------------------ */
template <size_t n, typename T, typename PT, typename IO>
class gsph_shared_base {
public:
    using type = T;
    using particleType = PT;
    __device__ gsph_shared_base() {
        __shared__ static T mem[n == 0 ? 1 : n];
        m_data = mem;
    }
    __device__ void load_into(size_t id, gsph_particle_record& p) const { IO::load(m_data[id], p); }
    __device__ void store_from(size_t id, const gsph_particle_record& p) { IO::store(m_data[id], p); }

private:
    T* m_data;
};
struct gsph_io_posm {
    __device__ static void load(const f4_t& v, gsph_particle_record& p) {
        p.pos = f3_t{v.x, v.y, v.z};
        p.mass = v.w;
    }
    __device__ static void store(f4_t& v, const gsph_particle_record& p) { v = f4_t{p.pos.x, p.pos.y, p.pos.z, p.mass}; }
};
struct gsph_io_vel {
    __device__ static void load(const f4_t& v, gsph_particle_record& p) { p.vel = f3_t{v.x, v.y, v.z}; }
    __device__ static void store(f4_t& v, const gsph_particle_record& p) { v = f4_t{p.vel.x, p.vel.y, p.vel.z, 0}; }
};
struct gsph_io_balsara {
    __device__ static void load(const f1_t& v, gsph_particle_record& p) { p.balsara = v; }
    __device__ static void store(f1_t& v, const gsph_particle_record& p) { v = p.balsara; }
};
struct gsph_io_density {
    __device__ static void load(const f1_t& v, gsph_particle_record& p) { p.density = v; }
    __device__ static void store(f1_t& v, const gsph_particle_record& p) { v = p.density; }
};
struct gsph_io_dstress {
    __device__ static void load(const m3_t& v, gsph_particle_record& p) { p.dstress = v; }
    __device__ static void store(m3_t& v, const gsph_particle_record& p) { v = p.dstress; }
};
template <size_t n>
using SHARED_POSM = gsph_shared_base<n, f4_t, Particle<POS, MASS>, gsph_io_posm>;
template <size_t n>
using SHARED_VEL = gsph_shared_base<n, f4_t, Particle<VEL>, gsph_io_vel>;
template <size_t n>
using SHARED_BALSARA = gsph_shared_base<n, f1_t, Particle<BALSARA>, gsph_io_balsara>;
template <size_t n>
using SHARED_DENSITY = gsph_shared_base<n, f1_t, Particle<DENSITY>, gsph_io_density>;
template <size_t n>
using SHARED_DSTRESS = gsph_shared_base<n, m3_t, Particle<DSTRESS>, gsph_io_dstress>;

/* SharedParticles (src/particles/SharedParticles.h:36-79): one shared-memory base per attribute group */
template <size_t n, template <size_t> class... TArgs>
class SharedParticles : public TArgs<n>... {
public:
    using particleType = merge_particles_t<typename TArgs<n>::particleType...>;
    __device__ SharedParticles() : TArgs<n>()... {}
    SharedParticles(const SharedParticles&) = delete;
    SharedParticles& operator=(const SharedParticles&) = delete;
    template <typename... A>
    __device__ Particle<A...> loadParticle(size_t id) const {
        Particle<A...> p{};
        int t[] = {0, (TArgs<n>::load_into(id, p), 1)...};
        (void)t;
        return p;
    }
    template <typename... A>
    __device__ void storeParticle(size_t id, const Particle<A...>& p) {
        int t[] = {0, (TArgs<n>::store_from(id, p), 1)...};
        (void)t;
    }
    __device__ size_t size() { return n; }
};

/* the reference's own launchers and kernels; its other particle headers are replaced by the above */
#define GRASPH2_PARTICE_ATTRIBUTES_H
#define GRASPH2_PARTICLE_BUFFER_IMPL_H
#define MPUTILS_PARTICLE_H
#define GRASPH2_HOSTPARTICLEBUFFER_H
#define GRASPH2_DEVICEPARTICLEBUFFER_H
#define GRASPH2_DEVICEPARTICLEREFERENCE_H
#define MPUTILS_SHAREDPARTICLES_H
#include <particles/algorithms.h>

#endif
