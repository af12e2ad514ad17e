/*
 * TEST INFRASTRUCTURE ONLY. Minimal stand-in for GraSPH2's particle engine (src/particles/), which
 * depends on mpUtils' template-metaprogramming library. It gives the reference's job structs the
 * names they use -- Particle<...>, the attribute tags, merge_particles_t, SharedParticles -- with
 * one flat record holding every attribute. A Particle<A...> remembers its attribute list A...,
 * so the parity driver loads and stores exactly the attributes the reference would
 * (load_type / pj_type / store_type), and value-initialises the rest, as the reference's
 * load_helper does (src/particles/algorithms.h:171-175, :241-254).
 *
 * It defines the include guard of src/particles/Particles.h, so that the reference's own
 * `#include "particles/Particles.h"` in the job headers resolves to this file's content.
 */
#ifndef MPUTILS_PARTICLES_H
#define MPUTILS_PARTICLES_H

#include <tuple>
#include <cstddef>
#include <cstdint>
#include "types.h"

struct particle_attrib {};

#define GSPH_SHIM_ATTR(NAME)                 \
    struct NAME : particle_attrib {};        \
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

struct SHARED_POSM {};
struct SHARED_VEL {};
struct SHARED_BALSARA {};
struct SHARED_DENSITY {};
struct SHARED_DSTRESS {};
template <size_t n, typename... A>
struct SharedParticles {};
template <typename... A>
class DeviceParticleBuffer;

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
    Particle() = default;
    template <typename... B>
    Particle(const Particle<B...>& o) : gsph_particle_record(static_cast<const gsph_particle_record&>(o)) {}
};

/* the two reference-binding forms used by src/integration.h:24 and :33 */
template <>
struct Particle<DENSITY, rDSTRESS> {
    f1_t density;
    m3_t& dstress;
    template <typename... B>
    Particle(Particle<B...>& o) : density(o.density), dstress(o.dstress) {}
};
template <>
struct Particle<rPOS, rVEL> {
    f3_t& pos;
    f3_t& vel;
    template <typename... B>
    Particle(Particle<B...>& o) : pos(o.pos), vel(o.vel) {}
};

template <typename A, typename B>
struct gsph_merge;
template <typename... A, typename... B>
struct gsph_merge<Particle<A...>, Particle<B...>> {
    using type = Particle<A..., B...>;
};
template <typename A, typename B>
using merge_particles_t = typename gsph_merge<A, B>::type;

#endif
