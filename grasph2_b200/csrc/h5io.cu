// h5io.cu -- HDF5 snapshots through the system's HDF5 library, loaded at run time.
//
// The reference writes HDF5 when it is built with HighFive and libhdf5 (STORE_HDF5, with the
// HDF5_AVAILABLE check of CMakeLists.txt:123-130 and outputSettings.h:30-33): one dataset per stored
// attribute, named as the attribute (POS, MASS, VEL, ..., src/ResultStorageManager.cu:191-227), of
// shape {N, components} and type float; its HDF5File particle source reads such files back
// (src/initialConditions/particleSources/HDF5File.h:38-150). Here the library's presence is checked when
// it is first needed: libhdf5 (1.10 or later, whose identifiers are 64-bit) is opened with dlopen and
// the dozen C functions used are looked up by name, so the product builds and runs without it and
// reports GSPH_E_UNSUPPORTED for HDF5 files when it is absent.
#include <dlfcn.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/grasph2_b200.h"

void set_global_error(const std::string& msg);  // capi.cu

namespace {

using hid_t = int64_t;
using herr_t = int;
using hsize_t = unsigned long long;
constexpr hid_t kP_DEFAULT = 0;      // H5P_DEFAULT
constexpr hid_t kS_ALL = 0;          // H5S_ALL
constexpr unsigned kF_TRUNC = 0x0002u, kF_RDONLY = 0x0000u;

struct H5 {
    void* lib = nullptr;
    bool ok = false;
    std::string why;
    herr_t (*open)();
    herr_t (*libversion)(unsigned*, unsigned*, unsigned*);
    herr_t (*eset_auto)(hid_t, void*, void*);
    hid_t (*fcreate)(const char*, unsigned, hid_t, hid_t);
    hid_t (*fopen)(const char*, unsigned, hid_t);
    herr_t (*fclose)(hid_t);
    hid_t (*screate_simple)(int, const hsize_t*, const hsize_t*);
    herr_t (*sclose)(hid_t);
    int (*sget_ndims)(hid_t);
    int (*sget_dims)(hid_t, hsize_t*, hsize_t*);
    hid_t (*dcreate)(hid_t, const char*, hid_t, hid_t, hid_t, hid_t, hid_t);
    hid_t (*dopen)(hid_t, const char*, hid_t);
    hid_t (*dget_space)(hid_t);
    herr_t (*dwrite)(hid_t, hid_t, hid_t, hid_t, hid_t, const void*);
    herr_t (*dread)(hid_t, hid_t, hid_t, hid_t, hid_t, void*);
    herr_t (*dclose)(hid_t);
    int (*lexists)(hid_t, const char*, hid_t);
    hid_t* native_float;
};

template <typename F>
bool sym(H5& h, F& f, const char* name) {
    f = reinterpret_cast<F>(dlsym(h.lib, name));
    if (!f) h.why = std::string("libhdf5 lacks ") + name;
    return f != nullptr;
}

H5& api() {
    static H5 h;
    static std::once_flag once;
    std::call_once(once, [] {
        for (const char* name : {"libhdf5.so", "libhdf5_serial.so", "libhdf5.so.310", "libhdf5.so.200",
                                 "libhdf5.so.103", "libhdf5_serial.so.103", "libhdf5_serial.so.100"}) {
            h.lib = dlopen(name, RTLD_NOW | RTLD_LOCAL);
            if (h.lib) break;
        }
        if (!h.lib) {
            h.why = "libhdf5 is not installed (no libhdf5.so on the library path)";
            return;
        }
        bool all = sym(h, h.open, "H5open") && sym(h, h.libversion, "H5get_libversion") &&
                   sym(h, h.eset_auto, "H5Eset_auto2") && sym(h, h.fcreate, "H5Fcreate") &&
                   sym(h, h.fopen, "H5Fopen") && sym(h, h.fclose, "H5Fclose") &&
                   sym(h, h.screate_simple, "H5Screate_simple") && sym(h, h.sclose, "H5Sclose") &&
                   sym(h, h.sget_ndims, "H5Sget_simple_extent_ndims") &&
                   sym(h, h.sget_dims, "H5Sget_simple_extent_dims") && sym(h, h.dcreate, "H5Dcreate2") &&
                   sym(h, h.dopen, "H5Dopen2") && sym(h, h.dget_space, "H5Dget_space") &&
                   sym(h, h.dwrite, "H5Dwrite") && sym(h, h.dread, "H5Dread") && sym(h, h.dclose, "H5Dclose") &&
                   sym(h, h.lexists, "H5Lexists") && sym(h, h.native_float, "H5T_NATIVE_FLOAT_g");
        if (!all) return;
        unsigned maj = 0, mnr = 0, rel = 0;
        if (h.open() < 0 || h.libversion(&maj, &mnr, &rel) < 0 || maj < 1 || (maj == 1 && mnr < 10)) {
            h.why = "libhdf5 " + std::to_string(maj) + "." + std::to_string(mnr) + " is older than 1.10";
            return;
        }
        h.eset_auto(0, nullptr, nullptr);  // errors are returned, not printed
        h.ok = true;
    });
    return h;
}

// dataset names: the reference's attribute class names (partice_attributes.h, debugName())
const char* const kNames[11] = {"POS", "MASS", "VEL", "ACC", "BALSARA", "XVEL",
                                "DENSITY", "DENSITY_DT", "DSTRESS", "DSTRESS_DT", "MAXVSIG"};
constexpr int kComps[11] = {3, 1, 3, 3, 1, 3, 1, 1, 9, 9, 1};

float* const* fields(const gsph_host_particles* h, float* (&a)[11]) {
    float* const v[11] = {h->pos, h->mass, h->vel, h->acc, h->balsara, h->xvel,
                          h->density, h->density_dt, h->dstress, h->dstress_dt, h->maxvsig};
    for (int b = 0; b < 11; ++b) a[b] = v[b];
    return a;
}

int h5fail(int code, const std::string& msg) {
    set_global_error(msg);
    return code;
}

}  // namespace

extern "C" {

int gsph_h5_available(void) { return api().ok ? 1 : 0; }

int gsph_h5_write(const char* filename, int64_t n, const gsph_host_particles* h, uint32_t mask) {
    if (!filename || !h || n < 0 || (mask & ~GSPH_ALL_ATTRIBS))
        return h5fail(GSPH_E_INVALID, "gsph_h5_write: filename, particles, n >= 0 and a valid mask are required");
    H5& x = api();
    if (!x.ok) return h5fail(GSPH_E_UNSUPPORTED, "HDF5 output unavailable: " + x.why);
    float* a[11];
    fields(h, a);
    for (int b = 0; b < 11; ++b)
        if ((mask >> b & 1u) && !a[b]) return h5fail(GSPH_E_INVALID, std::string("gsph_h5_write: ") + kNames[b] + " is NULL");
    const hid_t f = x.fcreate(filename, kF_TRUNC, kP_DEFAULT, kP_DEFAULT);
    if (f < 0) return h5fail(GSPH_E_INVALID, std::string("could not create HDF5 file ") + filename);
    int rc = GSPH_OK;
    for (int b = 0; b < 11 && rc == GSPH_OK; ++b) {
        if (!(mask >> b & 1u)) continue;
        const hsize_t dims[2] = {static_cast<hsize_t>(n), static_cast<hsize_t>(kComps[b])};
        const hid_t sp = x.screate_simple(2, dims, nullptr);
        const hid_t ds = sp < 0 ? -1 : x.dcreate(f, kNames[b], *x.native_float, sp, kP_DEFAULT, kP_DEFAULT, kP_DEFAULT);
        if (ds < 0 || (n > 0 && x.dwrite(ds, *x.native_float, kS_ALL, kS_ALL, kP_DEFAULT, a[b]) < 0))
            rc = h5fail(GSPH_E_INVALID, std::string("could not write dataset ") + kNames[b] + " of " + filename);
        if (ds >= 0) x.dclose(ds);
        if (sp >= 0) x.sclose(sp);
    }
    if (x.fclose(f) < 0 && rc == GSPH_OK) rc = h5fail(GSPH_E_INVALID, std::string("could not close ") + filename);
    return rc;
}

int gsph_h5_read(const char* filename, uint32_t mask, gsph_host_particles* out, int64_t cap, int64_t* n) {
    if (!filename || (mask & ~GSPH_ALL_ATTRIBS) || (mask && !out))
        return h5fail(GSPH_E_INVALID, "gsph_h5_read: filename and a valid mask (with out) are required");
    H5& x = api();
    if (!x.ok) return h5fail(GSPH_E_UNSUPPORTED, "HDF5 input unavailable: " + x.why);
    const hid_t f = x.fopen(filename, kF_RDONLY, kP_DEFAULT);
    if (f < 0) return h5fail(GSPH_E_INVALID, std::string("could not open HDF5 file ") + filename);
    float* a[11] = {};
    if (out) fields(out, a);
    int rc = GSPH_OK;
    int64_t count = -1;
    for (int b = 0; b < 11 && rc == GSPH_OK; ++b) {
        if (!(mask >> b & 1u) && !(b == 0 && mask == 0)) continue;
        if (x.lexists(f, kNames[b], kP_DEFAULT) <= 0) {  // the reference requires every attribute it reads
            if (mask >> b & 1u) rc = h5fail(GSPH_E_INVALID, std::string(filename) + " has no dataset " + kNames[b]);
            continue;
        }
        const hid_t ds = x.dopen(f, kNames[b], kP_DEFAULT);
        const hid_t sp = ds < 0 ? -1 : x.dget_space(ds);
        hsize_t dims[2] = {0, 0};
        const int nd = sp < 0 ? -1 : x.sget_ndims(sp);
        if (nd < 1 || nd > 2 || x.sget_dims(sp, dims, nullptr) < 0) {
            rc = h5fail(GSPH_E_INVALID, std::string("unreadable dataset ") + kNames[b]);
        } else {
            const int64_t rows = static_cast<int64_t>(dims[0]);
            const int comps = nd == 2 ? static_cast<int>(dims[1]) : 1;
            if (count >= 0 && rows != count) rc = h5fail(GSPH_E_INVALID, "datasets of different lengths");
            else if (comps != kComps[b]) rc = h5fail(GSPH_E_INVALID, std::string("dataset ") + kNames[b] + " has " +
                                                                    std::to_string(comps) + " components");
            count = rows;
            if (rc == GSPH_OK && (mask >> b & 1u) && rows <= cap && rows > 0 &&
                x.dread(ds, *x.native_float, kS_ALL, kS_ALL, kP_DEFAULT, a[b]) < 0)
                rc = h5fail(GSPH_E_INVALID, std::string("could not read dataset ") + kNames[b]);
        }
        if (sp >= 0) x.sclose(sp);
        if (ds >= 0) x.dclose(ds);
    }
    x.fclose(f);
    if (rc != GSPH_OK) return rc;
    if (n) *n = count < 0 ? 0 : count;
    if (count > cap && mask) return h5fail(GSPH_E_INVALID, "the file holds more particles than cap");
    return GSPH_OK;
}

}  // extern "C"
