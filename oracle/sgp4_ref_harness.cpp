// Test-only harness: the SGP4 propagator the reference links
// (mizuba/detail/sgp4/SGP4.{h,cpp}, Vallado's public C++ code), compiled in
// place from the reference tree by oracle/build.py into
// oracle/_ref/libsgp4_ref.so.  It pins this repository's own SGP4
// restatement and GPU polyjectory production the way mizuba's own tests pin
// make_sgp4_polyjectory against the sgp4 Python module (which wraps the same
// C++ code): mizuba/test/test_make_sgp4_polyjectory.py:32-67.
//
// The set-up is the one make_sgp4_polyjectory uses (make_sgp4_polyjectory.cpp:
// 719-745): WGS72 constants, the 'a' operation mode, the epoch as days from
// 1950 Jan 0.0 (UTC Julian date - 2433281.5), ndot = nddot = 0.
#include <cstdint>

#include "SGP4.h"

extern "C" {

// Propagates n_gpes element sets to n_times times (minutes since each
// element set's epoch).  out[g][t] = {x, y, z, vx, vy, vz} in km and km/s;
// err[g][t] = the propagator's error code (0 = success; the set-up's error
// code fills every time of an element set that fails to initialise).
void mzr_sgp4(const double *epoch_1950, const double *n0, const double *e0, const double *i0, const double *node0,
              const double *omega0, const double *m0, const double *bstar, std::uint64_t n_gpes,
              const double *tsince, std::uint64_t n_times, double *out, int *err)
{
    for (std::uint64_t g = 0; g < n_gpes; ++g) {
        elsetrec rec{};
        SGP4Funcs::sgp4init(wgs72, 'a', "", epoch_1950[g], bstar[g], 0., 0., e0[g], omega0[g], i0[g], m0[g], n0[g],
                            node0[g], rec);
        const int e_init = rec.error;
        for (std::uint64_t t = 0; t < n_times; ++t) {
            double *o = out + (g * n_times + t) * 6;
            if (e_init != 0) {
                err[g * n_times + t] = e_init;
                continue;
            }
            SGP4Funcs::sgp4(rec, tsince[t], o, o + 3);
            err[g * n_times + t] = rec.error;
        }
    }
}

// Whether the set-up classified the element set as deep space (period of at
// least 225 minutes: SDP4).
int mzr_sgp4_is_deep_space(double epoch_1950, double n0, double e0, double i0, double node0, double omega0, double m0,
                           double bstar)
{
    elsetrec rec{};
    SGP4Funcs::sgp4init(wgs72, 'a', "", epoch_1950, bstar, 0., 0., e0, omega0, i0, m0, n0, node0, rec);
    return rec.method == 'd';
}
}

extern "C" {

// A set-up element set for repeated propagation (the oracle's SGP4
// polyjectory production drives it): NULL and *err != 0 when the set-up
// fails; *deep = 1 for the deep-space branch.
void *mzr_sgp4_new(double epoch_1950, double n0, double e0, double i0, double node0, double omega0, double m0,
                   double bstar, int *err, int *deep)
{
    auto *rec = new elsetrec{};
    SGP4Funcs::sgp4init(wgs72, 'a', "", epoch_1950, bstar, 0., 0., e0, omega0, i0, m0, n0, node0, *rec);
    *err = rec->error;
    *deep = rec->method == 'd';
    if (*err != 0) {
        delete rec;
        return nullptr;
    }
    return rec;
}

int mzr_sgp4_at(void *h, double tsince, double *r, double *v)
{
    auto *rec = static_cast<elsetrec *>(h);
    SGP4Funcs::sgp4(*rec, tsince, r, v);
    return rec->error;
}

void mzr_sgp4_delete(void *h) { delete static_cast<elsetrec *>(h); }
}
