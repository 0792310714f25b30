// Pieces of the SGP4 polyjectory production shared by the GPU kernel and its
// host driver: double-length time arithmetic, UTC -> TAI Julian dates, and
// the Taylor step-size rule that sets the interpolation steps.
//
// The reference (mizuba/make_sgp4_polyjectory.cpp:764-913) chooses each
// interpolation step as the step an adaptive Taylor integrator of Keplerian
// motion (heyoka, tolerance 1e-14, positions in km, velocities in km/s, time
// in s, mu = 6.6743e-11 * 1e-9 * 5.9722e24) would take from the SGP4 state
// at the step's start.  heyoka is not part of the reference tree; its rule
// is the published one restated below: order p = ceil(-ln(tol) / 2 + 1) = 18
// and the Jorba-Zou step size (A. Jorba and M. Zou, Experimental Mathematics
// 14(1), 2005) with the safety factor of F. Biscani and D. Izzo, MNRAS 504
// (2021): h = rho_m / e^2 * exp(-0.7 / (p - 1)), rho_m = min over j in
// {p - 1, p} of (s / |x^[j]|)^(1/j), where x^[j] are the normalised Taylor
// coefficients of the state (infinity norm) and s = max(1, |x|) selects the
// relative or absolute regime.  The Taylor coefficients of the two-body
// problem come from the automatic-differentiation recurrences of r^2 and
// (r^2)^(-3/2).
#pragma once

#include <cmath>
#include <cstdint>

#include "sgp4.cuh"

namespace mzb
{
namespace sgp4pj
{

constexpr int ORDER = 18; // ceil(-ln(1e-14) / 2 + 1)
constexpr int OP1 = ORDER + 1;
constexpr double MU_KEPLER = 6.6743e-11 * 1e-9 * 5.9722e24; // km^3 / s^2, as the reference builds its dynamics

// Double-length numbers (hi + lo, |lo| <= ulp(hi) / 2), with the error-free
// sums of D. E. Knuth (TAOCP vol. 2, 4.2.2) and T. J. Dekker (Numer. Math.
// 18, 1971).
struct dfl {
    double hi, lo;
};

MZB_HD inline dfl two_sum(double a, double b)
{
    const double s = a + b;
    const double bb = s - a;
    return dfl{s, (a - (s - bb)) + (b - bb)};
}

MZB_HD inline dfl fast_two_sum(double a, double b)
{
    const double s = a + b;
    return dfl{s, b - (s - a)};
}

MZB_HD inline dfl dfl_norm(double hi, double lo) { return two_sum(hi, lo); }

MZB_HD inline dfl dfl_add(dfl a, dfl b)
{
    dfl s = two_sum(a.hi, b.hi);
    const dfl t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}

MZB_HD inline dfl dfl_neg(dfl a) { return dfl{-a.hi, -a.lo}; }
MZB_HD inline dfl dfl_sub(dfl a, dfl b) { return dfl_add(a, dfl_neg(b)); }
MZB_HD inline dfl dfl_add(dfl a, double b) { return dfl_add(a, dfl{b, 0.0}); }
MZB_HD inline bool dfl_lt(dfl a, dfl b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
MZB_HD inline bool dfl_le(dfl a, dfl b) { return !dfl_lt(b, a); }

// Normalised Taylor coefficients of Keplerian motion from the state
// (r [km], v [km/s]) up to ORDER, and the step size [s] of the rule above.
MZB_HD MZB_OUTLINE inline double kepler_step(const double r[3], const double v[3])
{
    double X[3][OP1 + 1], V[3][OP1 + 1], U[OP1], W[OP1];
    for (int i = 0; i < 3; ++i) {
        X[i][0] = r[i];
        V[i][0] = v[i];
    }
    const double alpha = -1.5;
    for (int k = 0; k < ORDER; ++k) {
        // U = x.x and W = U^alpha, order k.
        double u = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j <= k; ++j) u += X[i][j] * X[i][k - j];
        U[k] = u;
        if (k == 0) {
            W[0] = std::pow(U[0], alpha);
        } else {
            double w = 0.0;
            for (int j = 0; j < k; ++j) w += (alpha * double(k - j) - double(j)) * U[k - j] * W[j];
            W[k] = w / (double(k) * U[0]);
        }
        // x' = v, v' = -mu x W.
        for (int i = 0; i < 3; ++i) {
            double xw = 0.0;
            for (int j = 0; j <= k; ++j) xw += X[i][j] * W[k - j];
            X[i][k + 1] = V[i][k] / double(k + 1);
            V[i][k + 1] = -MU_KEPLER * xw / double(k + 1);
        }
    }
    double s = 0.0, np = 0.0, npm1 = 0.0;
    for (int i = 0; i < 3; ++i) {
        s = std::fmax(s, std::fmax(std::fabs(X[i][0]), std::fabs(V[i][0])));
        np = std::fmax(np, std::fmax(std::fabs(X[i][ORDER]), std::fabs(V[i][ORDER])));
        npm1 = std::fmax(npm1, std::fmax(std::fabs(X[i][ORDER - 1]), std::fabs(V[i][ORDER - 1])));
    }
    const double scale = s > 1.0 ? s : 1.0;
    const double rho_p = std::pow(scale / np, 1.0 / double(ORDER));
    const double rho_pm1 = std::pow(scale / npm1, 1.0 / double(ORDER - 1));
    const double rho_m = std::fmin(rho_p, rho_pm1);
    const double e = 2.718281828459045235360287471352662;
    return rho_m / (e * e) * std::exp(-0.7 / double(ORDER - 1));
}

// One interpolation job: one element set over [begin, end) (TAI Julian
// dates), the satellite's index and the job's place in the satellite's list.
struct job {
    double n0, e0, i0, node0, omega0, m0, bstar;
    double epoch1950; // the set-up's epoch: UTC Julian date - 2433281.5
    dfl epoch_tai, begin_tai, end_tai;
    uint32_t sat, k;
};

// Status codes of make_sgp4_polyjectory (the reference's sgp4_pj_status,
// mizuba/_sgp4_polyjectory.py): 1-6 from the propagator, then its own.
enum status : int {
    ST_OK = 0,
    ST_NONFINITE = 10,
    ST_REENTRY = 11,
    ST_EXIT = 12,
    ST_SMALL_STEP = 13,
    ST_INTERPOLATION = 14,
};

} // namespace sgp4pj
} // namespace mzb
