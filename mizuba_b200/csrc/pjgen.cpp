// Host-side synthetic polyjectory builder.
//
// mizuba builds its polyjectories with make_sgp4_polyjectory
// (mizuba/make_sgp4_polyjectory.cpp:478-913, :1461-1603), which needs heyoka
// and the SGP4 propagator.  This builder produces trajectories with the same
// structure so that the conjunction screen can be exercised at catalogue
// scale: per object a sequence of segments, each holding order-n polynomials
// (n = 18 by default) of x, y, z, vx, vy, vz and r = |(x, y, z)| in the
// mizuba layout [n_steps][order + 1][7], times in days from the epoch,
// positions in km and velocities in km/s.
//
// Motion model: Keplerian orbit with J2 secular drift of the node, argument
// of perigee and mean anomaly, plus a linear semi-major-axis decay from an
// exponential-atmosphere drag law scaled by bstar.  Objects whose perigee
// falls below 100 km altitude stop early (their trajectory ends there).
//
// Segmentation mimics the step-size control of a Taylor integrator on the
// Kepler problem: h = 0.86 * sqrt(r^3 / mu) at the segment start, r the
// orbital radius from the elements (0.86 is
// the step a tolerance-1e-14, order-18 Taylor scheme takes on a circular
// orbit, in units of the local dynamical time).  Each segment is fitted by
// sampling at the order+1 Chebyshev nodes of [0, h], Bjorck-Pereyra
// interpolation in the normalised time s = t / h (ascending nodes), and a
// midpoint error check; a segment whose positional error exceeds 1e-6 km is
// halved, at most 4 times (mirroring the bisection of
// make_sgp4_polyjectory.cpp:478-702).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace
{

constexpr double MU = 398600.8;   // km^3/s^2 (WGS72)
constexpr double RE = 6378.135;   // km (WGS72)
constexpr double J2 = 0.001082616; // WGS72
constexpr double DAY = 86400.0;
constexpr double PI = 3.14159265358979323846;

struct elems {
    double a, e, inc, raan, argp, m0, bstar;
};

struct orbit {
    elems el;
    double n0, raan_dot, argp_dot, m_dot, adot; // rad/s, km/s
    double t_end_days;                          // trajectory end (decay or span)
};

orbit make_orbit(const elems &el, double span_days)
{
    orbit o{};
    o.el = el;
    o.n0 = std::sqrt(MU / (el.a * el.a * el.a));
    const double p = el.a * (1 - el.e * el.e);
    const double f = J2 * (RE / p) * (RE / p);
    const double ci = std::cos(el.inc);
    o.raan_dot = -1.5 * f * o.n0 * ci;
    o.argp_dot = 0.75 * f * o.n0 * (5 * ci * ci - 1);
    o.m_dot = o.n0 * (1 + 0.75 * f * std::sqrt(1 - el.e * el.e) * (3 * ci * ci - 1));
    const double hp = el.a * (1 - el.e) - RE;
    // km/day decay, converted to km/s.
    const double adot_day = -60240.0 * el.bstar * std::exp(-(hp - 200.0) / 50.0);
    o.adot = adot_day / DAY;
    o.t_end_days = span_days;
    if (adot_day < 0) {
        // Perigee altitude reaches 100 km when a drops by (hp - 100) (e fixed).
        const double da = (hp - 100.0) / (1 - el.e);
        const double td = da / (-adot_day);
        if (td < span_days) o.t_end_days = td;
    }
    return o;
}

// State at time t (seconds): x, y, z, vx, vy, vz, r.  Returns the orbital
// radius a (1 - e cos E) computed from the elements (phase-independent for a
// circular orbit, so objects sharing a circular orbit share step lengths).
double state(const orbit &o, double t, double *s)
{
    const elems &el = o.el;
    const double a = el.a + o.adot * t;
    const double n = std::sqrt(MU / (a * a * a));
    // Mean anomaly: J2-corrected rate plus the quadratic drag term.
    const double ndot = -1.5 * o.n0 / el.a * o.adot;
    double M = el.m0 + o.m_dot * t + 0.5 * ndot * t * t;
    M = std::fmod(M, 2 * PI);
    const double e = el.e;
    double E = (e < 0.8) ? M : PI;
    for (int it = 0; it < 50; ++it) {
        const double d = (E - e * std::sin(E) - M) / (1 - e * std::cos(E));
        E -= d;
        if (std::fabs(d) < 1e-15) break;
    }
    const double cE = std::cos(E), sE = std::sin(E);
    const double sq = std::sqrt(1 - e * e);
    const double xp = a * (cE - e), yp = a * sq * sE;
    const double rr = a * (1 - e * cE);
    const double vfac = n * a * a / rr;
    const double vxp = -vfac * sE, vyp = vfac * sq * cE;
    const double W = el.raan + o.raan_dot * t, w = el.argp + o.argp_dot * t;
    const double cW = std::cos(W), sW = std::sin(W), cw = std::cos(w), sw = std::sin(w);
    const double ci = std::cos(el.inc), si = std::sin(el.inc);
    const double P[3] = {cW * cw - sW * sw * ci, sW * cw + cW * sw * ci, sw * si};
    const double Q[3] = {-cW * sw - sW * cw * ci, -sW * sw + cW * cw * ci, cw * si};
    for (int k = 0; k < 3; ++k) {
        s[k] = xp * P[k] + yp * Q[k];
        s[3 + k] = vxp * P[k] + vyp * Q[k];
    }
    s[6] = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    return rr;
}

// Bjorck-Pereyra solve of the Vandermonde system for ascending nodes x[0..m).
void bp_interp(const double *x, double *c, unsigned m)
{
    const unsigned n = m - 1;
    for (unsigned k = 0; k < n; ++k)
        for (unsigned j = n; j > k; --j) c[j] = (c[j] - c[j - 1]) / (x[j] - x[j - k - 1]);
    for (unsigned k = n; k-- > 0;)
        for (unsigned j = k; j < n; ++j) c[j] = c[j] - x[k] * c[j + 1];
}

struct builder {
    unsigned order;     // order of the stored polynomials
    unsigned fit_order; // order actually fitted (<= 24; higher orders are zero-padded,
                        // the monomial fit being too ill-conditioned beyond that)
    std::vector<double> cheb; // ascending Chebyshev nodes of [0, 1], fit_order + 1 of them
    double tol_km = 1e-6;

    // Fit one segment [t0, t0 + h] (days).  Writes [op1][7] coefficients in
    // days.  Returns the max midpoint position error (km).
    double fit(const orbit &o, double t0, double h, double *out) const
    {
        const unsigned op1 = fit_order + 1;
        for (unsigned k = 0; k < (order + 1) * 7u; ++k) out[k] = 0;
        std::vector<double> samp(op1 * 7), c(op1);
        double s[7];
        for (unsigned m = 0; m < op1; ++m) {
            state(o, (t0 + cheb[m] * h) * DAY, s);
            for (int v = 0; v < 7; ++v) samp[m * 7 + v] = s[v];
        }
        for (int v = 0; v < 7; ++v) {
            for (unsigned m = 0; m < op1; ++m) c[m] = samp[m * 7 + v];
            bp_interp(cheb.data(), c.data(), op1);
            double hp = 1;
            for (unsigned k = 0; k < op1; ++k) {
                out[k * 7 + v] = c[k] / hp;
                hp *= h;
            }
        }
        double err = 0;
        for (unsigned m = 0; m + 1 < op1; ++m) {
            const double tm = 0.5 * (cheb[m] + cheb[m + 1]) * h;
            state(o, (t0 + tm) * DAY, s);
            for (int v = 0; v < 3; ++v) {
                double r = out[fit_order * 7 + v];
                for (unsigned k = fit_order; k-- > 0;) r = out[k * 7 + v] + r * tm;
                err = std::max(err, std::fabs(r - s[v]));
            }
        }
        return err;
    }

    void build(const orbit &o, double t_start, std::vector<double> &traj, std::vector<double> &times,
               double &max_err) const
    {
        const unsigned op1 = order + 1;
        std::vector<double> seg(op1 * 7);
        double t = t_start;
        const double tend = o.t_end_days;
        times.push_back(t_start);
        double s[7];
        while (t < tend) {
            const double rr = state(o, t * DAY, s);
            double h = 0.86 * std::sqrt(rr * rr * rr / MU) / DAY;
            bool last = false;
            // Absorb a short remainder into this segment (no sliver segments,
            // whose scaled coefficients would overflow at high orders).
            if (t + 1.25 * h >= tend) {
                h = tend - t;
                last = true;
            }
            double err = fit(o, t, h, seg.data());
            // Halve at most 4 times: at high orders the monomial fit has an
            // error floor from conditioning that halving cannot remove.
            for (int b = 0; b < 4 && err > tol_km; ++b) {
                h *= 0.5;
                last = false;
                err = fit(o, t, h, seg.data());
            }
            max_err = std::max(max_err, err);
            traj.insert(traj.end(), seg.begin(), seg.end());
            t = last ? tend : t + h;
            times.push_back(t);
        }
    }
};

struct pjgen_out {
    std::vector<double> traj, time;
    std::vector<std::uint64_t> traj_off, time_off; // [n][2], [n]
    std::vector<std::int32_t> status;
    double max_err = 0, maxT = 0;
};

} // namespace

extern "C" {

// elems: n x 7 array (a [km], e, inc, raan, argp, M0 [rad], bstar [1/ER]).
// Trajectories cover [t_start, t_start + span_days] (days from the epoch).
// Returns an opaque handle; the arrays are read with the accessors below.
void *mzb_pjgen_build(const double *el, std::uint64_t n, double t_start, double span_days, std::uint32_t order,
                      int n_threads)
{
    auto *R = new pjgen_out;
    builder B;
    B.order = order;
    B.fit_order = order < 24 ? order : 24;
    const unsigned op1 = order + 1, fop1 = B.fit_order + 1;
    B.cheb.resize(fop1);
    for (unsigned m = 0; m < fop1; ++m)
        B.cheb[fop1 - 1 - m] = (std::cos((2. * m + 1.) / (2. * fop1) * PI) + 1.) / 2.;
    std::vector<std::vector<double>> trajs(n), times(n);
    std::vector<double> errs(std::max(1, n_threads), 0.0);
    std::vector<std::int32_t> st(n, 0);
    std::atomic<std::uint64_t> next{0};
    auto work = [&](int tid) {
        for (;;) {
            const auto i = next.fetch_add(1);
            if (i >= n) return;
            elems e{el[i * 7 + 0], el[i * 7 + 1], el[i * 7 + 2], el[i * 7 + 3],
                    el[i * 7 + 4], el[i * 7 + 5], el[i * 7 + 6]};
            const orbit o = make_orbit(e, t_start + span_days);
            if (o.t_end_days < t_start + span_days) st[i] = 11; // early termination (decay)
            if (o.t_end_days > t_start) B.build(o, t_start, trajs[i], times[i], errs[tid]);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < n_threads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &t : th) t.join();
    std::uint64_t toff = 0, tmoff = 0;
    for (std::uint64_t i = 0; i < n; ++i) {
        const std::uint64_t ns = trajs[i].size() / (op1 * 7);
        R->traj_off.push_back(toff);
        R->traj_off.push_back(ns);
        R->time_off.push_back(tmoff);
        toff += trajs[i].size();
        tmoff += times[i].size();
        if (!times[i].empty()) R->maxT = std::max(R->maxT, times[i].back());
    }
    R->traj.resize(toff);
    R->time.resize(tmoff);
    for (std::uint64_t i = 0; i < n; ++i) {
        std::memcpy(R->traj.data() + R->traj_off[2 * i], trajs[i].data(), trajs[i].size() * sizeof(double));
        std::memcpy(R->time.data() + R->time_off[i], times[i].data(), times[i].size() * sizeof(double));
    }
    R->status = st;
    for (double e : errs) R->max_err = std::max(R->max_err, e);
    return R;
}

std::uint64_t mzb_pjgen_traj_size(void *h) { return static_cast<pjgen_out *>(h)->traj.size(); }
std::uint64_t mzb_pjgen_time_size(void *h) { return static_cast<pjgen_out *>(h)->time.size(); }
const double *mzb_pjgen_traj(void *h) { return static_cast<pjgen_out *>(h)->traj.data(); }
const double *mzb_pjgen_time(void *h) { return static_cast<pjgen_out *>(h)->time.data(); }
const std::uint64_t *mzb_pjgen_traj_off(void *h) { return static_cast<pjgen_out *>(h)->traj_off.data(); }
const std::uint64_t *mzb_pjgen_time_off(void *h) { return static_cast<pjgen_out *>(h)->time_off.data(); }
const std::int32_t *mzb_pjgen_status(void *h) { return static_cast<pjgen_out *>(h)->status.data(); }
double mzb_pjgen_max_err(void *h) { return static_cast<pjgen_out *>(h)->max_err; }
double mzb_pjgen_maxT(void *h) { return static_cast<pjgen_out *>(h)->maxT; }
void mzb_pjgen_free(void *h) { delete static_cast<pjgen_out *>(h); }
}
