// CPU oracle for the SGP4 polyjectory production (TEST INFRASTRUCTURE ONLY).
//
// A serial restatement of mizuba's make_sgp4_polyjectory
// (mizuba/make_sgp4_polyjectory.cpp): the satellites' element-set spans
// (:1261-1330), the Keplerian step rule and the per-step loop (:764-913),
// the Chebyshev interpolation with error estimate and bisection
// (:325-700), in the reference's operation order.  The SGP4 propagation is
// supplied by the caller as three functions (set-up, propagate, release):
// the tests pass the reference's own propagator compiled in place
// (oracle/_ref/libsgp4_ref.so), which, as in the reference, handles the
// deep-space element sets too.  The third-party pieces (heyoka's double-
// length dates, UTC -> TAI and adaptive Taylor step) are restated from the
// published methods named beside them.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{

struct gpe {
    std::uint64_t norad_id;
    double epoch_jd1, epoch_jd2, n0, e0, i0, node0, omega0, m0, bstar;
};

using sgp4_new_fn = void *(*)(double, double, double, double, double, double, double, double, int *, int *);
using sgp4_at_fn = int (*)(void *, double, double *, double *);
using sgp4_del_fn = void (*)(void *);

// Double-length numbers: Knuth's two-sum, Dekker's fast two-sum.
struct dd {
    double hi, lo;
};
dd two_sum(double a, double b)
{
    const double s = a + b, bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
dd fast_two_sum(double a, double b)
{
    const double s = a + b;
    return {s, b - (s - a)};
}
dd add(dd a, dd b)
{
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}
dd sub(dd a, dd b) { return add(a, {-b.hi, -b.lo}); }
dd add(dd a, double b) { return add(a, dd{b, 0.0}); }
bool lt(dd a, dd b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }

// UTC -> TAI (IAU SOFA utctai, from 1972 on; TAI - UTC from IERS Bulletin C).
double tai_minus_utc(double jd0)
{
    static const double tab[][2] = {
        {2441317.5, 10}, {2441499.5, 11}, {2441683.5, 12}, {2442048.5, 13}, {2442413.5, 14}, {2442778.5, 15},
        {2443144.5, 16}, {2443509.5, 17}, {2443874.5, 18}, {2444239.5, 19}, {2444786.5, 20}, {2445151.5, 21},
        {2445516.5, 22}, {2446247.5, 23}, {2447161.5, 24}, {2447892.5, 25}, {2448257.5, 26}, {2448804.5, 27},
        {2449169.5, 28}, {2449534.5, 29}, {2450083.5, 30}, {2450630.5, 31}, {2451179.5, 32}, {2453736.5, 33},
        {2454832.5, 34}, {2456109.5, 35}, {2457204.5, 36}, {2457754.5, 37}};
    double d = tab[0][1];
    for (const auto &r : tab)
        if (jd0 >= r[0]) d = r[1];
    return d;
}
dd utc_to_tai(dd utc)
{
    if (utc.hi < 2441317.5) throw std::invalid_argument("UTC dates before 1972 are not supported");
    const double jd0 = std::floor(utc.hi - 0.5) + 0.5;
    dd fr = sub(utc, {jd0, 0.0});
    if (fr.hi < 0) fr = add(fr, 1.0);
    const double d0 = tai_minus_utc(jd0), d24 = tai_minus_utc(jd0 + 1.0);
    const double f = (fr.hi + fr.lo) * ((86400.0 + (d24 - d0)) / 86400.0);
    return add(add(dd{jd0, 0.0}, f), d0 / 86400.0);
}

constexpr int ORDER = 18, OP1 = 19;

// Keplerian step [s] from (r, v): Taylor coefficients by the
// automatic-differentiation recurrences of r^2 and (r^2)^(-3/2), then the
// Jorba-Zou step size with the exp(-0.7 / (p - 1)) safety factor of
// Biscani & Izzo (MNRAS 504, 2021), relative regime when |x| > 1.
double kepler_h(const double r[3], const double v[3])
{
    const double mu = 6.6743e-11 * 1e-9 * 5.9722e24;
    std::vector<std::vector<double>> X(3, std::vector<double>(OP1 + 1)), V(3, std::vector<double>(OP1 + 1));
    std::vector<double> U(OP1), W(OP1);
    for (int i = 0; i < 3; ++i) {
        X[i][0] = r[i];
        V[i][0] = v[i];
    }
    for (int k = 0; k < ORDER; ++k) {
        double u = 0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j <= k; ++j) u += X[i][j] * X[i][k - j];
        U[k] = u;
        if (k == 0) W[0] = std::pow(U[0], -1.5);
        else {
            double w = 0;
            for (int j = 0; j < k; ++j) w += (-1.5 * double(k - j) - double(j)) * U[k - j] * W[j];
            W[k] = w / (double(k) * U[0]);
        }
        for (int i = 0; i < 3; ++i) {
            double xw = 0;
            for (int j = 0; j <= k; ++j) xw += X[i][j] * W[k - j];
            X[i][k + 1] = V[i][k] / double(k + 1);
            V[i][k + 1] = -mu * xw / double(k + 1);
        }
    }
    double s = 0, np = 0, npm1 = 0;
    for (int i = 0; i < 3; ++i) {
        s = std::max({s, std::fabs(X[i][0]), std::fabs(V[i][0])});
        np = std::max({np, std::fabs(X[i][ORDER]), std::fabs(V[i][ORDER])});
        npm1 = std::max({npm1, std::fabs(X[i][ORDER - 1]), std::fabs(V[i][ORDER - 1])});
    }
    const double sc = s > 1 ? s : 1;
    const double rho = std::min(std::pow(sc / np, 1.0 / ORDER), std::pow(sc / npm1, 1.0 / (ORDER - 1)));
    const double e = 2.718281828459045235360287471352662;
    return rho / (e * e) * std::exp(-0.7 / double(ORDER - 1));
}

struct prop {
    sgp4_at_fn at;
    void *h;
    // x, y, z, vx, vy, vz, r at t minutes (gpe_eval_vallado, :194-230).
    int eval(double t, double o[7]) const
    {
        const int e = at(h, t, o, o + 3);
        o[6] = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
        return e;
    }
};

struct poly {
    double b, e;
    std::vector<double> cf; // [OP1][7]
};

// One step with bisection (:478-700).
int bisect(const prop &P, const double *cheb, double b0, double e0, double bs0, double es0, std::vector<poly> &out)
{
    std::vector<std::array<double, 4>> stack{{b0, e0, bs0, es0}};
    std::vector<poly> acc;
    while (!stack.empty()) {
        if (acc.size() > 20) return 14;
        const auto [b, e, bs, es] = stack.back();
        stack.pop_back();
        const double dur = e - b, dur_s = es - bs;
        if (!std::isfinite(dur) || !std::isfinite(dur_s)) return 10;
        double val[OP1][7], sp[OP1], al[OP1];
        for (int i = 0; i < OP1; ++i) {
            sp[i] = (cheb[i] + 1) / 2 * (dur_s * 1440.) + bs * 1440.;
            al[i] = (cheb[i] + 1) / 2 * dur;
        }
        for (int i = 0; i < OP1; ++i)
            if (const int c = P.eval(sp[i], val[i])) return c;
        poly p{b, e, std::vector<double>(OP1 * 7)};
        for (int v = 0; v < 7; ++v) {
            double f[OP1];
            for (int j = 0; j < OP1; ++j) f[j] = val[j][v];
            for (int k = 0; k < ORDER; ++k)
                for (int j = ORDER; j > k; --j) f[j] = (f[j] - f[j - 1]) / (al[j] - al[j - k - 1]);
            for (int k = ORDER - 1; k >= 0; --k)
                for (int j = k; j < ORDER; ++j) f[j] = f[j] - al[k] * f[j + 1];
            for (int j = 0; j < OP1; ++j) p.cf[j * 7 + v] = f[j];
        }
        if (dur < 5. / 86400.) {
            acc.push_back(std::move(p));
            continue;
        }
        double xyz[OP1][3];
        for (int i = 0; i < OP1; ++i) {
            const double ev = (i == 0 ? 0. : al[i - 1]) / 2 + al[i] / 2;
            for (int c = 0; c < 3; ++c) {
                double r = p.cf[ORDER * 7 + c];
                for (int o = 1; o <= ORDER; ++o) r = p.cf[(ORDER - o) * 7 + c] + r * ev;
                xyz[i][c] = r;
            }
        }
        double mid[OP1][7];
        for (int i = 0; i < OP1; ++i) {
            const double prev = i == 0 ? bs * 1440. : sp[i - 1];
            if (const int c = P.eval(prev / 2 + sp[i] / 2, mid[i])) return c;
        }
        double err2 = 0;
        for (int i = 0; i < OP1; ++i) {
            const double dx = xyz[i][0] - mid[i][0], dy = xyz[i][1] - mid[i][1], dz = xyz[i][2] - mid[i][2];
            const double e2 = dx * dx + dy * dy + dz * dz;
            if (!std::isfinite(e2)) return 10;
            err2 = std::max(err2, e2);
        }
        if (err2 < 1e-7 * 1e-7) {
            acc.push_back(std::move(p));
        } else {
            const double m = b + dur / 2, ms = bs + dur_s / 2;
            stack.push_back({b, m, bs, ms});
            stack.push_back({m, e, ms, es});
        }
    }
    std::sort(acc.begin(), acc.end(), [](const poly &x, const poly &y) { return x.b < y.b; });
    for (auto &p : acc) out.push_back(std::move(p));
    return 0;
}

thread_local std::string g_err2;

} // namespace

struct mzo_sgp4_pj {
    std::vector<double> traj, time;
    std::vector<std::uint64_t> toff, tmoff;
    std::vector<std::int32_t> status;
    double epoch[2];
};

extern "C" {

const char *mzo_sgp4_last_error(void) { return g_err2.c_str(); }

// The polyjectory of n element sets (sorted by NORAD ID, then epoch) over
// [jd_begin, jd_end).  Inputs are assumed valid (the GPU path's checks are
// tested separately).
int mzo_sgp4_polyjectory(const void *gpes_v, std::uint64_t n, double jd_begin, double jd_end, double reentry,
                         double exit_r, sgp4_new_fn f_new, sgp4_at_fn f_at, sgp4_del_fn f_del, mzo_sgp4_pj **out)
{
    try {
        const auto *g = static_cast<const gpe *>(gpes_v);
        auto *R = new mzo_sgp4_pj;
        double cheb[OP1];
        for (int i = 0; i < OP1; ++i) cheb[OP1 - 1 - i] = std::cos((2. * i + 1) / (2. * OP1) * 3.14159265358979323846);
        const dd jb{jd_begin, 0.0}, je{jd_end, 0.0};
        const dd pj_ep = utc_to_tai(jb);
        R->epoch[0] = pj_ep.hi;
        R->epoch[1] = pj_ep.lo;
        for (std::uint64_t i0 = 0; i0 < n;) {
            std::uint64_t i1 = i0 + 1;
            while (i1 < n && g[i1].norad_id == g[i0].norad_id) ++i1;
            std::uint64_t it = i0;
            while (it + 1 < i1 && !lt(jb, two_sum(g[it + 1].epoch_jd1, g[it + 1].epoch_jd2))) ++it;
            std::vector<poly> polys;
            int st = 0;
            dd ibeg = jb;
            for (;;) {
                bool last = false;
                dd iend;
                if (it + 1 == i1) {
                    iend = je;
                    last = true;
                } else {
                    const dd ne = two_sum(g[it + 1].epoch_jd1, g[it + 1].epoch_jd2);
                    if (!lt(ne, je)) {
                        iend = je;
                        last = true;
                    } else iend = ne;
                }
                // gpe_interpolate (:704-913).
                const gpe &e = g[it];
                const dd ep = two_sum(e.epoch_jd1, e.epoch_jd2);
                int err = 0, deep = 0;
                void *h = f_new(sub(ep, {2433281.5, 0.0}).hi, e.n0, e.e0, e.i0, e.node0, e.omega0, e.m0, e.bstar,
                                &err, &deep);
                if (err) {
                    st = err;
                    break;
                }
                const prop P{f_at, h};
                const dd ep_tai = utc_to_tai(ep), b_tai = utc_to_tai(ibeg), e_tai = utc_to_tai(iend);
                for (dd cur = b_tai;;) {
                    const double step_begin = sub(cur, pj_ep).hi;
                    const dd sb_s = sub(cur, ep_tai);
                    double r[3], v[3];
                    if ((st = f_at(h, sb_s.hi * 1440., r, v))) break;
                    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                    if (r2 < reentry * reentry) {
                        st = 11;
                        break;
                    }
                    if (r2 >= exit_r * exit_r) {
                        st = 12;
                        break;
                    }
                    const double hmax = sub(e_tai, cur).hi * 86400.;
                    double hs = kepler_h(r, v);
                    bool fin = false;
                    if (!std::isfinite(hs)) {
                        st = 10;
                        break;
                    }
                    if (hs >= hmax) {
                        hs = hmax;
                        fin = true;
                    } else if (hs < 1.) {
                        st = 13;
                        break;
                    }
                    const double step_end = step_begin + hs / 86400.;
                    const double se_s = add(sb_s, hs / 86400.).hi;
                    if ((st = bisect(P, cheb, step_begin, step_end, sb_s.hi, se_s, polys))) break;
                    if (fin) break;
                    cur = add(cur, hs / 86400.);
                }
                f_del(h);
                if (st || last) break;
                ibeg = two_sum(g[it + 1].epoch_jd1, g[it + 1].epoch_jd2);
                ++it;
            }
            R->toff.push_back(R->traj.size());
            R->toff.push_back(polys.size());
            R->tmoff.push_back(R->time.size());
            for (std::size_t k = 0; k < polys.size(); ++k) {
                R->traj.insert(R->traj.end(), polys[k].cf.begin(), polys[k].cf.end());
                if (k == 0) R->time.push_back(polys[k].b);
                R->time.push_back(polys[k].e);
            }
            R->status.push_back(st);
            i0 = i1;
        }
        *out = R;
        return 0;
    } catch (const std::exception &ex) {
        g_err2 = ex.what();
        return 1;
    }
}

std::uint64_t mzo_sgp4_pj_n_objs(const mzo_sgp4_pj *r) { return r->status.size(); }
std::uint64_t mzo_sgp4_pj_traj_size(const mzo_sgp4_pj *r) { return r->traj.size(); }
std::uint64_t mzo_sgp4_pj_time_size(const mzo_sgp4_pj *r) { return r->time.size(); }
void mzo_sgp4_pj_copy(const mzo_sgp4_pj *r, double *traj, std::uint64_t *toff, double *time, std::uint64_t *tmoff,
                      std::int32_t *status, double *epoch)
{
    std::copy(r->traj.begin(), r->traj.end(), traj);
    std::copy(r->toff.begin(), r->toff.end(), toff);
    std::copy(r->time.begin(), r->time.end(), time);
    std::copy(r->tmoff.begin(), r->tmoff.end(), tmoff);
    std::copy(r->status.begin(), r->status.end(), status);
    epoch[0] = r->epoch[0];
    epoch[1] = r->epoch[1];
}
void mzo_sgp4_pj_free(mzo_sgp4_pj *r) { delete r; }
}
