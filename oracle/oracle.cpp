// CPU oracle for the conjunction-detection hot path (TEST INFRASTRUCTURE ONLY).
//
// This file restates, in plain serial C++, the algorithm mizuba runs inside
// `conjunctions::conjunctions(pj, conj_thresh, conj_det_interval, otypes, ...)`.
// It is the checker for the CUDA path of this repository: only the test suite,
// the smoke check and the CPU-baseline leg of the benchmark load it.  The
// product path never links or calls it.
//
// Stage-by-stage correspondence with the reference (paths relative to the
// mizuba source tree):
//   validation + n_cd_steps ........ mizuba/conjunctions.cpp:263-340
//   get_cd_begin_end ................ mizuba/conjunctions.cpp:373-392
//   per-object AABB ................. mizuba/detect_conjunctions_aabbs.cpp:64-252, :300-398
//   polynomial translation .......... mizuba/detail/conjunctions_jit.cpp:68-115
//   Cargo-Shisha enclosure .......... mizuba/detail/conjunctions_jit.cpp:140-298, :302-323
//   Morton codes, sort, gather ...... mizuba/detect_conjunctions_morton.cpp:70-224
//                                     (+ bit layout of detail/mortonND_LUT.h Encode)
//   BVH (level order) ............... mizuba/detect_conjunctions_bvh.cpp:267-699
//   broad phase ..................... mizuba/detect_conjunctions_broad_phase.cpp:153-339
//   narrow phase .................... mizuba/detect_conjunctions_narrow_phase.cpp:57-769
//   Chebyshev eval + interpolation .. mizuba/detail/conjunctions_jit.cpp:333-390,
//                                     mizuba/detail/poly_utils.cpp:467-535
//   root isolation + polishing ...... mizuba/detail/poly_utils.cpp:151-460
//   Horner .......................... mizuba/detail/poly_utils.hpp:41-52
//   state evaluation ................ mizuba/polyjectory.cpp:1092-1159 (pj_eval_obj_state)
//   debug verifiers (run on any outputs, the GPU's included):
//     validate_global_aabbs ......... mizuba/detect_conjunctions_aabbs.cpp:260-282
//     verify_bvh_tree ............... mizuba/detect_conjunctions_bvh.cpp:60-255
//     verify_broad_phase ............ mizuba/detect_conjunctions_broad_phase.cpp:50-137
//
// Third-party arithmetic that the reference pulls from outside its tree is
// restated from the published mathematics:
//   * heyoka 7.3 fex_check: interval-arithmetic Horner enclosure over [0, h]
//     (fast exclusion check of Biscani & Izzo, MNRAS 2022);
//   * heyoka 7.3 poly_rtscc / poly_translate_1: reverse, Taylor shift by 1,
//     Descartes sign-change count (zeros skipped);
//   * Boost toms748_solve: Alefeld, Potra & Shi, ACM TOMS 21(3) 1995,
//     Algorithm 4.2 (two interpolation steps, double-length secant, bisection
//     safeguard, mu = 1/2) with the relative 4-eps bracket tolerance;
//   * heyoka `sum` code generation: pairwise summation (the same reduction
//     mizuba itself uses in conjunctions_jit.cpp pairwise_reduce).
// The exact floating-point operation order inside heyoka's JIT is not
// observable here; this file fixes one order (no FMA contraction, compiled
// with -ffp-contract=off) and the CUDA kernels are checked against it.

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

namespace
{

constexpr unsigned MAX_OP1 = 57; // binomials stay exact integers up to order 56

struct bvh_node {
    std::uint32_t begin, end;
    std::int32_t left, right;
    float lb[4], ub[4];
};
static_assert(sizeof(bvh_node) == 48);

struct aabb_collision {
    std::uint32_t i, j;
};
static_assert(sizeof(aabb_collision) == 8);

struct conj {
    std::uint32_t i, j;
    double tca, dca;
    double ri[3], vi[3], rj[3], vj[3];
};
static_assert(sizeof(conj) == 120);

bool conj_less(const conj &a, const conj &b)
{
    // Defaulted operator<=> of the reference struct: member-wise lexicographic.
    if (a.i != b.i) return a.i < b.i;
    if (a.j != b.j) return a.j < b.j;
    if (a.tca != b.tca) return a.tca < b.tca;
    if (a.dca != b.dca) return a.dca < b.dca;
    const double *pa[4] = {a.ri, a.vi, a.rj, a.vj}, *pb[4] = {b.ri, b.vi, b.rj, b.vj};
    for (int v = 0; v < 4; ++v)
        for (int k = 0; k < 3; ++k)
            if (pa[v][k] != pb[v][k]) return pa[v][k] < pb[v][k];
    return false;
}

// Binomial coefficients as exact doubles (Pascal's triangle).
struct binom_table {
    double c[MAX_OP1][MAX_OP1]{};
    binom_table()
    {
        for (unsigned n = 0; n < MAX_OP1; ++n) {
            c[n][0] = c[n][n] = 1;
            for (unsigned k = 1; k < n; ++k) c[n][k] = c[n - 1][k - 1] + c[n - 1][k];
        }
    }
};
const binom_table BT;

// Pairwise reduction with summation (conjunctions_jit.cpp:146-168 pattern).
double pw_sum(double *v, unsigned n)
{
    while (n > 1) {
        unsigned m = 0;
        for (unsigned i = 0; i < n; i += 2) v[m++] = (i + 1 == n) ? v[i] : v[i] + v[i + 1];
        n = m;
    }
    return v[0];
}

// NaN-propagating min / max selects (conjunctions_jit.cpp:140-143).
double hy_min(double a, double b) { return (b == b) ? ((b < a) ? b : a) : b; }
double hy_max(double a, double b) { return (b == b) ? ((a < b) ? b : a) : b; }

template <typename F>
double pw_reduce(double *v, unsigned n, F f)
{
    while (n > 1) {
        unsigned m = 0;
        for (unsigned i = 0; i < n; i += 2) v[m++] = (i + 1 == n) ? v[i] : f(v[i], v[i + 1]);
        n = m;
    }
    return v[0];
}

// Powers of a by square-halving (conjunctions_jit.cpp:85-95).
void powers(double a, unsigned order, double *p)
{
    p[0] = 1;
    if (order >= 1) p[1] = a;
    for (unsigned i = 2; i <= order; ++i) p[i] = (i % 2 == 0) ? p[i / 2] * p[i / 2] : p[i / 2 + 1] * p[i / 2];
}

// c'_i = sum_{k>=i} (c_k * C(k, k-i)) * a^(k-i), pairwise summed over k
// (conjunctions_jit.cpp:68-115).  Input coefficients at c[k*stride].
void poly_translate(const double *c, std::size_t stride, unsigned order, double a, double *out)
{
    double ap[MAX_OP1], tmp[MAX_OP1];
    powers(a, order, ap);
    for (unsigned i = 0; i <= order; ++i) {
        unsigned m = 0;
        for (unsigned k = i; k <= order; ++k) tmp[m++] = (c[k * stride] * BT.c[k][k - i]) * ap[k - i];
        out[i] = pw_sum(tmp, m);
    }
}

// Cargo-Shisha enclosure over [lb, ub] (conjunctions_jit.cpp:179-267).  With
// lb_zero the translation is skipped, as heyoka folds away a translation by the
// literal zero used by the cs_enc cfunc (conjunctions_jit.cpp:302-323).
void cs_enclosure(const double *c, std::size_t stride, unsigned order, double lb, double ub, bool lb_zero,
                  double &mn, double &mx)
{
    double t[MAX_OP1], dp[MAX_OP1], b[MAX_OP1], bb[MAX_OP1];
    double delta;
    if (lb_zero) {
        for (unsigned k = 0; k <= order; ++k) t[k] = c[k * stride];
        delta = ub;
    } else {
        poly_translate(c, stride, order, lb, t);
        delta = ub - lb;
    }
    powers(delta, order, dp);
    for (unsigned i = 0; i <= order; ++i) t[i] = (t[i] * dp[i]) / BT.c[order][i];
    b[0] = t[0];
    for (unsigned k = 1; k <= order; ++k) {
        for (unsigned j = 0; j + k <= order; ++j) t[j] = t[j] + t[j + 1];
        b[k] = t[0];
    }
    std::memcpy(bb, b, sizeof(double) * (order + 1));
    mn = pw_reduce(b, order + 1, hy_min);
    mx = pw_reduce(bb, order + 1, hy_max);
}

template <typename T>
T horner(const T *c, unsigned order, T x, std::size_t stride = 1)
{
    T r = c[order * stride];
    for (unsigned o = 1; o <= order; ++o) r = c[(order - o) * stride] + r * x;
    return r;
}

struct pj_view {
    const double *traj;
    const std::uint64_t *traj_off; // [n][2] = (offset in doubles, n_steps)
    const double *time;
    const std::uint64_t *time_off;
    std::uint64_t n;
    unsigned order;
    double maxT;
    std::uint64_t nsteps(std::uint64_t i) const { return traj_off[2 * i + 1]; }
    const double *tr(std::uint64_t i) const { return traj + traj_off[2 * i]; }
    const double *tm(std::uint64_t i) const { return time + time_off[i]; }
};

std::string fmt_d(double x)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.17g", x);
    return buf;
}

// get_cd_begin_end (conjunctions.cpp:373-392).
void cd_begin_end(double maxT, std::size_t k, double interval, std::size_t n_steps, double &b, double &e)
{
    b = interval * static_cast<double>(k);
    e = (k == n_steps - 1) ? maxT : interval * static_cast<double>(k + 1);
    if (!std::isfinite(b) || !std::isfinite(e) || !(e > b) || b < 0 || e > maxT)
        throw std::invalid_argument("Invalid conjunction step time range: [" + fmt_d(b) + ", " + fmt_d(e) + ")");
}

// Half-open range of trajectory steps overlapping [cb, ce) (aabbs.cpp:130-142).
// Returns indices into the time array: steps are [it-1, it) for it in [tb, te).
void step_range(const double *t, std::uint64_t ns, double cb, double ce, std::uint64_t &tb, std::uint64_t &te)
{
    const double *b = std::upper_bound(t + 1, t + ns + 1, cb);
    const double *e = std::lower_bound(b, t + ns + 1, ce);
    e += (e != t + ns + 1);
    tb = b - t;
    te = e - t;
}

float lb_make_float(double x, std::uint64_t obj)
{
    float r = std::nextafter(static_cast<float>(x), -std::numeric_limits<float>::infinity());
    if (!std::isfinite(r))
        throw std::invalid_argument("The computation of the bounding box for the object at index " + std::to_string(obj)
                                    + " produced the non-finite lower bound " + fmt_d(r));
    return r;
}
float ub_make_float(double x, std::uint64_t obj)
{
    float r = std::nextafter(static_cast<float>(x), std::numeric_limits<float>::infinity());
    if (!std::isfinite(r))
        throw std::invalid_argument("The computation of the bounding box for the object at index " + std::to_string(obj)
                                    + " produced the non-finite upper bound " + fmt_d(r));
    return r;
}

// compute_object_aabb (aabbs.cpp:64-252).
void object_aabb(const pj_view &pj, std::uint64_t i, double cb, double ce, double thresh, float *lb, float *ub)
{
    const float inf = std::numeric_limits<float>::infinity();
    for (int d = 0; d < 4; ++d) lb[d] = inf, ub[d] = -inf;
    const auto ns = pj.nsteps(i);
    if (ns == 0) return;
    const double *t = pj.tm(i);
    if (t[0] >= ce || t[ns] <= cb) return;
    const double r = thresh / 2;
    const unsigned op1 = pj.order + 1;
    std::uint64_t tb, te;
    step_range(t, ns, cb, ce, tb, te);
    for (auto it = tb; it != te; ++it) {
        const double s0 = t[it - 1];
        const double ev_lb = std::max(cb, s0), ev_ub = std::min(ce, t[it]);
        const double h_lb = ev_lb - s0, h_ub = ev_ub - s0;
        const double *cf = pj.tr(i) + (it - 1) * op1 * 7;
        const int vars[4] = {0, 1, 2, 6};
        for (int d = 0; d < 4; ++d) {
            double mn, mx;
            cs_enclosure(cf + vars[d], 7, pj.order, h_lb, h_ub, false, mn, mx);
            mn = mn - r;
            mx = mx + r;
            lb[d] = std::min(lb[d], lb_make_float(mn, i));
            ub[d] = std::max(ub[d], ub_make_float(mx, i));
        }
    }
}

// disc_single_coord (morton.cpp:70-99).
std::uint64_t disc(float x, float mn, float mx)
{
    const float isize = mx - mn;
    float rx = (x - mn) / isize;
    rx = rx >= 0.f ? rx : 0.f;
    rx *= static_cast<float>(std::uint64_t(1) << 16);
    const auto v = static_cast<std::uint64_t>(rx);
    return std::min(v, (std::uint64_t(1) << 16) - 1);
}

// 4-D interleave: bit k of field d goes to bit 4k+d (mortonND_LUT.h Encode,
// field0 at the least significant position).
std::uint64_t morton4(std::uint64_t n0, std::uint64_t n1, std::uint64_t n2, std::uint64_t n3)
{
    const std::uint64_t f[4] = {n0, n1, n2, n3};
    std::uint64_t r = 0;
    for (unsigned k = 0; k < 16; ++k)
        for (unsigned d = 0; d < 4; ++d) r |= ((f[d] >> k) & 1u) << (4 * k + d);
    return r;
}

struct counters {
    unsigned long long cand = 0, dist2 = 0, roots = 0, fex = 0, noroot = 0, minima = 0, discarded = 0;
};

// ---------------------------------------------------------------- root finding

int sgn(double v) { return (0. < v) - (v < 0.); }

double poly_eval_1(const double *a, double x, unsigned n)
{
    double r = a[n] * n;
    for (unsigned i = 1; i < n; ++i) r = a[n - i] * (n - i) + r * x;
    return r;
}

// Fast exclusion check: interval Horner of p over [0, h]; true = no root.
bool fex_excludes(const double *p, unsigned n, double h)
{
    double lo = p[n], hi = p[n];
    for (unsigned o = 1; o <= n; ++o) {
        const double a = lo * h, b = hi * h;
        const double plo = std::min(0., std::min(a, b)), phi = std::max(0., std::max(a, b));
        lo = p[n - o] + plo;
        hi = p[n - o] + phi;
    }
    return lo > 0 || hi < 0;
}

// Taylor shift by 1: out_i = sum_{k>=i} C(k, i) in_k, pairwise summed.
void translate1(const double *in, unsigned n, double *out)
{
    double tmp[MAX_OP1];
    for (unsigned i = 0; i <= n; ++i) {
        unsigned m = 0;
        for (unsigned k = i; k <= n; ++k) tmp[m++] = BT.c[k][i] * in[k];
        out[i] = pw_sum(tmp, m);
    }
}

unsigned sign_changes(const double *c, unsigned n)
{
    unsigned cnt = 0;
    int prev = 0;
    for (unsigned k = 0; k <= n; ++k) {
        const int s = sgn(c[k]);
        if (s != 0) {
            if (prev != 0 && s != prev) ++cnt;
            prev = s;
        }
    }
    return cnt;
}

// ---- TOMS 748 (Alefeld, Potra, Shi 1995, Algorithm 4.2).
struct toms_state {
    const double *p;
    unsigned n;
    int evals = 0;
    double f(double x)
    {
        ++evals;
        return horner(p, n, x);
    }
};

bool tol_ok(double a, double b)
{
    const double eps = 4 * std::numeric_limits<double>::epsilon();
    return std::fabs(a - b) <= eps * std::min(std::fabs(a), std::fabs(b));
}

double secant_step(double a, double b, double fa, double fb)
{
    const double e5 = 5 * std::numeric_limits<double>::epsilon();
    const double c = a - (fa / (fb - fa)) * (b - a);
    if (c <= a + std::fabs(a) * e5 || c >= b - std::fabs(b) * e5) return (a + b) / 2;
    return c;
}

double guarded_div(double num, double den, double fallback)
{
    if (std::fabs(den) < 1 && std::fabs(den * std::numeric_limits<double>::max()) <= std::fabs(num)) return fallback;
    return num / den;
}

// Newton steps on the quadratic through (a,fa),(b,fb),(d,fd) (paper: NEWQUA).
double newton_quadratic(double a, double b, double d, double fa, double fb, double fd, int k)
{
    const double big = std::numeric_limits<double>::max();
    const double f_ab = guarded_div(fb - fa, b - a, big);
    double f_abd = guarded_div(fd - fb, d - b, big);
    f_abd = guarded_div(f_abd - f_ab, d - a, 0);
    if (f_abd == 0) return secant_step(a, b, fa, fb);
    double c = (sgn(f_abd) * sgn(fa) > 0) ? a : b;
    for (int i = 0; i < k; ++i)
        c -= guarded_div(fa + (f_ab + f_abd * (c - b)) * (c - a), f_ab + f_abd * (2 * c - a - b), 1 + c - a);
    if (c <= a || c >= b) c = secant_step(a, b, fa, fb);
    return c;
}

// Inverse cubic interpolation through four points (paper: IPZERO).
double inverse_cubic(double a, double b, double d, double e, double fa, double fb, double fd, double fe)
{
    const double q11 = (d - e) * fd / (fe - fd);
    const double q21 = (b - d) * fb / (fd - fb);
    const double q31 = (a - b) * fa / (fb - fa);
    const double d21 = (b - d) * fd / (fd - fb);
    const double d31 = (a - b) * fb / (fb - fa);
    const double q22 = (d21 - q11) * fb / (fe - fb);
    const double q32 = (d31 - q21) * fa / (fd - fa);
    const double d32 = (d31 - q21) * fd / (fd - fa);
    const double q33 = (d32 - q22) * fa / (fe - fa);
    double c = q31 + q32 + q33 + a;
    if (c <= a || c >= b) c = newton_quadratic(a, b, d, fa, fb, fd, 3);
    return c;
}

// Shrink [a, b] around c (paper: BRACKT), keeping c off the endpoints.
void bracket_at(toms_state &st, double &a, double &b, double c, double &fa, double &fb, double &d, double &fd)
{
    const double t = 2 * std::numeric_limits<double>::epsilon();
    if ((b - a) < 2 * t * a) c = a + (b - a) / 2;
    else if (c <= a + std::fabs(a) * t) c = a + std::fabs(a) * t;
    else if (c >= b - std::fabs(b) * t) c = b - std::fabs(b) * t;
    const double fc = st.f(c);
    if (fc == 0) {
        a = c;
        fa = 0;
        d = 0;
        fd = 0;
        return;
    }
    if (sgn(fa) * sgn(fc) < 0) {
        d = b;
        fd = fb;
        b = c;
        fb = fc;
    } else {
        d = a;
        fd = fa;
        a = c;
        fa = fc;
    }
}

bool near_equal_values(double fa, double fb, double fd, double fe)
{
    const double m = std::numeric_limits<double>::min() * 32;
    return std::fabs(fa - fb) < m || std::fabs(fa - fd) < m || std::fabs(fa - fe) < m || std::fabs(fb - fd) < m
           || std::fabs(fb - fe) < m || std::fabs(fd - fe) < m;
}

// Returns (root, flag): flag 0 success, EDOM on a non-bracketing interval,
// -1 when the evaluation budget (100) is exhausted.
std::pair<double, int> toms748(const double *p, unsigned n, double lo, double hi)
{
    constexpr int budget = 100;
    toms_state st{p, n};
    double a = lo, b = hi;
    double fa = st.f(a), fb = st.f(b);
    if (!(a < b)) return {0, EDOM};
    if (tol_ok(a, b) || fa == 0 || fb == 0) {
        if (fa == 0) b = a;
        else if (fb == 0) a = b;
        return {a / 2 + b / 2, 0};
    }
    if (sgn(fa) * sgn(fb) > 0) return {0, EDOM};
    double d = 0, fd = 0, e = 1e5, fe = 1e5;
    auto done = [&]() { return st.evals >= budget || fa == 0 || tol_ok(a, b); };
    // 4.2.1 secant, 4.2.2 quadratic.
    bracket_at(st, a, b, secant_step(a, b, fa, fb), fa, fb, d, fd);
    if (!done()) {
        const double c = newton_quadratic(a, b, d, fa, fb, fd, 2);
        e = d;
        fe = fd;
        bracket_at(st, a, b, c, fa, fb, d, fd);
    }
    while (!done()) {
        const double a0 = a, b0 = b;
        // 4.2.3: first interpolation step.
        double c = near_equal_values(fa, fb, fd, fe) ? newton_quadratic(a, b, d, fa, fb, fd, 2)
                                                     : inverse_cubic(a, b, d, e, fa, fb, fd, fe);
        e = d;
        fe = fd;
        bracket_at(st, a, b, c, fa, fb, d, fd);
        if (done()) break;
        // 4.2.4: second interpolation step.
        c = near_equal_values(fa, fb, fd, fe) ? newton_quadratic(a, b, d, fa, fb, fd, 3)
                                              : inverse_cubic(a, b, d, e, fa, fb, fd, fe);
        bracket_at(st, a, b, c, fa, fb, d, fd);
        if (done()) break;
        // 4.2.5: double-length secant from the endpoint with the smaller |f|.
        double u, fu;
        if (std::fabs(fa) < std::fabs(fb)) u = a, fu = fa;
        else u = b, fu = fb;
        c = u - 2 * (fu / (fb - fa)) * (b - a);
        if (std::fabs(c - u) > (b - a) / 2) c = a + (b - a) / 2;
        e = d;
        fe = fd;
        bracket_at(st, a, b, c, fa, fb, d, fd);
        if (done()) break;
        // 4.2.7: bisect when the bracket did not halve.
        if ((b - a) < 0.5 * (b0 - a0)) continue;
        e = d;
        fe = fd;
        bracket_at(st, a, b, a + (b - a) / 2, fa, fb, d, fd);
    }
    if (fa == 0) b = a;
    else if (fb == 0) a = b;
    const double root = a / 2 + b / 2;
    if (st.evals >= budget && !(fa == 0 || tol_ok(a, b))) return {root, -1};
    return {root, 0};
}

// run_poly_root_finding (poly_utils.cpp:272-460) for direction = +1.  Appends
// roots (already scaled to [0, rf_int)) to out; returns the fex_check flag.
bool run_root_finding(const double *poly, unsigned n, double rf_int, std::uint32_t i, std::uint32_t j,
                      std::vector<double> &out)
{
    if (fex_excludes(poly, n, rf_int)) return true;
    struct wentry {
        double lb, ub;
        double p[MAX_OP1];
    };
    std::vector<wentry> wl;
    std::vector<std::pair<double, double>> isol;
    auto add_root = [&](double root) {
        if (!std::isfinite(root))
            throw std::invalid_argument("Polynomial root finding produced a non-finite root of " + fmt_d(root)
                                        + " involving objects " + std::to_string(i) + " and " + std::to_string(j));
        const double der = poly_eval_1(poly, root, n);
        if (!std::isfinite(der))
            throw std::invalid_argument("Polynomial root finding produced the root " + fmt_d(root)
                                        + " with nonfinite derivative " + fmt_d(der) + " involving objects "
                                        + std::to_string(i) + " and " + std::to_string(j));
        if (sgn(der) == 1) out.push_back(root);
    };
    wentry first{0, 1, {}};
    {
        double f = 1;
        for (unsigned k = 0; k <= n; ++k) {
            first.p[k] = f * poly[k];
            f *= rf_int;
        }
    }
    wl.push_back(first);
    double r1[MAX_OP1], r2[MAX_OP1];
    do {
        const wentry cur = wl.back();
        wl.pop_back();
        bool tail_finite = true;
        for (unsigned k = 1; k <= n; ++k) tail_finite = tail_finite && std::isfinite(cur.p[k]);
        if (cur.p[0] == 0 && tail_finite) add_root(cur.lb * rf_int);
        for (unsigned k = 0; k <= n; ++k) r1[k] = cur.p[n - k];
        translate1(r1, n, r2);
        const unsigned nsc = sign_changes(r2, n);
        if (nsc == 1) {
            isol.emplace_back(cur.lb, cur.ub);
        } else if (nsc > 1) {
            wentry left{}, right{};
            double f = 1;
            for (unsigned k = 0; k <= n; ++k) {
                left.p[n - k] = f * cur.p[n - k];
                f *= 2;
            }
            translate1(left.p, n, right.p);
            const double mid = cur.lb / 2 + cur.ub / 2;
            left.lb = cur.lb;
            left.ub = mid;
            right.lb = mid;
            right.ub = cur.ub;
            wl.push_back(left);
            wl.push_back(right);
        }
        if (wl.size() > 250u || isol.size() > n)
            throw std::invalid_argument("The polynomial root isolation algorithm failed: the working list size is "
                                        + std::to_string(wl.size()) + " and the number of isolating intervals is "
                                        + std::to_string(isol.size()));
    } while (!wl.empty());
    if (!isol.empty()) {
        double sp[MAX_OP1];
        double f = 1;
        for (unsigned k = 0; k <= n; ++k) {
            sp[k] = f * poly[k];
            f *= rf_int;
        }
        for (auto [lb, ub] : isol) {
            if (std::isfinite(lb) && std::isfinite(ub) && ub > lb) ub = std::nextafter(ub, lb);
            const auto [root, flag] = toms748(sp, n, lb, ub);
            if (flag == -1) throw std::invalid_argument("Polynomial root finding failed due to too many iterations");
            if (flag != 0)
                throw std::invalid_argument("Polynomial root finding returned a nonzero errno with code '"
                                            + std::to_string(flag) + "'");
            add_root(root * rf_int);
        }
    }
    return false;
}

// ------------------------------------------------------------------ one step

struct step_out {
    std::vector<bvh_node> tree;
    std::vector<aabb_collision> bp;
    std::vector<conj> conjs;
    counters cnt;
};

struct ctx {
    pj_view pj;
    double thresh, interval;
    std::size_t n_cd_steps;
    const std::int32_t *otypes;
    bool skip_cd;
    std::vector<double> cheb; // (cos((2i+1)pi/(2m))+1)/2, ascending
};

void narrow_pair(const ctx &C, double cb, double ce, std::uint32_t i, std::uint32_t j, step_out &so)
{
    const pj_view &pj = C.pj;
    const unsigned n = pj.order, op1 = n + 1;
    const double thresh2 = C.thresh * C.thresh;
    const auto nsi = pj.nsteps(i), nsj = pj.nsteps(j);
    const double *ti = pj.tm(i), *tj = pj.tm(j);
    std::uint64_t bi, ei, bj, ej;
    step_range(ti, nsi, cb, ce, bi, ei);
    step_range(tj, nsj, cb, ce, bj, ej);
    thread_local std::vector<double> pti, ptj, ptd2, ptd2p, roots;
    pti.resize(7 * op1);
    ptj.resize(7 * op1);
    ptd2.resize(op1);
    ptd2p.resize(op1);
    double xe[6][MAX_OP1], f[MAX_OP1], al[MAX_OP1];
    for (auto it_i = bi, it_j = bj; it_i != ei && it_j != ej;) {
        const double si = ti[it_i - 1], sj = tj[it_j - 1];
        const double lb_i = std::max(cb, si), ub_i = std::min(ce, ti[it_i]);
        const double lb_j = std::max(cb, sj), ub_j = std::min(ce, tj[it_j]);
        const bool overlap = ub_i > lb_j && lb_i < ub_j;
        if (overlap) {
            ++so.cnt.cand;
            const double lb_rf = std::max(lb_i, lb_j), ub_rf = std::min(ub_i, ub_j);
            const double di = lb_rf - si, dj = lb_rf - sj, rf_int = ub_rf - lb_rf;
            if (!std::isfinite(di) || !std::isfinite(dj) || !std::isfinite(rf_int) || di < 0 || dj < 0 || rf_int < 0)
                throw std::invalid_argument("During the narrow phase collision detection of objects "
                                            + std::to_string(i) + " and " + std::to_string(j)
                                            + ", an invalid time interval for polynomial root finding was generated");
            const double *pi = pj.tr(i) + (it_i - 1) * op1 * 7, *pjp = pj.tr(j) + (it_j - 1) * op1 * 7;
            // pta7 translation, stored back in the [op1][7] layout.
            if (di != 0) {
                double tmp[MAX_OP1];
                for (int v = 0; v < 7; ++v) {
                    poly_translate(pi + v, 7, n, di, tmp);
                    for (unsigned k = 0; k <= n; ++k) pti[k * 7 + v] = tmp[k];
                }
                pi = pti.data();
            }
            if (dj != 0) {
                double tmp[MAX_OP1];
                for (int v = 0; v < 7; ++v) {
                    poly_translate(pjp + v, 7, n, dj, tmp);
                    for (unsigned k = 0; k <= n; ++k) ptj[k * 7 + v] = tmp[k];
                }
                pjp = ptj.data();
            }
            // Chebyshev evaluation (conjunctions_jit.cpp:333-383) and dist^2.
            for (unsigned m = 0; m < op1; ++m) al[m] = C.cheb[m] * rf_int;
            for (int v = 0; v < 3; ++v)
                for (unsigned m = 0; m < op1; ++m) {
                    xe[v][m] = horner(pi + v, n, al[m], 7);
                    xe[v + 3][m] = horner(pjp + v, n, al[m], 7);
                }
            for (unsigned m = 0; m < op1; ++m) {
                const double dx = xe[0][m] - xe[3][m], dy = xe[1][m] - xe[4][m], dz = xe[2][m] - xe[5][m];
                f[m] = dx * dx + dy * dy + dz * dz;
            }
            // Bjorck-Pereyra (poly_utils.cpp:467-535).
            double cprev[MAX_OP1], cnext[MAX_OP1];
            std::memcpy(cprev, f, sizeof(double) * op1);
            for (unsigned k = 0; k < n; ++k) {
                for (unsigned jj = 0; jj < op1; ++jj)
                    cnext[jj] = (jj <= k) ? cprev[jj] : (cprev[jj] - cprev[jj - 1]) / (al[jj] - al[jj - k - 1]);
                std::memcpy(cprev, cnext, sizeof(double) * op1);
            }
            for (unsigned idx = 0; idx < n; ++idx) {
                const unsigned k = n - idx - 1;
                for (unsigned jj = 0; jj < op1; ++jj)
                    cnext[jj] = (jj < k || jj == n) ? cprev[jj] : cprev[jj] - al[k] * cprev[jj + 1];
                std::memcpy(cprev, cnext, sizeof(double) * op1);
            }
            for (unsigned k = 0; k < op1; ++k) ptd2[k] = cprev[k];
            double emin, emax;
            cs_enclosure(ptd2.data(), 1, n, 0, rf_int, true, emin, emax);
            if (!std::isfinite(emin) || !std::isfinite(emax))
                throw std::invalid_argument("Non-finite value(s) detected during conjunction tracking for objects "
                                            + std::to_string(i) + " and " + std::to_string(j));
            if (emin < thresh2) {
                for (unsigned k = 0; k < n; ++k) ptd2p[k] = (k + 1u) * ptd2[k + 1];
                ptd2p[n] = 0;
                roots.clear();
                const bool fex = run_root_finding(ptd2p.data(), n, rf_int, i, j, roots);
                ++so.cnt.roots;
                so.cnt.fex += fex;
                so.cnt.noroot += roots.empty();
                so.cnt.minima += roots.size();
                auto add_conj = [&](double tm) {
                    conj c{};
                    c.i = i;
                    c.j = j;
                    for (int v = 0; v < 3; ++v) {
                        c.ri[v] = horner(pi + v, n, tm, 7);
                        c.vi[v] = horner(pi + 3 + v, n, tm, 7);
                        c.rj[v] = horner(pjp + v, n, tm, 7);
                        c.vj[v] = horner(pjp + 3 + v, n, tm, 7);
                    }
                    const double dx = c.ri[0] - c.rj[0], dy = c.ri[1] - c.rj[1], dz = c.ri[2] - c.rj[2];
                    c.dca = std::sqrt((dx * dx) + (dy * dy) + (dz * dz));
                    c.tca = lb_rf + tm;
                    so.conjs.push_back(c);
                };
                for (double tm : roots) {
                    const double d2 = horner(ptd2.data(), n, tm);
                    if (!std::isfinite(d2))
                        throw std::invalid_argument("A non-finite conjunction distance square of " + fmt_d(d2)
                                                    + " was computed for the objects at indices " + std::to_string(i)
                                                    + " and " + std::to_string(j));
                    if (d2 < thresh2) add_conj(tm);
                    else ++so.cnt.discarded;
                }
                // End-of-data minimum (narrow.cpp:629-673).
                if ((it_i + 1 == nsi + 1 && ti[it_i] == ub_rf) || (it_j + 1 == nsj + 1 && tj[it_j] == ub_rf)) {
                    const double tm = std::nextafter(rf_int, -1.);
                    const double dv = horner(ptd2p.data(), n, tm);
                    if (!std::isfinite(dv))
                        throw std::invalid_argument(
                            "An invalid value of " + fmt_d(dv)
                            + " was computed for the derivative of the distance square function at the upper "
                              "boundary of a trajectory");
                    if (dv < 0) {
                        const double d2 = horner(ptd2.data(), n, tm);
                        if (!std::isfinite(d2))
                            throw std::invalid_argument("An invalid value of " + fmt_d(d2)
                                                        + " was computed for a candidate minimum of the distance "
                                                          "square function at the upper boundary of a trajectory");
                        if (d2 < thresh2) add_conj(tm);
                    }
                }
                // Start-of-data minimum (narrow.cpp:683-714).
                if ((it_i == 1 && lb_rf == ti[0]) || (it_j == 1 && lb_rf == tj[0])) {
                    const double dv = horner(ptd2p.data(), n, 0.);
                    if (!std::isfinite(dv))
                        throw std::invalid_argument(
                            "An invalid value of " + fmt_d(dv)
                            + " was computed for the derivative of the distance square function at the lower "
                              "boundary of a trajectory");
                    if (dv > 0) {
                        const double d2 = horner(ptd2.data(), n, 0.);
                        if (!std::isfinite(d2))
                            throw std::invalid_argument("An invalid value of " + fmt_d(d2)
                                                        + " was computed for a candidate minimum of the distance "
                                                          "square function at the lower boundary of a trajectory");
                        if (d2 < thresh2) add_conj(0.);
                    }
                }
            } else {
                ++so.cnt.dist2;
            }
        }
        const bool inc_i = ti[it_i] <= tj[it_j], inc_j = tj[it_j] <= ti[it_i];
        it_i += inc_i;
        it_j += inc_j;
    }
}

void run_step(const ctx &C, std::size_t k, float *aabbs, std::uint64_t *mcodes, std::uint32_t *vidx,
              float *srt_aabbs, std::uint64_t *srt_mcodes, double *cd_end, step_out &so)
{
    const pj_view &pj = C.pj;
    const std::uint64_t N = pj.n;
    double cb, ce;
    cd_begin_end(pj.maxT, k, C.interval, C.n_cd_steps, cb, ce);
    const float inf = std::numeric_limits<float>::infinity();
    float glb[4] = {inf, inf, inf, inf}, gub[4] = {-inf, -inf, -inf, -inf};
    for (std::uint64_t i = 0; i < N; ++i) {
        float *lb = aabbs + i * 8, *ub = lb + 4;
        object_aabb(pj, i, cb, ce, C.thresh, lb, ub);
        for (int d = 0; d < 4; ++d) {
            glb[d] = std::min(glb[d], lb[d]);
            gub[d] = std::max(gub[d], ub[d]);
        }
    }
    for (int d = 0; d < 4; ++d) {
        if (std::isfinite(glb[d]) && !std::isfinite(gub[d] - glb[d]))
            throw std::invalid_argument("A global bounding box with non-finite size was generated");
        aabbs[N * 8 + d] = glb[d];
        aabbs[N * 8 + 4 + d] = gub[d];
    }
    *cd_end = ce;
    // Morton codes.
    for (std::uint64_t i = 0; i < N; ++i) {
        const float *lb = aabbs + i * 8, *ub = lb + 4;
        if (std::isfinite(lb[0])) {
            std::uint64_t q[4];
            for (int d = 0; d < 4; ++d) q[d] = disc(lb[d] / 2 + ub[d] / 2, glb[d], gub[d]);
            mcodes[i] = morton4(q[0], q[1], q[2], q[3]);
        } else {
            mcodes[i] = ~std::uint64_t(0);
        }
        vidx[i] = static_cast<std::uint32_t>(i);
    }
    std::stable_sort(vidx, vidx + N, [&](std::uint32_t a, std::uint32_t b) {
        if (std::isinf(aabbs[a * 8])) return false;
        if (std::isinf(aabbs[b * 8])) return true;
        return mcodes[a] < mcodes[b];
    });
    for (std::uint64_t p = 0; p < N; ++p) {
        std::memcpy(srt_aabbs + p * 8, aabbs + std::uint64_t(vidx[p]) * 8, 32);
        srt_mcodes[p] = mcodes[vidx[p]];
    }
    std::memcpy(srt_aabbs + N * 8, aabbs + N * 8, 32);

    // BVH (bvh.cpp:267-699).
    std::uint32_t neff = 0;
    while (neff < N && !std::isinf(srt_aabbs[std::uint64_t(neff) * 8])) ++neff;
    auto &tree = so.tree;
    tree.clear();
    if (neff > 0) {
        std::vector<std::uint32_t> split{0}, nn_level;
        tree.push_back({0, neff, -1, -1, {inf, inf, inf, inf}, {-inf, -inf, -inf, -inf}});
        std::size_t lbeg = 0, lend = 1;
        std::vector<std::size_t> level_begin;
        while (lbeg != lend) {
            level_begin.push_back(lbeg);
            std::vector<std::uint32_t> nolc(lend - lbeg), nc(lend - lbeg);
            for (std::size_t nd = lbeg; nd < lend; ++nd) {
                bvh_node &node = tree[nd];
                bool leaf = false;
                std::uint32_t pos = 0;
                if (node.end - node.begin > 1 && split[nd] < 64) {
                    for (;;) {
                        const std::uint64_t mask = std::uint64_t(1) << (63 - split[nd]);
                        pos = static_cast<std::uint32_t>(
                            std::partition_point(srt_mcodes + node.begin, srt_mcodes + node.end,
                                                 [mask](std::uint64_t c) { return (c & mask) == 0; })
                            - srt_mcodes);
                        if (pos != node.begin && pos != node.end) break;
                        if (++split[nd] == 64) {
                            leaf = true;
                            break;
                        }
                    }
                } else {
                    leaf = true;
                }
                if (leaf) {
                    nc[nd - lbeg] = 0;
                    for (std::uint32_t o = node.begin; o < node.end; ++o)
                        for (int d = 0; d < 4; ++d) {
                            node.lb[d] = std::min(node.lb[d], srt_aabbs[std::uint64_t(o) * 8 + d]);
                            node.ub[d] = std::max(node.ub[d], srt_aabbs[std::uint64_t(o) * 8 + 4 + d]);
                        }
                } else {
                    nc[nd - lbeg] = 2;
                    nolc[nd - lbeg] = pos - node.begin;
                }
            }
            std::size_t nnext = 0;
            const std::size_t cur_size = tree.size();
            for (std::size_t nd = lbeg; nd < lend; ++nd) {
                if (nc[nd - lbeg] == 0) continue;
                const std::size_t lc = cur_size + nnext;
                nnext += 2;
                const std::uint32_t b = tree[nd].begin, e = tree[nd].end, ls = nolc[nd - lbeg];
                tree[nd].left = static_cast<std::int32_t>(lc);
                tree[nd].right = static_cast<std::int32_t>(lc + 1);
                tree.push_back({b, b + ls, -1, -1, {inf, inf, inf, inf}, {-inf, -inf, -inf, -inf}});
                tree.push_back({b + ls, e, -1, -1, {inf, inf, inf, inf}, {-inf, -inf, -inf, -inf}});
                split.push_back(split[nd] + 1);
                split.push_back(split[nd] + 1);
            }
            lbeg = lend;
            lend = tree.size();
        }
        for (std::size_t l = level_begin.size(); l-- > 0;) {
            const std::size_t b = level_begin[l], e = (l + 1 < level_begin.size()) ? level_begin[l + 1] : tree.size();
            for (std::size_t nd = b; nd < e; ++nd) {
                bvh_node &node = tree[nd];
                if (node.left == -1) continue;
                const bvh_node &L = tree[node.left], &R = tree[node.right];
                for (int d = 0; d < 4; ++d) {
                    node.lb[d] = std::min(L.lb[d], R.lb[d]);
                    node.ub[d] = std::max(L.ub[d], R.ub[d]);
                }
            }
        }
    }
    if (C.skip_cd || tree.empty()) return;

    // Broad phase (broad_phase.cpp:153-339).
    std::vector<std::int32_t> stack;
    for (std::uint32_t p = 0; p < neff; ++p) {
        const std::uint32_t op = vidx[p];
        const std::int32_t ot = C.otypes[op];
        const float *lb = srt_aabbs + std::uint64_t(p) * 8, *ub = lb + 4;
        stack.assign(1, 0);
        do {
            const bvh_node &nd = tree[stack.back()];
            stack.pop_back();
            const bool ov = (ub[0] >= nd.lb[0] && lb[0] <= nd.ub[0]) && (ub[1] >= nd.lb[1] && lb[1] <= nd.ub[1])
                            && (ub[2] >= nd.lb[2] && lb[2] <= nd.ub[2]) && (ub[3] >= nd.lb[3] && lb[3] <= nd.ub[3]);
            if (!ov) continue;
            if (nd.left == -1) {
                for (std::uint32_t q = nd.begin; q != nd.end; ++q) {
                    const std::uint32_t oq = vidx[q];
                    if (op >= oq) continue;
                    if (ot + C.otypes[oq] <= 3) so.bp.push_back({op, oq});
                }
            } else {
                stack.push_back(nd.left);
                stack.push_back(nd.right);
            }
        } while (!stack.empty());
    }
    std::sort(so.bp.begin(), so.bp.end(),
              [](const aabb_collision &a, const aabb_collision &b) { return a.i != b.i ? a.i < b.i : a.j < b.j; });

    // Narrow phase.
    for (const auto &pr : so.bp) narrow_pair(C, cb, ce, pr.i, pr.j, so);
    std::sort(so.conjs.begin(), so.conjs.end(), [](const conj &a, const conj &b) {
        if (a.tca == b.tca) return conj_less(a, b);
        return a.tca < b.tca;
    });
}

thread_local std::string g_err;

} // namespace

struct mzo_result {
    std::size_t n_cd_steps = 0, step_begin = 0, n_run = 0, n_objs = 0;
    std::vector<float> aabbs, srt_aabbs;
    std::vector<std::uint64_t> mcodes, srt_mcodes;
    std::vector<std::uint32_t> vidx;
    std::vector<double> cd_end;
    std::vector<step_out> steps;
    std::vector<conj> conjs;
    counters cnt;
};

extern "C" {

const char *mzo_last_error(void) { return g_err.c_str(); }

// Runs the restated pipeline over conjunction steps [step_begin, step_end)
// (clamped to n_cd_steps) with n_threads worker threads.  Returns 0 on success.
int mzo_run(const double *traj, const std::uint64_t *traj_off, const double *time, const std::uint64_t *time_off,
            std::uint64_t n_objs, std::uint32_t order, double maxT, double conj_thresh, double conj_det_interval,
            const std::int32_t *otypes, std::uint64_t step_begin, std::uint64_t step_end, int n_threads,
            mzo_result **out)
{
    try {
        if (order < 2 || order + 1 > MAX_OP1) throw std::invalid_argument("unsupported polynomial order");
        if (!std::isfinite(conj_thresh) || conj_thresh <= 0)
            throw std::invalid_argument("The conjunction threshold must be finite and positive, but instead a value of "
                                        + fmt_d(conj_thresh) + " was provided");
        if (!std::isfinite(conj_thresh * conj_thresh))
            throw std::invalid_argument("A conjunction threshold of " + fmt_d(conj_thresh)
                                        + " is too large and results in an overflow error");
        if (!std::isfinite(conj_det_interval) || conj_det_interval <= 0)
            throw std::invalid_argument(
                "The conjunction detection interval must be finite and positive, but instead a value of "
                + fmt_d(conj_det_interval) + " was provided");
        std::vector<std::int32_t> ot(n_objs, 1);
        bool skip_cd = true;
        if (otypes) {
            for (std::uint64_t i = 0; i < n_objs; ++i) {
                const auto v = otypes[i];
                if (v != 1 && v != 2 && v != 4)
                    throw std::invalid_argument(
                        "The value of an object type must be one of [1, 2, 4], but a value of " + std::to_string(v)
                        + " was detected instead");
                skip_cd = skip_cd && (v != 1);
                ot[i] = v;
            }
        } else {
            skip_cd = false;
        }
        const double nsd = std::ceil(maxT / conj_det_interval);
        if (!(nsd >= 1) || !(nsd < 1e15)) throw std::invalid_argument("invalid number of conjunction steps");
        const auto n_cd_steps = static_cast<std::size_t>(nsd);
        ctx C{{traj, traj_off, time, time_off, n_objs, order, maxT}, conj_thresh, conj_det_interval, n_cd_steps,
              ot.data(), skip_cd, {}};
        const unsigned op1 = order + 1;
        C.cheb.resize(op1);
        for (unsigned m = 0; m < op1; ++m)
            C.cheb[op1 - 1 - m] = (std::cos((2. * m + 1.) / (2. * op1) * 3.14159265358979323846) + 1.) / 2.;

        auto *R = new mzo_result;
        R->n_cd_steps = n_cd_steps;
        R->n_objs = n_objs;
        R->step_begin = std::min<std::size_t>(step_begin, n_cd_steps);
        const std::size_t se = std::min<std::size_t>(step_end, n_cd_steps);
        R->n_run = se > R->step_begin ? se - R->step_begin : 0;
        const std::size_t nr = R->n_run, N = n_objs;
        R->aabbs.resize(nr * (N + 1) * 8);
        R->srt_aabbs.resize(nr * (N + 1) * 8);
        R->mcodes.resize(nr * N);
        R->srt_mcodes.resize(nr * N);
        R->vidx.resize(nr * N);
        R->cd_end.resize(nr);
        R->steps.resize(nr);
        std::atomic<std::size_t> next{0};
        std::exception_ptr eptr;
        std::mutex emtx;
        auto worker = [&]() {
            for (;;) {
                const std::size_t s = next.fetch_add(1);
                if (s >= nr) return;
                try {
                    run_step(C, R->step_begin + s, R->aabbs.data() + s * (N + 1) * 8, R->mcodes.data() + s * N,
                             R->vidx.data() + s * N, R->srt_aabbs.data() + s * (N + 1) * 8,
                             R->srt_mcodes.data() + s * N, R->cd_end.data() + s, R->steps[s]);
                } catch (...) {
                    std::lock_guard lk(emtx);
                    if (!eptr) eptr = std::current_exception();
                    next.store(nr);
                    return;
                }
            }
        };
        const int nt = std::max(1, n_threads);
        std::vector<std::thread> th;
        for (int t = 1; t < nt; ++t) th.emplace_back(worker);
        worker();
        for (auto &t : th) t.join();
        if (eptr) {
            delete R;
            std::rethrow_exception(eptr);
        }
        for (auto &so : R->steps) {
            R->conjs.insert(R->conjs.end(), so.conjs.begin(), so.conjs.end());
            R->cnt.cand += so.cnt.cand;
            R->cnt.dist2 += so.cnt.dist2;
            R->cnt.roots += so.cnt.roots;
            R->cnt.fex += so.cnt.fex;
            R->cnt.noroot += so.cnt.noroot;
            R->cnt.minima += so.cnt.minima;
            R->cnt.discarded += so.cnt.discarded;
        }
        *out = R;
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    } catch (...) {
        g_err = "unknown error";
        return 1;
    }
}

std::uint64_t mzo_n_cd_steps(const mzo_result *r) { return r->n_cd_steps; }
std::uint64_t mzo_n_run(const mzo_result *r) { return r->n_run; }
const float *mzo_aabbs(const mzo_result *r) { return r->aabbs.data(); }
const float *mzo_srt_aabbs(const mzo_result *r) { return r->srt_aabbs.data(); }
const std::uint64_t *mzo_mcodes(const mzo_result *r) { return r->mcodes.data(); }
const std::uint64_t *mzo_srt_mcodes(const mzo_result *r) { return r->srt_mcodes.data(); }
const std::uint32_t *mzo_srt_idx(const mzo_result *r) { return r->vidx.data(); }
const double *mzo_cd_end_times(const mzo_result *r) { return r->cd_end.data(); }
std::uint64_t mzo_bvh_size(const mzo_result *r, std::uint64_t s) { return r->steps[s].tree.size(); }
const void *mzo_bvh(const mzo_result *r, std::uint64_t s) { return r->steps[s].tree.data(); }
std::uint64_t mzo_bp_size(const mzo_result *r, std::uint64_t s) { return r->steps[s].bp.size(); }
const void *mzo_bp(const mzo_result *r, std::uint64_t s) { return r->steps[s].bp.data(); }
std::uint64_t mzo_conj_size(const mzo_result *r) { return r->conjs.size(); }
const void *mzo_conj(const mzo_result *r) { return r->conjs.data(); }
void mzo_np_report(const mzo_result *r, unsigned long long *o)
{
    o[0] = r->cnt.cand;
    o[1] = r->cnt.dist2;
    o[2] = r->cnt.roots;
    o[3] = r->cnt.fex;
    o[4] = r->cnt.noroot;
    o[5] = r->cnt.minima;
    o[6] = r->cnt.discarded;
}
void mzo_free(mzo_result *r) { delete r; }

// State of object obj at time tm (pj_eval_obj_state, polyjectory.cpp:1092-1159):
// NaN when the object has no data at tm, else the 7 variables by Horner's
// scheme on the segment found by upper_bound over the time points 1..n_steps.
// Evaluates n (object, time) pairs into out[n][7]; a non-finite time returns 1
// with the reference's message.
int mzo_state_eval(const double *traj, const std::uint64_t *traj_off, const double *time,
                   const std::uint64_t *time_off, std::uint32_t order, const std::uint64_t *objs, const double *tms,
                   std::uint64_t n, double *out)
{
    try {
        const std::uint64_t op1 = order + 1u;
        for (std::uint64_t e = 0; e < n; ++e) {
            const double tm = tms[e];
            if (!std::isfinite(tm))
                throw std::invalid_argument("An non-finite evaluation time of " + fmt_d(tm)
                                            + " was detected during the evaluation of a polyjectory");
            const std::uint64_t obj = objs[e];
            const std::uint64_t nsteps = traj_off[2 * obj + 1];
            double *o = out + 7 * e;
            const double *t = time + time_off[obj];
            if (nsteps == 0 || tm < t[0] || tm >= t[nsteps]) {
                for (int v = 0; v < 7; ++v) o[v] = std::numeric_limits<double>::quiet_NaN();
                continue;
            }
            const double *it = std::upper_bound(t + 1, t + nsteps + 1, tm);
            const double h = tm - *(it - 1);
            const std::uint64_t step = static_cast<std::uint64_t>(it - (t + 1));
            const double *seg = traj + traj_off[2 * obj] + step * op1 * 7;
            for (int v = 0; v < 7; ++v) o[v] = horner(seg + v, order, h, 7);
        }
        return 0;
    } catch (const std::exception &ex) {
        g_err = ex.what();
        return 1;
    }
}

// ---- Debug verifiers of the reference, as host checks on any outputs.
//
// mizuba runs these as assertions in debug builds; here they take the arrays
// as they leave the CUDA path (or the oracle) and return 0, or 1 with the
// failed check in mzo_last_error().  They check properties, not equality with
// another implementation, so they also cover steps the oracle does not run.

// The global box of a step (row n_objs of the step's aabbs) is the min/max of
// the object boxes (validate_global_aabbs, detect_conjunctions_aabbs.cpp:260-282).
int mzo_validate_global_aabbs(const float *aabbs, std::uint64_t n_objs)
{
    const float inf = std::numeric_limits<float>::infinity();
    float lb[4] = {inf, inf, inf, inf}, ub[4] = {-inf, -inf, -inf, -inf};
    for (std::uint64_t i = 0; i < n_objs; ++i)
        for (int d = 0; d < 4; ++d) {
            lb[d] = std::min(lb[d], aabbs[i * 8 + d]);
            ub[d] = std::max(ub[d], aabbs[i * 8 + 4 + d]);
        }
    for (int d = 0; d < 4; ++d)
        if (!(lb[d] == aabbs[n_objs * 8 + d]) || !(ub[d] == aabbs[n_objs * 8 + 4 + d])) {
            g_err = "global box differs from the min/max of the object boxes in dimension " + std::to_string(d);
            return 1;
        }
    return 0;
}

// Structure of one step's tree (verify_bvh_tree and verify_node_aabb,
// detect_conjunctions_bvh.cpp:60-255).  The tree covers the n_eff sorted
// objects with finite boxes.  The per-node split index, parent and level
// size of the reference's auxiliary data are not outputs; they are derived
// here from the tree itself: the parent from the child links, the split
// index of an internal node from the first differing bit of the codes at the
// boundary between its children.  On top of the reference's checks, the
// breadth-first numbering is checked: children adjacent (right = left + 1)
// and numbered in the order of their parents.
int mzo_verify_bvh_tree(const std::uint64_t *srt_mcodes, const float *srt_aabbs, std::uint64_t n_objs,
                        const void *tree_v, std::uint64_t n_nodes)
{
    const auto *tree = static_cast<const bvh_node *>(tree_v);
    auto fail = [](const std::string &m, std::uint64_t i) {
        g_err = "BVH node " + std::to_string(i) + ": " + m;
        return 1;
    };
    std::uint64_t n_eff = 0;
    while (n_eff < n_objs && !std::isinf(srt_aabbs[n_eff * 8])) ++n_eff;
    for (std::uint64_t k = n_eff; k < n_objs; ++k)
        if (!std::isinf(srt_aabbs[k * 8])) return fail("finite box after the first infinite one", k);
    if (n_eff == 0) {
        if (n_nodes != 0) return fail("non-empty tree without objects", 0);
        return 0;
    }
    if (n_nodes == 0 || n_nodes > 2 * n_eff - 1) return fail("tree size out of range", n_nodes);
    if (tree[0].begin != 0 || tree[0].end != n_eff) return fail("root does not cover the objects", 0);
    std::vector<std::int64_t> parent(n_nodes, -1);
    std::vector<int> split(n_nodes, -1);
    std::vector<char> seen(n_eff, 0);
    std::int64_t last_left = 0;
    auto first_diff = [](std::uint64_t a, std::uint64_t b) { return a == b ? 64 : __builtin_clzll(a ^ b); };
    for (std::uint64_t i = 0; i < n_nodes; ++i) {
        const bvh_node &nd = tree[i];
        if (!(nd.end > nd.begin) || nd.end > n_eff) return fail("empty or out-of-range object range", i);
        if ((nd.left == -1) != (nd.right == -1)) return fail("exactly one child", i);
        if (nd.left == -1) {
            // A leaf: one object, or several sharing one code.
            for (std::uint32_t k = nd.begin; k < nd.end; ++k) {
                if (seen[k]) return fail("object in two leaves", i);
                seen[k] = 1;
                if (srt_mcodes[k] != srt_mcodes[nd.begin]) return fail("multi-object leaf with distinct codes", i);
            }
        } else {
            const std::int64_t l = nd.left, r = nd.right;
            if (l <= std::int64_t(i) || r <= std::int64_t(i) || std::uint64_t(r) >= n_nodes)
                return fail("child index out of range", i);
            if (r != l + 1) return fail("children not adjacent", i);
            if (l <= last_left) return fail("children not in breadth-first order", i);
            last_left = l;
            const bvh_node &L = tree[l], &R = tree[r];
            if (L.begin != nd.begin || !(L.end < nd.end) || R.begin != L.end || R.end != nd.end)
                return fail("children ranges do not split the node's range", i);
            const int sp = first_diff(srt_mcodes[L.end - 1], srt_mcodes[L.end]);
            if (sp >= 64) return fail("split between equal codes", i);
            if (sp > 0) {
                const std::uint64_t pre = srt_mcodes[nd.begin] >> (64 - sp);
                for (std::uint32_t k = nd.begin + 1; k < nd.end; ++k)
                    if ((srt_mcodes[k] >> (64 - sp)) != pre) return fail("codes do not share the split prefix", i);
            } else if (i != 0) {
                return fail("split at bit 0 below the root", i);
            }
            split[i] = sp;
            if (parent[l] != -1 || parent[r] != -1) return fail("node with two parents", i);
            parent[l] = parent[r] = std::int64_t(i);
        }
        if (i > 0) {
            const std::int64_t pa = parent[i];
            if (pa < 0 || pa >= std::int64_t(i)) return fail("missing or later parent", i);
            const bvh_node &P = tree[pa];
            if (nd.begin < P.begin || nd.end > P.end || (nd.begin != P.begin && nd.end != P.end))
                return fail("range not at an end of the parent's range", i);
            if (nd.left != -1 && !(split[i] > split[pa])) return fail("split index not below the parent's", i);
        }
        // The node's box is the min/max of its objects' sorted boxes.
        const float inf = std::numeric_limits<float>::infinity();
        float lb[4] = {inf, inf, inf, inf}, ub[4] = {-inf, -inf, -inf, -inf};
        for (std::uint32_t k = nd.begin; k < nd.end; ++k)
            for (int d = 0; d < 4; ++d) {
                lb[d] = std::min(lb[d], srt_aabbs[std::uint64_t(k) * 8 + d]);
                ub[d] = std::max(ub[d], srt_aabbs[std::uint64_t(k) * 8 + 4 + d]);
            }
        for (int d = 0; d < 4; ++d)
            if (std::memcmp(&lb[d], &nd.lb[d], 4) != 0 || std::memcmp(&ub[d], &nd.ub[d], 4) != 0)
                return fail("box is not the min/max of its objects' boxes", i);
    }
    for (std::uint64_t k = 0; k < n_eff; ++k)
        if (!seen[k]) return fail("object in no leaf", k);
    return 0;
}

// Broad-phase pairs of one step against the N^2 overlap test
// (verify_broad_phase, detect_conjunctions_broad_phase.cpp:50-137): pairs
// (i, j) with i < j, strictly increasing (so unique), and every pair of
// objects whose boxes overlap (closed intervals in x, y, z, r, otype sum at
// most 3) present.  The converse is not required (multi-object leaves
// over-approximate), but *n_true receives the number of true overlaps, so
// the caller can report how far the list exceeds them.  Unlike the
// reference's version (skipped above 10,000 objects) this runs at any size,
// over n_threads threads.
int mzo_verify_broad_phase(const float *aabbs, std::uint64_t n_objs, const std::int32_t *otypes, const void *pairs_v,
                           std::uint64_t n_pairs, int n_threads, std::uint64_t *n_true)
{
    const auto *pairs = static_cast<const aabb_collision *>(pairs_v);
    for (std::uint64_t k = 0; k < n_pairs; ++k) {
        if (!(pairs[k].i < pairs[k].j) || pairs[k].j >= n_objs) {
            g_err = "pair " + std::to_string(k) + " is not (i, j) with i < j < n_objs";
            return 1;
        }
        if (k > 0 && !(pairs[k - 1].i < pairs[k].i || (pairs[k - 1].i == pairs[k].i && pairs[k - 1].j < pairs[k].j))) {
            g_err = "pairs not strictly increasing at " + std::to_string(k);
            return 1;
        }
    }
    // Row starts of the sorted pair list, for lookups by i.
    std::vector<std::uint64_t> row(n_objs + 1, 0);
    for (std::uint64_t k = 0; k < n_pairs; ++k) ++row[pairs[k].i + 1];
    for (std::uint64_t i = 0; i < n_objs; ++i) row[i + 1] += row[i];
    std::atomic<std::uint64_t> next{0}, count{0};
    std::atomic<std::int64_t> missing_i{-1}, missing_j{-1};
    auto worker = [&]() {
        std::uint64_t local = 0;
        for (;;) {
            const std::uint64_t i = next.fetch_add(1);
            if (i >= n_objs) break;
            const float *a = aabbs + i * 8;
            const std::int32_t oi = otypes ? otypes[i] : 1;
            const aabb_collision *rb = pairs + row[i], *re = pairs + row[i + 1];
            for (std::uint64_t j = i + 1; j < n_objs; ++j) {
                const float *b = aabbs + j * 8;
                const bool ov = a[4] >= b[0] && a[0] <= b[4] && a[5] >= b[1] && a[1] <= b[5] && a[6] >= b[2] &&
                                a[2] <= b[6] && a[7] >= b[3] && a[3] <= b[7] && oi + (otypes ? otypes[j] : 1) <= 3;
                if (!ov) continue;
                ++local;
                const aabb_collision key{std::uint32_t(i), std::uint32_t(j)};
                if (!std::binary_search(rb, re, key, [](const aabb_collision &x, const aabb_collision &y) {
                        return x.j < y.j;
                    })) {
                    std::int64_t exp = -1;
                    if (missing_i.compare_exchange_strong(exp, std::int64_t(i))) missing_j = std::int64_t(j);
                }
            }
        }
        count += local;
    };
    std::vector<std::thread> th;
    for (int t = 1; t < std::max(1, n_threads); ++t) th.emplace_back(worker);
    worker();
    for (auto &t : th) t.join();
    if (n_true) *n_true = count.load();
    if (missing_i.load() >= 0) {
        g_err = "overlapping boxes of objects " + std::to_string(missing_i.load()) + " and "
                + std::to_string(missing_j.load()) + " are not in the pair list";
        return 1;
    }
    if (count.load() > n_pairs) {
        g_err = "fewer pairs than true overlaps";
        return 1;
    }
    return 0;
}
}
