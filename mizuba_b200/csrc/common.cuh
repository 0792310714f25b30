// Shared device-side definitions for the conjunction-screening kernels.
#pragma once

#include <cmath>
#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#include "mizuba_b200.h"

namespace mzb
{

constexpr int MIN_OP1 = 3;   // order >= 2 (mizuba/polyjectory.cpp:438)
constexpr int MAX_OP1 = 33;  // orders 2..32 are compiled
constexpr int BINOM_N = 64;

// Output records, byte-identical to mizuba's structs
// (mizuba/conjunctions.hpp:65-94).
struct bvh_node {
    uint32_t begin, end;
    int32_t left, right;
    float lb[4], ub[4];
};
static_assert(sizeof(bvh_node) == 48, "bvh_node layout");

// Traversal copy of a BVH node for the broad-phase walk: one 32-byte sector
// per visit instead of the 48-byte node plus a 4-byte rope.  The box is
// quantised to 15 bits per bound on the step's global-box grid, lower bounds
// rounded down and upper bounds up, with one monotone map for every box of
// the step, so a quantised overlap test never rejects boxes whose exact test
// passes: internal nodes are pruned conservatively and leaf members keep the
// exact test, which gives the same pairs.  Bounds are packed two dimensions
// per word: q[0] = lo(x) | lo(y) << 16, q[1] = lo(z) | lo(r) << 16, q[2] and
// q[3] the upper bounds with bit 15 of each half set (see walk_overlap).
struct walk_node {
    uint32_t q[4];
    int32_t left, rope;
    uint32_t begin, end;
};
static_assert(sizeof(walk_node) == 32, "walk_node layout");

constexpr uint32_t WALK_QMAX = 32767;
constexpr uint32_t WALK_H = 0x80008000u;

// Per-step quantisation grid: origin and scale of each dimension (scale 0
// for a dimension in which every box of the step has the same bounds).
struct walk_grid {
    float g0[4], sc[4];
};
__device__ __forceinline__ walk_grid make_walk_grid(const float *gbox)
{
    walk_grid g;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const float lo = gbox[d], hi = gbox[4 + d];
        g.g0[d] = lo;
        g.sc[d] = (hi > lo) ? __fdiv_rn(float(WALK_QMAX), __fsub_rn(hi, lo)) : 0.0f;
    }
    return g;
}
// (v - g0) * sc with two roundings is monotone in v; floor / ceil and the
// clamp keep it so.
__device__ __forceinline__ uint32_t walk_q(float v, const walk_grid &g, int d, bool up)
{
    const float f = __fmul_rn(__fsub_rn(v, g.g0[d]), g.sc[d]);
    const float r = up ? ceilf(f) : floorf(f);
    return uint32_t(fminf(fmaxf(r, 0.0f), float(WALK_QMAX)));
}
__device__ __forceinline__ uint4 walk_box(const float *lb, const float *ub, const walk_grid &g)
{
    return make_uint4(walk_q(lb[0], g, 0, false) | (walk_q(lb[1], g, 1, false) << 16),
                      walk_q(lb[2], g, 2, false) | (walk_q(lb[3], g, 3, false) << 16),
                      (walk_q(ub[0], g, 0, true) | (walk_q(ub[1], g, 1, true) << 16)) | WALK_H,
                      (walk_q(ub[2], g, 2, true) | (walk_q(ub[3], g, 3, true) << 16)) | WALK_H);
}
// Closed-interval overlap of two quantised boxes, all four dimensions.  With
// every bound below 2^15 and the upper bounds carrying bit 15, the halfword
// (hi | 2^15) - lo never borrows from its neighbour and keeps bit 15 exactly
// when hi >= lo: four subtractions test the eight bound pairs.
__device__ __forceinline__ bool walk_overlap(const uint4 &a, const uint4 &b)
{
    const uint32_t m = (a.z - b.x) & (a.w - b.y) & (b.z - a.x) & (b.w - a.y);
    return (m & WALK_H) == WALK_H;
}

struct conj_rec {
    uint32_t i, j;
    double tca, dca;
    double ri[3], vi[3], rj[3], vj[3];
};
static_assert(sizeof(conj_rec) == 120, "conj layout");

// Device view of a polyjectory (segment coefficients relaid var-major).
struct dev_pj {
    int order, op1;
    uint64_t n_objs;
    double maxT;
    const double *coef;       // [gseg][7][row_ld(op1)], rows zero-padded
    const double *time;       // mizuba layout: per object n_steps+1 times
    const uint64_t *seg_off;  // per object: first global segment
    const uint64_t *time_off; // per object: offset into time
    const uint32_t *nseg;     // per object: number of segments
};

// Row stride of the coefficient array in HBM: order + 1 rounded up to an even
// number of doubles, so that every row of one variable's coefficients starts
// on a 16-byte boundary and can be read with 16-byte loads.
__host__ __device__ constexpr int row_ld(int op1) { return (op1 + 1) & ~1; }

// Coefficients of variable v of global segment gseg.
template <int OP1>
__device__ __forceinline__ const double *coef_row(const dev_pj &pj, uint64_t gseg, int v)
{
    return pj.coef + (gseg * 7 + uint64_t(v)) * row_ld(OP1);
}

// One row into registers with 16-byte loads (the row start is 16-byte
// aligned by the layout).
template <int OP1>
__device__ __forceinline__ void load_row(const double *__restrict__ row, double (&c)[OP1])
{
    const double2 *r2 = reinterpret_cast<const double2 *>(row);
#pragma unroll
    for (int k = 0; k < OP1 / 2; ++k) {
        const double2 v = __ldg(r2 + k);
        c[2 * k] = v.x;
        c[2 * k + 1] = v.y;
    }
    if (OP1 & 1) c[OP1 - 1] = __ldg(row + OP1 - 1);
}

// First-error-wins device status word.  The host turns it into the
// reference's exception message.
struct dev_status {
    int code;
    uint32_t a, b;
    uint32_t pad;
    double x, y;
};

enum err_code : int {
    ERR_NONE = 0,
    ERR_AABB_LB = 1,
    ERR_AABB_UB = 2,
    ERR_GLOBAL_AABB = 3,
    ERR_NP_INTERVAL = 4,
    ERR_NP_NONFINITE = 5,
    ERR_ISOLATION = 6,
    ERR_TOMS_ITER = 7,
    ERR_TOMS_ERRNO = 8,
    ERR_ROOT_NONFINITE = 9,
    ERR_ROOT_DER = 10,
    ERR_CONJ_D2 = 11,
    ERR_UB_DER = 12,
    ERR_UB_D2 = 13,
    ERR_LB_DER = 14,
    ERR_LB_D2 = 15,
    ERR_CAPACITY = 20,
};

__device__ __forceinline__ void set_error(dev_status *st, int code, uint32_t a, uint32_t b, double x, double y)
{
    if (atomicCAS(&st->code, 0, code) == 0) {
        st->a = a;
        st->b = b;
        st->x = x;
        st->y = y;
    }
}

// Binomial coefficients C(n, k) as exact doubles (Pascal's triangle).  Each
// translation unit holds its own copy, filled once by upload_binom_table().
static __constant__ double c_binom[BINOM_N][BINOM_N];

static inline cudaError_t upload_binom_table()
{
    static double h[BINOM_N][BINOM_N];
    for (int n = 0; n < BINOM_N; ++n) {
        for (int k = 0; k < BINOM_N; ++k) h[n][k] = 0;
        h[n][0] = h[n][n] = 1;
        for (int k = 1; k < n; ++k) h[n][k] = h[n - 1][k - 1] + h[n - 1][k];
    }
    return cudaMemcpyToSymbol(c_binom, h, sizeof(h));
}

// Ascending Chebyshev nodes of [0, 1] for one order, passed by value to the
// kernels: (cos((2i+1) pi / (2 op1)) + 1) / 2, reversed
// (conjunctions_jit.cpp:346-361).  Computed on the host with the C library
// cos, exactly as the reference builds these constants.
struct cheb_nodes {
    double v[MAX_OP1];
};

static inline cheb_nodes make_cheb_nodes(int op1)
{
    cheb_nodes c{};
    for (int m = 0; m < op1; ++m)
        c.v[op1 - 1 - m] = (std::cos((2. * m + 1.) / (2. * op1) * 3.14159265358979323846) + 1.) / 2.;
    return c;
}

// ------------------------------------------------------------------ helpers

// NaN-propagating selects (conjunctions_jit.cpp:140-143).
struct hy_min_op {
    __device__ __forceinline__ double operator()(double a, double b) const { return (b == b) ? ((b < a) ? b : a) : b; }
};
struct hy_max_op {
    __device__ __forceinline__ double operator()(double a, double b) const { return (b == b) ? ((a < b) ? b : a) : b; }
};
struct add_op {
    __device__ __forceinline__ double operator()(double a, double b) const { return a + b; }
};

// Pairwise reduction of v[0..N) (conjunctions_jit.cpp:146-168): adjacent
// pairs are combined level by level, an odd tail element is carried up.
template <int N>
struct pw {
    template <typename F>
    __device__ __forceinline__ static double reduce(double *v, F f)
    {
        constexpr int M = (N + 1) / 2;
#pragma unroll
        for (int i = 0; i < N / 2; ++i) v[i] = f(v[2 * i], v[2 * i + 1]);
        if constexpr (N % 2 == 1) v[M - 1] = v[N - 1];
        return pw<M>::reduce(v, f);
    }
};
template <>
struct pw<1> {
    template <typename F>
    __device__ __forceinline__ static double reduce(double *v, F)
    {
        return v[0];
    }
};

// Powers by square-halving (conjunctions_jit.cpp:85-95).
template <int OP1>
__device__ __forceinline__ void powers(double a, double (&p)[OP1])
{
    p[0] = 1.0;
    p[1] = a;
#pragma unroll
    for (int i = 2; i < OP1; ++i) p[i] = (i % 2 == 0) ? p[i / 2] * p[i / 2] : p[i / 2 + 1] * p[i / 2];
}

// One output coefficient of the translation x -> x + a:
// out_I = sum_{k >= I} (c_k * C(k, k - I)) * a^(k - I), pairwise summed.
template <int OP1, int I>
__device__ __forceinline__ double translate_coef(const double (&c)[OP1], const double (&ap)[OP1])
{
    constexpr int M = OP1 - I;
    double t[M];
#pragma unroll
    for (int k = 0; k < M; ++k) t[k] = (c[I + k] * c_binom[I + k][k]) * ap[k];
    return pw<M>::reduce(t, add_op{});
}

template <int OP1, int... I>
__device__ __forceinline__ void translate_impl(const double (&c)[OP1], const double (&ap)[OP1], double (&out)[OP1],
                                               std::integer_sequence<int, I...>)
{
    ((out[I] = translate_coef<OP1, I>(c, ap)), ...);
}

// Polynomial translation (conjunctions_jit.cpp:68-115); out may not alias c.
template <int OP1>
__device__ __forceinline__ void translate(const double (&c)[OP1], double a, double (&out)[OP1])
{
    double ap[OP1];
    powers<OP1>(a, ap);
    translate_impl<OP1>(c, ap, out, std::make_integer_sequence<int, OP1>{});
}

// Cargo-Shisha enclosure of an already-translated polynomial t over
// [0, delta] (conjunctions_jit.cpp:199-264).  t is consumed.
template <int OP1>
__device__ __forceinline__ void cs_from_translated(double (&t)[OP1], double delta, double &mn, double &mx)
{
    constexpr int n = OP1 - 1;
    double dp[OP1];
    powers<OP1>(delta, dp);
#pragma unroll
    for (int i = 0; i < OP1; ++i) t[i] = (t[i] * dp[i]) / c_binom[n][i];
    double b[OP1], bb[OP1];
    b[0] = t[0];
#pragma unroll
    for (int k = 1; k < OP1; ++k) {
#pragma unroll
        for (int j = 0; j + k < OP1; ++j) t[j] = t[j] + t[j + 1];
        b[k] = t[0];
    }
#pragma unroll
    for (int k = 0; k < OP1; ++k) bb[k] = b[k];
    mn = pw<OP1>::reduce(b, hy_min_op{});
    mx = pw<OP1>::reduce(bb, hy_max_op{});
}

// Horner (mizuba/detail/poly_utils.hpp:41-52), compile-time order.
template <int OP1>
__device__ __forceinline__ double horner(const double (&c)[OP1], double x)
{
    double r = c[OP1 - 1];
#pragma unroll
    for (int o = 1; o < OP1; ++o) r = c[OP1 - 1 - o] + r * x;
    return r;
}

// Runtime-order Horner over a strided array.
__device__ __forceinline__ double horner_rt(const double *c, int n, double x, int stride = 1)
{
    double r = c[n * stride];
    for (int o = 1; o <= n; ++o) r = c[(n - o) * stride] + r * x;
    return r;
}

// First step index it in [1, ns] with t[it] > v (std::upper_bound on t+1..t+ns+1).
__device__ __forceinline__ uint32_t upper_bound_t(const double *t, uint32_t lo, uint32_t hi, double v)
{
    // search in [lo, hi)
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (!(v < t[mid])) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint32_t lower_bound_t(const double *t, uint32_t lo, uint32_t hi, double v)
{
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (t[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Range [tb, te) of time indices `it` whose step [t[it-1], t[it]) overlaps
// [cb, ce) (detect_conjunctions_aabbs.cpp:130-142).
__device__ __forceinline__ void step_range(const double *t, uint32_t ns, double cb, double ce, uint32_t &tb,
                                           uint32_t &te)
{
    tb = upper_bound_t(t, 1, ns + 1, cb);
    te = lower_bound_t(t, tb, ns + 1, ce);
    te += (te != ns + 1);
}

// Order-preserving map of a float's bits to uint32 (for atomic min/max).
__device__ __forceinline__ uint32_t f2ord(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// std::nextafter(float x, +-inf) for finite or infinite x.
__device__ __forceinline__ float next_down(float x)
{
    if (x != x) return x;
    if (x == -INFINITY) return x;
    if (x == 0.0f) return -1.401298464e-45f;
    const uint32_t u = __float_as_uint(x);
    return __uint_as_float(x > 0.0f ? u - 1 : u + 1);
}
__device__ __forceinline__ float next_up(float x)
{
    if (x != x) return x;
    if (x == INFINITY) return x;
    if (x == 0.0f) return 1.401298464e-45f;
    const uint32_t u = __float_as_uint(x);
    return __uint_as_float(x > 0.0f ? u + 1 : u - 1);
}

__device__ __forceinline__ float fmin_ref(float a, float b) { return (b < a) ? b : a; }   // std::min(a, b)
__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }   // std::max(a, b)

} // namespace mzb

// Dispatch over the compiled orders: calls F<OP1>(args...) through a switch.
#define MZB_FOR_EACH_OP1(X)                                                                                          \
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) X(19) X(20) X(21) X(22)  \
        X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32) X(33)
