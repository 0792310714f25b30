// SGP4 polyjectory production on the GPU (mizuba's make_sgp4_polyjectory,
// mizuba/make_sgp4_polyjectory.cpp:478-913 and :1461-1603).
//
// For every satellite the reference walks its element sets in epoch order,
// each over the span up to the next set's epoch.  Within a span it takes
// steps of Keplerian motion from the SGP4 state at each step's start
// (sgp4pj.cuh), interpolates the SGP4 state (x, y, z, vx, vy, vz, r) at the
// order + 1 Chebyshev nodes of the step with Bjorck-Pereyra, estimates the
// position error at the midpoints between nodes against SGP4 itself, and
// bisects the step while the error is 1e-7 km or more (steps under 5 s are
// accepted as they are; more than 20 polynomials in one step is an error).
//
// Near-Earth and deep-space element sets alike (sgp4.cuh).  Here one warp
// runs one (satellite, element set) span: lanes 0..18 evaluate
// SGP4 at the 19 nodes (and then at the 19 midpoints) of a step in parallel,
// lanes 0..6 interpolate one state variable each, and the bisection stack
// lives in the warp's shared memory.  Accepted polynomials are appended to a
// pool (one atomic per polynomial) with their (span, sequence) tags; a
// gather pass lays the pool out as the polyjectory's trajectory and time
// arrays.
#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "sgp4pj.cuh"

namespace mzb
{
namespace sgp4pj
{

constexpr int WARPS = 4;
constexpr int STACK = 40;
constexpr int MAX_POLYS = 20;                  // make_sgp4_polyjectory.cpp:495-502
constexpr double MIN_STEP = 5.0 / 86400.0;     // days, make_sgp4_polyjectory.cpp:487
constexpr double ERR_THRESH = 1e-7;            // km, make_sgp4_polyjectory.cpp:490

struct seg_rec {
    uint32_t job, seq;
    double t0, t1;
};

struct nodes_t {
    double c[OP1]; // Chebyshev nodes of [-1, 1], ascending
};

struct warp_smem {
    double val[OP1][7];
    double cf[OP1][7];
    double stk[STACK][4];
    double acc_t0[MAX_POLYS + 2], acc_t1[MAX_POLYS + 2];
    unsigned long long acc_slot[MAX_POLYS + 2];
};

// SGP4 state at t [min]: x, y, z, vx, vy, vz and the radius.
__device__ __forceinline__ int state7(const sgp4::sat &s, double t, double o[7])
{
    double r[3], v[3];
    const int e = sgp4::propagate(s, t, r, v);
    o[0] = r[0];
    o[1] = r[1];
    o[2] = r[2];
    o[3] = v[0];
    o[4] = v[1];
    o[5] = v[2];
    o[6] = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    return e;
}

// The lowest lane's non-zero code (the reference checks the nodes in order).
__device__ __forceinline__ int first_code(int code)
{
    const unsigned m = __ballot_sync(0xffffffffu, code != 0);
    return m ? __shfl_sync(0xffffffffu, code, __ffs(m) - 1) : 0;
}

// Interpolation of one step [b, e) (days from the polyjectory epoch; bs, es
// the same instants in days from the element set's epoch) with bisection
// (make_sgp4_polyjectory.cpp:478-700).  Warp-collective.  Returns 0 and the
// accepted polynomials (pool slots and time spans in S.acc_*), or a status.
__device__ int interpolate_step(const sgp4::sat &sat, const nodes_t &nd, double b0, double e0, double bs0,
                                double es0, warp_smem &S, int &n_acc, double *__restrict__ pool, uint64_t cap,
                                unsigned long long *pool_count, int *overflow)
{
    const unsigned lane = threadIdx.x & 31;
    int sp = 0;
    if (lane == 0) {
        S.stk[0][0] = b0;
        S.stk[0][1] = e0;
        S.stk[0][2] = bs0;
        S.stk[0][3] = es0;
    }
    sp = 1;
    n_acc = 0;
    __syncwarp();
    while (sp > 0) {
        if (n_acc > MAX_POLYS) return ST_INTERPOLATION;
        --sp;
        const double b = S.stk[sp][0], e = S.stk[sp][1], bs = S.stk[sp][2], es = S.stk[sp][3];
        __syncwarp();
        const double dur = e - b, dur_s = es - bs;
        if (!isfinite(dur) || !isfinite(dur_s)) return ST_NONFINITE;
        // SGP4 at the nodes (minutes from the element set's epoch).
        double st[7];
        int code = 0;
        if (lane < OP1) {
            const double tp = (nd.c[lane] + 1) / 2 * (dur_s * 1440.) + bs * 1440.;
            code = state7(sat, tp, st);
            if (code == 0)
                for (int v = 0; v < 7; ++v) S.val[lane][v] = st[v];
        }
        code = first_code(code);
        if (code) return code;
        __syncwarp();
        // Bjorck-Pereyra on the nodes of [0, dur], one variable per lane
        // (vm_interp, mizuba/detail/poly_utils.cpp:467-535).
        if (lane < 7) {
            double f[OP1], al[OP1];
#pragma unroll
            for (int j = 0; j < OP1; ++j) {
                f[j] = S.val[j][lane];
                al[j] = (nd.c[j] + 1) / 2 * dur;
            }
#pragma unroll
            for (int k = 0; k < ORDER; ++k)
#pragma unroll
                for (int j = ORDER; j > k; --j) f[j] = (f[j] - f[j - 1]) / (al[j] - al[j - k - 1]);
#pragma unroll
            for (int k = ORDER - 1; k >= 0; --k)
#pragma unroll
                for (int j = k; j < ORDER; ++j) f[j] = f[j] - al[k] * f[j + 1];
#pragma unroll
            for (int j = 0; j < OP1; ++j) S.cf[j][lane] = f[j];
        }
        __syncwarp();
        bool accept = dur < MIN_STEP;
        if (!accept) {
            // Position error halfway between the nodes
            // (eval_interp_error2, make_sgp4_polyjectory.cpp:325-410).
            double err2 = 0;
            code = 0;
            int nonfinite = 0;
            if (lane < OP1) {
                const double a_cur = (nd.c[lane] + 1) / 2 * dur;
                const double a_prev = lane == 0 ? 0. : (nd.c[lane - 1] + 1) / 2 * dur;
                const double ev = a_prev / 2 + a_cur / 2;
                double xyz[3];
                for (int v = 0; v < 3; ++v) {
                    double r = S.cf[ORDER][v];
                    for (int o = 1; o <= ORDER; ++o) r = S.cf[ORDER - o][v] + r * ev;
                    xyz[v] = r;
                }
                const double s_cur = (nd.c[lane] + 1) / 2 * (dur_s * 1440.) + bs * 1440.;
                const double s_prev = lane == 0 ? bs * 1440. : (nd.c[lane - 1] + 1) / 2 * (dur_s * 1440.) + bs * 1440.;
                code = state7(sat, s_prev / 2 + s_cur / 2, st);
                const double dx = xyz[0] - st[0], dy = xyz[1] - st[1], dz = xyz[2] - st[2];
                err2 = dx * dx + dy * dy + dz * dz;
                nonfinite = !isfinite(err2);
            }
            code = first_code(code);
            if (code) return code;
            if (__any_sync(0xffffffffu, nonfinite)) return ST_NONFINITE;
            for (int o = 16; o > 0; o >>= 1) err2 = fmax(err2, __shfl_xor_sync(0xffffffffu, err2, o));
            accept = err2 < ERR_THRESH * ERR_THRESH;
        }
        if (accept) {
            unsigned long long slot = 0;
            if (lane == 0) slot = atomicAdd(pool_count, 1ull);
            slot = __shfl_sync(0xffffffffu, slot, 0);
            if (slot < cap) {
                double *dst = pool + slot * uint64_t(OP1 * 7);
                for (int k = lane; k < OP1 * 7; k += 32) dst[k] = S.cf[k / 7][k % 7];
            } else if (lane == 0) {
                *overflow = 1;
            }
            if (lane == 0) {
                S.acc_slot[n_acc] = slot;
                S.acc_t0[n_acc] = b;
                S.acc_t1[n_acc] = e;
            }
            ++n_acc;
        } else {
            if (sp + 2 > STACK) return ST_INTERPOLATION;
            const double mid = b + dur / 2, mid_s = bs + dur_s / 2;
            if (lane == 0) {
                S.stk[sp][0] = b;
                S.stk[sp][1] = mid;
                S.stk[sp][2] = bs;
                S.stk[sp][3] = mid_s;
                S.stk[sp + 1][0] = mid;
                S.stk[sp + 1][1] = e;
                S.stk[sp + 1][2] = mid_s;
                S.stk[sp + 1][3] = es;
            }
            sp += 2;
        }
        __syncwarp();
    }
    return 0;
}

// Each warp takes the next job of `order` (the jobs by decreasing expected
// work: mean motion times span) from the counter *next until none is left,
// so that the long low-orbit spans start first and the short ones fill in
// at the end, and warps of one SM tend to run the same propagator branch.
__global__ void __launch_bounds__(32 * WARPS, 4) k_sgp4_pj(const job *__restrict__ jobs, uint32_t n_jobs,
                                                        const uint32_t *__restrict__ order, uint32_t *next,
                                                        dfl pj_epoch, double reentry, double exit_r, nodes_t nd,
                                                        double *__restrict__ pool, seg_rec *__restrict__ recs,
                                                        uint64_t cap, unsigned long long *pool_count, int *overflow,
                                                        int *__restrict__ job_status,
                                                        uint32_t *__restrict__ job_committed, uint64_t max_steps)
{
    __shared__ warp_smem smem[WARPS];
    const unsigned w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    warp_smem &S = smem[w];
    for (;;) {
        uint32_t kq = 0;
        if (lane == 0) kq = atomicAdd(next, 1u);
        kq = __shfl_sync(0xffffffffu, kq, 0);
        if (kq >= n_jobs) break;
        const uint32_t jb = order[kq];
        const job J = jobs[jb];
        int st = 0;
        uint32_t committed = 0;
        sgp4::sat sat;
        st = sgp4::setup(J.n0, J.e0, J.i0, J.node0, J.omega0, J.m0, J.bstar, J.epoch1950, sat);
        dfl cur = J.begin_tai;
        // Every step but the last is at least 1 s long, so max_steps bounds
        // the loop; reaching it reports the small-step status.
        for (uint64_t it = 0; st == 0; ++it) {
            if (it >= max_steps) {
                st = ST_SMALL_STEP;
                break;
            }
            const double step_begin = dfl_sub(cur, pj_epoch).hi;
            const dfl sb_s = dfl_sub(cur, J.epoch_tai);
            double r[3], v[3];
            int e = sgp4::propagate(sat, sb_s.hi * 1440., r, v);
            if (e) {
                st = e;
                break;
            }
            const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (r2 < reentry * reentry) {
                st = ST_REENTRY;
                break;
            }
            if (r2 >= exit_r * exit_r) {
                st = ST_EXIT;
                break;
            }
            const double hmax = dfl_sub(J.end_tai, cur).hi * 86400.;
            double h = kepler_step(r, v);
            bool last = false;
            if (!isfinite(h)) {
                st = ST_NONFINITE;
                break;
            }
            if (h >= hmax) {
                h = hmax;
                last = true;
            } else if (h < 1.) {
                st = ST_SMALL_STEP;
                break;
            }
            const double step_end = step_begin + h / 86400.;
            const double se_s = dfl_add(sb_s, h / 86400.).hi;
            int n_acc = 0;
            st = interpolate_step(sat, nd, step_begin, step_end, sb_s.hi, se_s, S, n_acc, pool, cap, pool_count,
                                  overflow);
            if (st) break;
            // The step's polynomials in time order, tagged (span, sequence).
            if (lane == 0) {
                for (int a = 1; a < n_acc; ++a)
                    for (int c = a; c > 0 && S.acc_t0[c] < S.acc_t0[c - 1]; --c) {
                        const double t0 = S.acc_t0[c], t1 = S.acc_t1[c];
                        const unsigned long long sl = S.acc_slot[c];
                        S.acc_t0[c] = S.acc_t0[c - 1];
                        S.acc_t1[c] = S.acc_t1[c - 1];
                        S.acc_slot[c] = S.acc_slot[c - 1];
                        S.acc_t0[c - 1] = t0;
                        S.acc_t1[c - 1] = t1;
                        S.acc_slot[c - 1] = sl;
                    }
                for (int a = 0; a < n_acc; ++a)
                    if (S.acc_slot[a] < cap) recs[S.acc_slot[a]] = seg_rec{jb, committed + a, S.acc_t0[a], S.acc_t1[a]};
            }
            __syncwarp();
            committed += uint32_t(n_acc);
            if (last) break;
            cur = dfl_add(cur, h / 86400.);
        }
        if (lane == 0) {
            job_status[jb] = st;
            job_committed[jb] = committed;
        }
        __syncwarp();
    }
}

// Lays the pool out as the polyjectory: segment dest = seg_base[job] + seq,
// its coefficients (mizuba layout [order + 1][7]) and its end time; the
// first segment of each satellite also writes the start time.
__global__ void k_sgp4_gather(const double *__restrict__ pool, const seg_rec *__restrict__ recs, uint64_t n_slots,
                              const uint64_t *__restrict__ seg_base, const uint32_t *__restrict__ keep,
                              const uint32_t *__restrict__ job_sat, const uint64_t *__restrict__ sat_seg_off,
                              const uint64_t *__restrict__ sat_time_off, double *__restrict__ traj,
                              double *__restrict__ time, unsigned long long *bad_seg)
{
    const uint64_t per = uint64_t(OP1) * 7;
    for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < n_slots * per;
         g += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t slot = g / per, k = g % per;
        const seg_rec rc = recs[slot];
        if (rc.job == 0xffffffffu || rc.seq >= keep[rc.job]) continue;
        const uint64_t dest = seg_base[rc.job] + rc.seq;
        const double v = pool[slot * per + k];
        // The polyjectory constructor's finiteness check (polyjectory.cpp:
        // 558-569), on the coefficients as they are laid out.
        if (!isfinite(v)) atomicMin(bad_seg, (unsigned long long)dest);
        traj[dest * per + k] = v;
        if (k == 0) {
            const uint32_t sat = job_sat[rc.job];
            const uint64_t local = dest - sat_seg_off[sat];
            time[sat_time_off[sat] + local + 1] = rc.t1;
            if (local == 0) time[sat_time_off[sat]] = rc.t0;
        }
    }
}

__global__ void k_sgp4_propagate(const job *__restrict__ jobs, uint64_t n, const double *__restrict__ tsince,
                                 uint64_t n_t, double *__restrict__ out, int *__restrict__ err)
{
    for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < n * n_t;
         g += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t i = g / n_t, t = g % n_t;
        const job J = jobs[i];
        double *o = out + g * 6;
        sgp4::sat sat;
        int e = sgp4::setup(J.n0, J.e0, J.i0, J.node0, J.omega0, J.m0, J.bstar, J.epoch1950, sat);
        if (e == 0) e = sgp4::propagate(sat, tsince[t], o, o + 3);
        err[g] = e;
    }
}

} // namespace sgp4pj

// ------------------------------------------------------------ host driver

namespace
{

[[noreturn]] void sgp4_cuda_fail(cudaError_t e, const char *what)
{
    throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
#define SK(x)                                                                                                        \
    do {                                                                                                               \
        const cudaError_t e_ = (x);                                                                                    \
        if (e_ != cudaSuccess) sgp4_cuda_fail(e_, #x);                                                                 \
    } while (0)

template <typename T>
struct devbuf {
    T *p = nullptr;
    size_t n = 0;
    devbuf() = default;
    explicit devbuf(size_t count) { alloc(count); }
    devbuf(const devbuf &) = delete;
    devbuf &operator=(const devbuf &) = delete;
    ~devbuf()
    {
        if (p) cudaFree(p);
    }
    void alloc(size_t count)
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (count) SK(cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T)));
    }
};

std::string fmt_g(double x)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.17g", x);
    return buf;
}

// TAI - UTC in seconds from 1972 on (IERS Bulletin C): the Julian date of
// 0h UTC on which each value takes effect.
struct leap {
    double jd;
    double dat;
};
const leap LEAPS[] = {
    {2441317.5, 10}, {2441499.5, 11}, {2441683.5, 12}, {2442048.5, 13}, {2442413.5, 14}, {2442778.5, 15},
    {2443144.5, 16}, {2443509.5, 17}, {2443874.5, 18}, {2444239.5, 19}, {2444786.5, 20}, {2445151.5, 21},
    {2445516.5, 22}, {2446247.5, 23}, {2447161.5, 24}, {2447892.5, 25}, {2448257.5, 26}, {2448804.5, 27},
    {2449169.5, 28}, {2449534.5, 29}, {2450083.5, 30}, {2450630.5, 31}, {2451179.5, 32}, {2453736.5, 33},
    {2454832.5, 34}, {2456109.5, 35}, {2457204.5, 36}, {2457754.5, 37},
};

double dat_at(double jd0)
{
    double d = LEAPS[0].dat;
    for (const leap &l : LEAPS)
        if (jd0 >= l.jd) d = l.dat;
    return d;
}

} // namespace

namespace sgp4pj
{

// UTC -> TAI for a double-length Julian date, from 1972 on, the way the IAU
// SOFA library's utctai does it: the instant's UTC day starts at jd0 (0h),
// TAI - UTC at 0h (dat0) applies to the whole day, and on a day that ends
// with a leap second the day's fraction is stretched over 86400 + 1 SI
// seconds.
dfl utc_to_tai(dfl utc)
{
    if (utc.hi < LEAPS[0].jd) throw std::invalid_argument("UTC dates before 1972 are not supported by make_sgp4_polyjectory()");
    const double jd0 = std::floor(utc.hi - 0.5) + 0.5;
    dfl frac = dfl_sub(utc, dfl{jd0, 0.0});
    if (frac.hi < 0) frac = dfl_add(frac, 1.0);
    const double dat0 = dat_at(jd0), dat24 = dat_at(jd0 + 1.0);
    const double dleap = dat24 - dat0;
    const double scale = (86400.0 + dleap) / 86400.0;
    const double f = (frac.hi + frac.lo) * scale;
    return dfl_add(dfl_add(dfl{jd0, 0.0}, f), dat0 / 86400.0);
}

void gpe_check(const gpe_host *g, uint64_t n, double jd_begin, double jd_end, double reentry, double exit_r)
{
    if (!std::isfinite(jd_begin) || !std::isfinite(jd_end) || !(jd_begin < jd_end))
        throw std::invalid_argument("Invalid Julian date interval [" + fmt_g(jd_begin) + ", " + fmt_g(jd_end)
                                    + ") supplied to make_sgp4_polyjectory(): the begin/end dates must be finite and "
                                      "the end date must be strictly after the begin date");
    if (std::isnan(reentry) || std::isnan(exit_r))
        throw std::invalid_argument("The reentry/exit radiuses in make_sgp4_polyjectory() cannot be NaN");
    if (!(reentry < exit_r))
        throw std::invalid_argument("The reentry radius (" + fmt_g(reentry) + ") must be less than the exit radius ("
                                    + fmt_g(exit_r) + ") in make_sgp4_polyjectory()");
    if (n == 0) throw std::invalid_argument("make_sgp4_polyjectory() requires a non-empty array of GPEs in input");
    // make_sgp4_polyjectory.cpp:123-148: every field finite, in field order.
    static const char *names[] = {"epoch_jd1", "epoch_jd2", "n0", "e0", "i0", "node0", "omega0", "m0", "bstar"};
    for (uint64_t i = 0; i < n; ++i) {
        const double f[] = {g[i].epoch_jd1, g[i].epoch_jd2, g[i].n0,     g[i].e0,   g[i].i0,
                            g[i].node0,     g[i].omega0,    g[i].m0,     g[i].bstar};
        for (int k = 0; k < 9; ++k)
            if (!std::isfinite(f[k]))
                throw std::invalid_argument(std::string("Invalid GPE detected by make_sgp4_polyjectory(): the '")
                                            + names[k] + "' of the GPE at index " + std::to_string(i)
                                            + " is not finite");
    }
    // make_sgp4_polyjectory.cpp:150-185: sorted by NORAD ID, then epoch,
    // and no two sets of one satellite with the same epoch.
    for (uint64_t i = 0; i + 1 < n; ++i) {
        const gpe_host &a = g[i], &b = g[i + 1];
        bool unsorted = b.norad_id < a.norad_id;
        if (b.norad_id == a.norad_id) {
            const dfl ea = dfl_norm(a.epoch_jd1, a.epoch_jd2), eb = dfl_norm(b.epoch_jd1, b.epoch_jd2);
            unsorted = dfl_lt(eb, ea);
            if (!unsorted && !dfl_lt(ea, eb))
                throw std::invalid_argument("Two GPEs with identical NORAD ID " + std::to_string(a.norad_id)
                                            + " and epoch (" + fmt_g(b.epoch_jd1) + ", " + fmt_g(b.epoch_jd2)
                                            + ") were identified by make_sgp4_polyjectory() - this is not allowed");
        }
        if (unsorted)
            throw std::invalid_argument("The set of GPEs passed to make_sgp4_polyjectory() is not sorted correctly: "
                                        "it must be ordered first by NORAD ID and then by epoch");
    }
}

sgp4_pj_out *make_sgp4_pj(const gpe_host *g, uint64_t n, double jd_begin, double jd_end, double reentry,
                          double exit_r)
{
    gpe_check(g, n, jd_begin, jd_end, reentry, exit_r);
    auto out = std::make_unique<sgp4_pj_out>();
    const dfl jb{jd_begin, 0.0}, je{jd_end, 0.0};
    out->epoch = utc_to_tai(jb);
    // Satellites (runs of equal NORAD IDs) and their spans
    // (make_sgp4_polyjectory.cpp:1261-1330).
    std::vector<job> jobs;
    std::vector<uint32_t> sat_first_job;
    uint32_t n_sats = 0;
    for (uint64_t i0 = 0; i0 < n;) {
        uint64_t i1 = i0 + 1;
        while (i1 < n && g[i1].norad_id == g[i0].norad_id) ++i1;
        // The last set with epoch <= jd_begin (or the first set).
        uint64_t it = i0;
        while (it + 1 < i1 && dfl_le(dfl_norm(g[it + 1].epoch_jd1, g[it + 1].epoch_jd2), jb)) ++it;
        sat_first_job.push_back(uint32_t(jobs.size()));
        dfl ibeg = jb;
        for (uint32_t k = 0;; ++k) {
            bool last = false;
            dfl iend;
            if (it + 1 == i1) {
                iend = je;
                last = true;
            } else {
                const dfl ne = dfl_norm(g[it + 1].epoch_jd1, g[it + 1].epoch_jd2);
                if (!dfl_lt(ne, je)) {
                    iend = je;
                    last = true;
                } else {
                    iend = ne;
                }
            }
            const gpe_host &e = g[it];
            job J{};
            J.n0 = e.n0;
            J.e0 = e.e0;
            J.i0 = e.i0;
            J.node0 = e.node0;
            J.omega0 = e.omega0;
            J.m0 = e.m0;
            J.bstar = e.bstar;
            J.epoch1950 = dfl_sub(dfl_norm(e.epoch_jd1, e.epoch_jd2), dfl{2433281.5, 0.0}).hi;
            J.epoch_tai = utc_to_tai(dfl_norm(e.epoch_jd1, e.epoch_jd2));
            J.begin_tai = utc_to_tai(ibeg);
            J.end_tai = utc_to_tai(iend);
            J.sat = n_sats;
            J.k = k;
            jobs.push_back(J);
            if (last) break;
            ibeg = dfl_norm(g[it + 1].epoch_jd1, g[it + 1].epoch_jd2);
            ++it;
        }
        ++n_sats;
        i0 = i1;
    }
    sat_first_job.push_back(uint32_t(jobs.size()));
    const uint32_t n_jobs = uint32_t(jobs.size());

    nodes_t nd{};
    for (int i = 0; i < OP1; ++i)
        nd.c[OP1 - 1 - i] = std::cos((2. * i + 1) / (2. * OP1) * 3.14159265358979323846);

    devbuf<job> d_jobs(n_jobs);
    SK(cudaMemcpy(d_jobs.p, jobs.data(), n_jobs * sizeof(job), cudaMemcpyHostToDevice));
    // Execution order: decreasing mean motion x span length (the number of
    // Keplerian steps a span takes grows with both).
    std::vector<uint32_t> order(n_jobs);
    for (uint32_t j = 0; j < n_jobs; ++j) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        const double wa = jobs[a].n0 * dfl_sub(jobs[a].end_tai, jobs[a].begin_tai).hi;
        const double wb = jobs[b].n0 * dfl_sub(jobs[b].end_tai, jobs[b].begin_tai).hi;
        return wa > wb;
    });
    devbuf<uint32_t> d_order(n_jobs), d_next(1);
    SK(cudaMemcpy(d_order.p, order.data(), n_jobs * sizeof(uint32_t), cudaMemcpyHostToDevice));
    devbuf<int> d_status(n_jobs), d_overflow(1);
    devbuf<uint32_t> d_committed(n_jobs);
    devbuf<unsigned long long> d_count(1);
    const double span_s = (jd_end - jd_begin) * 86400.0;
    const uint64_t max_steps = uint64_t(span_s) + 16;
    // Pool capacity: about 150 steps a day per span for low orbits, grown
    // and rerun on overflow.
    uint64_t cap = uint64_t(n_jobs) * 64 + uint64_t(std::ceil(std::max(1.0, jd_end - jd_begin)) * 160.0) * n_sats;
    devbuf<double> pool;
    devbuf<seg_rec> recs;
    unsigned long long count = 0;
    int dev = 0, n_sm = 148;
    SK(cudaGetDevice(&dev));
    SK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    struct ev_pair {
        cudaEvent_t a = nullptr, b = nullptr;
        ev_pair()
        {
            SK(cudaEventCreate(&a));
            SK(cudaEventCreate(&b));
        }
        ~ev_pair()
        {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
        float ms() const
        {
            float t = 0;
            cudaEventElapsedTime(&t, a, b);
            return t;
        }
    } ev_k, ev_g;
    for (;;) {
        pool.alloc(cap * OP1 * 7);
        recs.alloc(cap);
        SK(cudaMemset(recs.p, 0xff, cap * sizeof(seg_rec)));
        SK(cudaMemset(d_count.p, 0, sizeof(unsigned long long)));
        SK(cudaMemset(d_overflow.p, 0, sizeof(int)));
        SK(cudaMemset(d_next.p, 0, sizeof(uint32_t)));
        const unsigned grid = unsigned(std::min<uint64_t>((n_jobs + WARPS - 1) / WARPS, uint64_t(n_sm) * 16));
        SK(cudaEventRecord(ev_k.a));
        k_sgp4_pj<<<grid, 32 * WARPS>>>(d_jobs.p, n_jobs, d_order.p, d_next.p, out->epoch, reentry, exit_r, nd, pool.p,
                                          recs.p, cap,
                                          d_count.p, d_overflow.p, d_status.p, d_committed.p, max_steps);
        SK(cudaEventRecord(ev_k.b));
        ++out->n_launches;
        SK(cudaGetLastError());
        SK(cudaMemcpy(&count, d_count.p, sizeof(count), cudaMemcpyDeviceToHost));
        if (count <= cap) break;
        cap = count + count / 8 + 1024;
    }
    out->kernel_ms = ev_k.ms();
    std::vector<int> status(n_jobs);
    std::vector<uint32_t> committed(n_jobs);
    SK(cudaMemcpy(status.data(), d_status.p, n_jobs * sizeof(int), cudaMemcpyDeviceToHost));
    SK(cudaMemcpy(committed.data(), d_committed.p, n_jobs * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    // Per satellite: its spans in order up to the first that failed (the
    // failing span keeps the steps completed before the error).
    std::vector<uint64_t> seg_base(n_jobs, 0), sat_seg_off(n_sats), sat_time_off(n_sats);
    std::vector<uint32_t> keep(n_jobs, 0), job_sat(n_jobs);
    out->status.assign(n_sats, 0);
    out->traj_off.resize(2 * size_t(n_sats));
    out->time_off.resize(n_sats);
    uint64_t seg_cursor = 0, time_cursor = 0;
    for (uint32_t s = 0; s < n_sats; ++s) {
        sat_seg_off[s] = seg_cursor;
        sat_time_off[s] = time_cursor;
        uint64_t nseg = 0;
        for (uint32_t j = sat_first_job[s]; j < sat_first_job[s + 1]; ++j) {
            job_sat[j] = s;
            seg_base[j] = seg_cursor + nseg;
            keep[j] = committed[j];
            nseg += committed[j];
            if (status[j] != 0) {
                out->status[s] = status[j];
                for (uint32_t q = j + 1; q < sat_first_job[s + 1]; ++q) job_sat[q] = s;
                break;
            }
        }
        out->traj_off[2 * s] = seg_cursor * OP1 * 7;
        out->traj_off[2 * s + 1] = nseg;
        out->time_off[s] = time_cursor;
        seg_cursor += nseg;
        time_cursor += nseg ? nseg + 1 : 0;
    }
    devbuf<uint64_t> d_seg_base(n_jobs), d_sat_seg_off(n_sats), d_sat_time_off(n_sats);
    devbuf<uint32_t> d_keep(n_jobs), d_job_sat(n_jobs);
    SK(cudaMemcpy(d_seg_base.p, seg_base.data(), n_jobs * 8, cudaMemcpyHostToDevice));
    SK(cudaMemcpy(d_keep.p, keep.data(), n_jobs * 4, cudaMemcpyHostToDevice));
    SK(cudaMemcpy(d_job_sat.p, job_sat.data(), n_jobs * 4, cudaMemcpyHostToDevice));
    SK(cudaMemcpy(d_sat_seg_off.p, sat_seg_off.data(), n_sats * 8, cudaMemcpyHostToDevice));
    SK(cudaMemcpy(d_sat_time_off.p, sat_time_off.data(), n_sats * 8, cudaMemcpyHostToDevice));
    out->n_traj = seg_cursor * OP1 * 7;
    if (out->n_traj) SK(cudaMalloc(reinterpret_cast<void **>(&out->d_traj), out->n_traj * sizeof(double)));
    devbuf<double> d_time(time_cursor);
    devbuf<unsigned long long> d_bad(1);
    SK(cudaMemset(d_bad.p, 0xff, sizeof(unsigned long long)));
    if (seg_cursor) {
        SK(cudaEventRecord(ev_g.a));
        k_sgp4_gather<<<n_sm * 8, 256>>>(pool.p, recs.p, count, d_seg_base.p, d_keep.p, d_job_sat.p,
                                          d_sat_seg_off.p, d_sat_time_off.p, out->d_traj, d_time.p, d_bad.p);
        SK(cudaEventRecord(ev_g.b));
        ++out->n_launches;
        SK(cudaGetLastError());
    }
    out->time.resize(time_cursor);
    unsigned long long bad = ~0ull;
    if (seg_cursor) {
        SK(cudaMemcpy(out->time.data(), d_time.p, out->time.size() * 8, cudaMemcpyDeviceToHost));
        SK(cudaMemcpy(&bad, d_bad.p, sizeof(bad), cudaMemcpyDeviceToHost));
        out->gather_ms = ev_g.ms();
    }
    if (bad != ~0ull) {
        uint32_t s = 0;
        while (s + 1 < n_sats && sat_seg_off[s + 1] <= bad) ++s;
        throw std::invalid_argument("A non-finite value was found in the trajectory at index " + std::to_string(s));
    }
    for (uint32_t s = 0; s < n_sats; ++s)
        if (out->traj_off[2 * s + 1]) {
            const double te = out->time[out->time_off[s] + out->traj_off[2 * s + 1]];
            out->maxT = std::max(out->maxT, te);
        }
    return out.release();
}

void free_sgp4_pj(sgp4_pj_out *p) { delete p; }

void sgp4_propagate(const gpe_host *g, uint64_t n, const double *tsince, uint64_t n_t, double *out, int32_t *err)
{
    if (n == 0 || n_t == 0) return;
    std::vector<double> keep_t;
    const double *ht = tsince;
    {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, tsince) == cudaSuccess && pa.type == cudaMemoryTypeDevice) {
            keep_t.resize(n_t);
            SK(cudaMemcpy(keep_t.data(), tsince, n_t * 8, cudaMemcpyDeviceToHost));
            ht = keep_t.data();
        }
        cudaGetLastError();
    }
    for (uint64_t k = 0; k < n_t; ++k)
        if (!std::isfinite(ht[k]))
            throw std::invalid_argument("A non-finite propagation time was passed to mzb_sgp4_propagate()");
    std::vector<job> jobs(n);
    for (uint64_t i = 0; i < n; ++i) {
        job &J = jobs[i];
        J.n0 = g[i].n0;
        J.e0 = g[i].e0;
        J.i0 = g[i].i0;
        J.node0 = g[i].node0;
        J.omega0 = g[i].omega0;
        J.m0 = g[i].m0;
        J.bstar = g[i].bstar;
        J.epoch1950 = dfl_sub(dfl_norm(g[i].epoch_jd1, g[i].epoch_jd2), dfl{2433281.5, 0.0}).hi;
    }
    devbuf<job> d_jobs(n);
    devbuf<double> d_t(n_t), d_out(n * n_t * 6);
    devbuf<int> d_err(n * n_t);
    SK(cudaMemcpy(d_jobs.p, jobs.data(), n * sizeof(job), cudaMemcpyHostToDevice));
    SK(cudaMemcpy(d_t.p, tsince, n_t * 8, cudaMemcpyDefault));
    k_sgp4_propagate<<<148 * 8, 128>>>(d_jobs.p, n, d_t.p, n_t, d_out.p, d_err.p);
    SK(cudaGetLastError());
    SK(cudaMemcpy(out, d_out.p, n * n_t * 6 * 8, cudaMemcpyDefault));
    SK(cudaMemcpy(err, d_err.p, n * n_t * 4, cudaMemcpyDefault));
}

} // namespace sgp4pj
} // namespace mzb
