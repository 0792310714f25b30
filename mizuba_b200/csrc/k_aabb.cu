// Stage 1 and 2 of a conjunction step: per-object AABBs (Cargo-Shisha
// enclosures of the segment polynomials, rounded outward to float) with the
// step's global box, then 64-bit Morton codes of the box centres.
//
// Reference: mizuba/detect_conjunctions_aabbs.cpp:64-398 and
// mizuba/detect_conjunctions_morton.cpp:70-175.
#include <algorithm>
#include <utility>

#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

// mizuba layout [gseg][k][7] -> working layout [gseg][7][row_ld(op1)], so
// that one variable's coefficients are contiguous and 16-byte aligned (the
// padding entry of odd orders + 1 is zero).  The lowest segment holding a
// non-finite coefficient is recorded in *bad_seg (the polyjectory
// constructor's data check, polyjectory.cpp:558-569, done on the copy the
// upload makes anyway).
__global__ void k_relayout(const double *__restrict__ src, double *__restrict__ dst, uint64_t n_seg, int op1,
                           unsigned long long *bad_seg)
{
    const uint64_t ld = uint64_t(row_ld(op1));
    const uint64_t per_dst = ld * 7, per_src = uint64_t(op1) * 7;
    const uint64_t total = n_seg * per_dst;
    for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < total; g += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t seg = g / per_dst, r = g % per_dst;
        const uint64_t v = r / ld, k = r % ld;
        const double x = (k < uint64_t(op1)) ? src[seg * per_src + k * 7 + v] : 0.0;
        if (!isfinite(x)) atomicMin(bad_seg, (unsigned long long)seg);
        dst[g] = x;
    }
}

// Polyjectory upload straight from device-accessible (pinned) host memory,
// one time chunk at a time, into the working layout of k_relayout.  Chunk
// [t_lo, t_hi) takes every object's segments whose start time lies in it
// (the first chunk also the earlier ones, the last chunk the later ones), so
// the chunks partition the segments and a conjunction step needs only the
// chunks that start before its end.  One warp per object: its segments are
// contiguous in the host buffer, read by consecutive lanes.
constexpr int UPLOAD_ILP = 16;

__global__ void __launch_bounds__(256) k_upload_chunk(const double *__restrict__ src, double *__restrict__ dst,
                                                      const uint64_t *__restrict__ seg_off,
                                                      const uint64_t *__restrict__ time_off,
                                                      const uint32_t *__restrict__ nseg,
                                                      const double *__restrict__ time, uint64_t n_objs, int op1,
                                                      double t_lo, double t_hi, bool first, bool last,
                                                      unsigned long long *bad_seg)
{
    const uint64_t warp = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t ld = uint32_t(row_ld(op1)), per_dst = ld * 7, per_src = uint32_t(op1) * 7;
    for (uint64_t i = warp; i < n_objs; i += nwarps) {
        const uint32_t ns = nseg[i];
        if (ns == 0) continue;
        const double *t = time + time_off[i];
        // First segment whose start time is >= x.
        auto first_at = [&](double x) {
            uint32_t lo = 0, hi = ns;
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo) / 2;
                if (t[mid] < x) lo = mid + 1;
                else hi = mid;
            }
            return lo;
        };
        const uint32_t a = first ? 0u : first_at(t_lo), b = last ? ns : first_at(t_hi);
        if (a >= b) continue;
        const uint64_t s0 = seg_off[i] + a;
        const double *sp = src + s0 * per_src;
        double *dp = dst + s0 * per_dst;
        const uint32_t n_el = (b - a) * per_src;
        auto put = [&](uint32_t e, double x) {
            const uint32_t sg = e / per_src, r = e % per_src;
            if (!isfinite(x)) atomicMin(bad_seg, (unsigned long long)(s0 + sg));
            dp[uint64_t(sg) * per_dst + (r % 7) * ld + r / 7] = x;
        };
        // 16-byte host reads (two coefficients per lane and read): an
        // element of odd address first, then pairs, then an odd last one.
        const uint32_t lead = (reinterpret_cast<uintptr_t>(sp) & 15u) ? 1u : 0u;
        const uint32_t n_pairs = (n_el - lead) / 2;
        if (lane == 0 && lead) put(0, sp[0]);
        if (lane == 0 && ((n_el - lead) & 1u)) put(n_el - 1, sp[n_el - 1]);
        const double2 *sp2 = reinterpret_cast<const double2 *>(sp + lead);
        // UPLOAD_ILP independent host reads in flight per lane before their
        // stores: the copy is bound by the bytes in flight over the link
        // (its latency grows while the outputs stream back over it), not by
        // the number of threads.
        for (uint32_t p0 = lane; p0 < n_pairs; p0 += 32 * UPLOAD_ILP) {
            double2 v[UPLOAD_ILP];
#pragma unroll
            for (int u = 0; u < UPLOAD_ILP; ++u) {
                const uint32_t q = p0 + 32 * u;
                v[u] = (q < n_pairs) ? sp2[q] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < UPLOAD_ILP; ++u) {
                const uint32_t q = p0 + 32 * u;
                if (q < n_pairs) {
                    put(lead + 2 * q, v[u].x);
                    put(lead + 2 * q + 1, v[u].y);
                }
            }
        }
        for (uint32_t e = lane; e < (b - a) * 7 * (ld - uint32_t(op1)); e += 32) // zero padding of odd orders + 1
            dp[uint64_t(e / 7) * per_dst + (e % 7) * ld + uint32_t(op1)] = 0.0;
    }
}

void launch_upload_chunk(const double *src, double *dst, const uint64_t *seg_off, const uint64_t *time_off,
                         const uint32_t *nseg, const double *time, uint64_t n_objs, int op1, double t_lo,
                         double t_hi, bool first, bool last, unsigned long long *bad_seg, cudaStream_t stream)
{
    // Few CTAs: the copy is bound by the host link (16 16-byte reads in
    // flight per lane), and an SM holding an upload CTA cannot also take a
    // one-pass BVH CTA or a pair of sort CTAs (each needs the SM's whole
    // register file) while the earlier chunks' steps are screened.  On the
    // day's end-to-end call (10 chunks, 48-step batches), measured on one
    // box: 16 CTAs 62.2 ms, 24 60.9, 32 60.1; on another, 32 62.5, 48 64.8,
    // 64 65.9, 96 67.9.
    k_upload_chunk<<<32, 256, 0, stream>>>(src, dst, seg_off, time_off, nseg, time, n_objs, op1, t_lo, t_hi,
                                                first, last, bad_seg);
}

// Staged upload (mzb_pj_create_async): host threads pack the segments of one
// time chunk of the polyjectory into pieces that the copy engine moves into a
// device staging buffer; each piece is a header (run count, data offset in
// bytes, then the runs) followed by the runs' coefficients in mizuba's
// layout.  A run is a range of consecutive segments of one object.  One warp
// per run relays the coefficients into the working layout of k_relayout and
// records the lowest non-finite segment.
__global__ void __launch_bounds__(256) k_relayout_runs(const char *__restrict__ piece, double *__restrict__ dst,
                                                       int op1, unsigned long long *bad_seg)
{
    const uint64_t n_runs = reinterpret_cast<const uint64_t *>(piece)[0];
    const uint64_t data_off = reinterpret_cast<const uint64_t *>(piece)[1];
    const stage_run *runs = reinterpret_cast<const stage_run *>(piece + 16);
    const double *data = reinterpret_cast<const double *>(piece + data_off);
    const uint64_t warp = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t ld = uint32_t(row_ld(op1)), per_dst = ld * 7, per_src = uint32_t(op1) * 7;
    for (uint64_t r = warp; r < n_runs; r += nwarps) {
        const stage_run run = runs[r];
        const double *sp = data + uint64_t(run.src_seg) * per_src;
        double *dp = dst + run.dst_seg * per_dst;
        const uint64_t n_el = uint64_t(run.n_seg) * per_src;
        for (uint64_t e = lane; e < n_el; e += 32) {
            const double x = sp[e];
            const uint64_t sg = e / per_src, rr = e % per_src;
            if (!isfinite(x)) atomicMin(bad_seg, (unsigned long long)(run.dst_seg + sg));
            dp[sg * per_dst + (rr % 7) * ld + rr / 7] = x;
        }
        for (uint64_t e = lane; e < uint64_t(run.n_seg) * 7 * (ld - uint32_t(op1)); e += 32) // pad of odd orders + 1
            dp[(e / 7) * per_dst + (e % 7) * ld + uint32_t(op1)] = 0.0;
    }
}

void launch_relayout_runs(const char *piece, uint64_t n_runs, double *coef, int op1, unsigned long long *bad_seg,
                          cudaStream_t stream)
{
    if (n_runs == 0) return;
    const uint64_t blocks = std::min<uint64_t>((n_runs + 7) / 8, 148 * 4);
    k_relayout_runs<<<unsigned(blocks), 256, 0, stream>>>(piece, coef, op1, bad_seg);
}

// Cargo-Shisha box of one segment over [h_lb, h_ub] for x, y, z and r, widened
// by the conjunction radius and rounded outward to float (aabbs.cpp:146-231),
// folded into (lb, ub) with std::min / std::max semantics.
template <int OP1>
__device__ __forceinline__ void segment_box(const double *__restrict__ cf, double h_lb, double h_ub, double radius,
                                            uint32_t obj, float *lb, float *ub, dev_status *st)
{
#pragma unroll 1
    for (int d = 0; d < 4; ++d) {
        const int v = (d == 3) ? 6 : d;
        double c[OP1], tr[OP1];
        load_row<OP1>(cf + v * row_ld(OP1), c);
        translate<OP1>(c, h_lb, tr);
        double mn, mx;
        cs_from_translated<OP1>(tr, h_ub - h_lb, mn, mx);
        mn = mn - radius;
        mx = mx + radius;
        const float fl = next_down(__double2float_rn(mn));
        const float fu = next_up(__double2float_rn(mx));
        if (!isfinite(fl)) set_error(st, ERR_AABB_LB, obj, 0, fl, 0);
        if (!isfinite(fu)) set_error(st, ERR_AABB_UB, obj, 0, fu, 0);
        lb[d] = fmin_ref(lb[d], fl);
        ub[d] = fmax_ref(ub[d], fu);
    }
}

// Pass 1, one thread per (step, object): the first overlapping segment
// (aabbs.cpp:64-252).  Objects with further overlapping segments in the step
// are queued for pass 2, so that warps here do uniform work.
template <int OP1>
__global__ void __launch_bounds__(128) k_aabb(dev_pj pj, const double2 *__restrict__ cd_bounds, uint32_t s_first,
                                              uint32_t n_batch, double radius, float *__restrict__ aabbs,
                                              uint2 *__restrict__ more, unsigned long long *more_count,
                                              uint2 *__restrict__ srange, dev_status *st)
{
    const uint64_t N = pj.n_objs;
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const bool active = gid < N * n_batch;
    const uint32_t b = active ? uint32_t(gid / N) : 0;
    const uint64_t i = active ? gid % N : 0;
    float lb[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    float ub[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    bool queue = false;
    if (active) {
        const double2 cbe = cd_bounds[s_first + b];
        const double cb = cbe.x, ce = cbe.y;
        const uint32_t ns = pj.nseg[i];
        uint2 rng = make_uint2(0, 0); // empty: no segment overlaps the step
        if (ns > 0) {
            const double *t = pj.time + pj.time_off[i];
            if (!(t[0] >= ce || t[ns] <= cb)) {
                uint32_t tb, te;
                step_range(t, ns, cb, ce, tb, te);
                rng = make_uint2(tb, te);
                if (tb != te) {
                    const uint32_t it = tb;
                    const double s0 = t[it - 1];
                    const double ev_lb = (cb < s0) ? s0 : cb;       // std::max(cb, s0)
                    const double ev_ub = (t[it] < ce) ? t[it] : ce; // std::min(ce, t[it])
                    segment_box<OP1>(coef_row<OP1>(pj, pj.seg_off[i] + it - 1, 0), ev_lb - s0, ev_ub - s0,
                                     radius, uint32_t(i), lb, ub, st);
                    queue = te - tb > 1;
                }
            }
        }
        float4 *o = reinterpret_cast<float4 *>(aabbs + ((uint64_t(s_first) + b) * (N + 1) + i) * 8);
        o[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
        o[1] = make_float4(ub[0], ub[1], ub[2], ub[3]);
        srange[uint64_t(b) * N + i] = rng;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, queue);
    if (queue) {
        const unsigned lane = threadIdx.x & 31;
        const int leader = __ffs(mask) - 1;
        unsigned long long base = 0;
        if (int(lane) == leader) base = atomicAdd(more_count, (unsigned long long)__popc(mask));
        base = __shfl_sync(mask, base, leader);
        unsigned lt;
        asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
        more[base + __popc(mask & lt)] = make_uint2(b, uint32_t(i));
    }
}

// Pass 2: the remaining overlapping segments of the queued objects, in time
// order, folded into the boxes written by pass 1 (persistent grid).
template <int OP1>
__global__ void __launch_bounds__(128) k_aabb_more(dev_pj pj, const double2 *__restrict__ cd_bounds,
                                                   uint32_t s_first, double radius, float *__restrict__ aabbs,
                                                   const uint2 *__restrict__ more,
                                                   const unsigned long long *more_count, dev_status *st)
{
    const uint64_t N = pj.n_objs;
    const uint64_t n = *more_count;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
        const uint2 e = more[k];
        const uint32_t b = e.x, i = e.y;
        const double2 cbe = cd_bounds[s_first + b];
        const double cb = cbe.x, ce = cbe.y;
        const uint32_t ns = pj.nseg[i];
        const double *t = pj.time + pj.time_off[i];
        uint32_t tb, te;
        step_range(t, ns, cb, ce, tb, te);
        float4 *o = reinterpret_cast<float4 *>(aabbs + ((uint64_t(s_first) + b) * (N + 1) + i) * 8);
        const float4 l0 = o[0], u0 = o[1];
        float lb[4] = {l0.x, l0.y, l0.z, l0.w}, ub[4] = {u0.x, u0.y, u0.z, u0.w};
        for (uint32_t it = tb + 1; it != te; ++it) {
            const double s0 = t[it - 1];
            const double ev_lb = (cb < s0) ? s0 : cb;
            const double ev_ub = (t[it] < ce) ? t[it] : ce;
            segment_box<OP1>(coef_row<OP1>(pj, pj.seg_off[i] + it - 1, 0), ev_lb - s0, ev_ub - s0, radius, i, lb,
                             ub, st);
        }
        o[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
        o[1] = make_float4(ub[0], ub[1], ub[2], ub[3]);
    }
}

// ---------------------------------------------------------------- mixed form
//
// The same enclosure, computed with FMA-native formulations: Taylor shift by
// synthetic division (n(n+1)/2 FMAs), scaling by powers of delta, the
// binomial division replaced by a multiplication with 1/C(n, i), and the
// Bernstein difference table.  The result differs from the plain form's by
// rounding only; both are within E = (8n + 16) u P of the exact Cargo-Shisha
// bounds, where P = sum_k |c_k| (a + delta)^k bounds every intermediate
// magnitude.  Widening by 2E before the outward float rounding therefore
// yields boxes that contain the plain form's boxes, so the broad phase of the
// mixed form finds a superset of the plain form's overlapping pairs.
//
// With scr != nullptr the same pass also writes the distance screen's model
// of the portion (see screen_keeps): position and velocity at the portion
// midpoint tm = (h_lb + h_ub) / 2 (FP32, rounded to nearest), and |A| rounded
// up, where A_c = sum_k k (k - 1) |c_k| h_ub^(k-2) bounds |x_c''| on [0, h_ub].
template <int OP1>
__device__ __forceinline__ void segment_box_mixed(const double *__restrict__ cf, const double *__restrict__ inv_binom,
                                                  double h_lb, double h_ub, double radius, uint32_t obj, float *lb,
                                                  float *ub, dev_status *st, float4 *__restrict__ scr)
{
    constexpr int n = OP1 - 1;
    const double delta = h_ub - h_lb;
    const double span = h_lb + delta;
    const double tmr = (h_lb + h_ub) / 2;
    float sp[3], sv[3];
    double a2 = 0;
#pragma unroll 1
    for (int d = 0; d < 4; ++d) {
        const int v = (d == 3) ? 6 : d;
        double t[OP1];
        load_row<OP1>(cf + v * row_ld(OP1), t);
        if (scr && d < 3) {
            double p = t[n], dp = 0, acc = double(n) * (n - 1) * fabs(t[n]);
#pragma unroll
            for (int k = n - 1; k >= 0; --k) {
                dp = fma(dp, tmr, p);
                p = fma(p, tmr, t[k]);
                if (k >= 2) acc = fma(acc, h_ub, double(k) * (k - 1) * fabs(t[k]));
            }
            sp[d] = __double2float_rn(p);
            sv[d] = __double2float_rn(dp);
            a2 = fma(acc, acc, a2);
        }
        // P = sum |c_k| span^k (Horner on absolute values).
        double P = fabs(t[n]);
#pragma unroll
        for (int k = n - 1; k >= 0; --k) P = fma(P, span, fabs(t[k]));
        // Taylor shift by h_lb.
#pragma unroll
        for (int i = 0; i < n; ++i)
#pragma unroll
            for (int k = n - 1; k >= i; --k) t[k] = fma(h_lb, t[k + 1], t[k]);
        double dp = 1.0;
#pragma unroll
        for (int i = 0; i < OP1; ++i) {
            t[i] = (t[i] * dp) * __ldg(inv_binom + i);
            dp *= delta;
        }
        double mn = t[0], mx = t[0];
#pragma unroll
        for (int k = 1; k < OP1; ++k) {
#pragma unroll
            for (int j = 0; j + k < OP1; ++j) t[j] = t[j] + t[j + 1];
            mn = fmin(mn, t[0]);
            mx = fmax(mx, t[0]);
        }
        const double E = 2.0 * (8.0 * n + 16.0) * 1.1102230246251565e-16 * P * 1.0001;
        mn = (mn - E) - radius;
        mx = (mx + E) + radius;
        const float fl = next_down(__double2float_rd(mn));
        const float fu = next_up(__double2float_ru(mx));
        if (!isfinite(fl)) set_error(st, ERR_AABB_LB, obj, 0, fl, 0);
        if (!isfinite(fu)) set_error(st, ERR_AABB_UB, obj, 0, fu, 0);
        lb[d] = fmin_ref(lb[d], fl);
        ub[d] = fmax_ref(ub[d], fu);
    }
    if (scr) {
        // sqrt is correctly rounded; the factor covers its half ulp and the
        // accumulation before the upward conversion.
        const float a = __double2float_ru(sqrt(a2) * (1.0 + 1e-12));
        scr[0] = make_float4(sp[0], sp[1], sp[2], sv[0]);
        scr[1] = make_float4(sv[1], sv[2], a, 0.f);
    }
}

template <int OP1>
__global__ void __launch_bounds__(128) k_aabb_mixed(dev_pj pj, const double2 *__restrict__ cd_bounds,
                                                    const double *__restrict__ inv_binom, uint32_t s_first,
                                                    uint32_t n_batch, double radius, float *__restrict__ aabbs,
                                                    uint2 *__restrict__ more, unsigned long long *more_count,
                                                    float4 *__restrict__ scr, uint2 *__restrict__ srange,
                                                    dev_status *st)
{
    const uint64_t N = pj.n_objs;
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const bool active = gid < N * n_batch;
    const uint32_t b = active ? uint32_t(gid / N) : 0;
    const uint64_t i = active ? gid % N : 0;
    float lb[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    float ub[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    bool queue = false;
    if (active) {
        const double2 cbe = cd_bounds[s_first + b];
        const double cb = cbe.x, ce = cbe.y;
        const uint32_t ns = pj.nseg[i];
        uint2 rng = make_uint2(0, 0); // empty: no segment overlaps the step
        if (ns > 0) {
            const double *t = pj.time + pj.time_off[i];
            if (!(t[0] >= ce || t[ns] <= cb)) {
                uint32_t tb, te;
                step_range(t, ns, cb, ce, tb, te);
                rng = make_uint2(tb, te);
                if (tb != te) {
                    const uint32_t it = tb;
                    const double s0 = t[it - 1];
                    const double ev_lb = (cb < s0) ? s0 : cb;
                    const double ev_ub = (t[it] < ce) ? t[it] : ce;
                    segment_box_mixed<OP1>(coef_row<OP1>(pj, pj.seg_off[i] + it - 1, 0), inv_binom, ev_lb - s0,
                                           ev_ub - s0, radius, uint32_t(i), lb, ub, st,
                                           scr ? scr + (uint64_t(b) * N + i) * 4 : nullptr);
                    queue = te - tb > 1;
                }
            }
        }
        float4 *o = reinterpret_cast<float4 *>(aabbs + ((uint64_t(s_first) + b) * (N + 1) + i) * 8);
        o[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
        o[1] = make_float4(ub[0], ub[1], ub[2], ub[3]);
        srange[uint64_t(b) * N + i] = rng;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, queue);
    if (queue) {
        const unsigned lane = threadIdx.x & 31;
        const int leader = __ffs(mask) - 1;
        unsigned long long base = 0;
        if (int(lane) == leader) base = atomicAdd(more_count, (unsigned long long)__popc(mask));
        base = __shfl_sync(mask, base, leader);
        unsigned lt;
        asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
        more[base + __popc(mask & lt)] = make_uint2(b, uint32_t(i));
    }
}

template <int OP1>
__global__ void __launch_bounds__(128) k_aabb_mixed_more(dev_pj pj, const double2 *__restrict__ cd_bounds,
                                                         const double *__restrict__ inv_binom, uint32_t s_first,
                                                         double radius, float *__restrict__ aabbs,
                                                         const uint2 *__restrict__ more,
                                                         const unsigned long long *more_count,
                                                         float4 *__restrict__ scr, dev_status *st)
{
    const uint64_t N = pj.n_objs;
    const uint64_t n = *more_count;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
        const uint2 e = more[k];
        const uint32_t b = e.x, i = e.y;
        const double2 cbe = cd_bounds[s_first + b];
        const double cb = cbe.x, ce = cbe.y;
        const double *t = pj.time + pj.time_off[i];
        uint32_t tb, te;
        step_range(t, pj.nseg[i], cb, ce, tb, te);
        float4 *o = reinterpret_cast<float4 *>(aabbs + ((uint64_t(s_first) + b) * (N + 1) + i) * 8);
        const float4 l0 = o[0], u0 = o[1];
        float lb[4] = {l0.x, l0.y, l0.z, l0.w}, ub[4] = {u0.x, u0.y, u0.z, u0.w};
        for (uint32_t it = tb + 1; it != te; ++it) {
            const double s0 = t[it - 1];
            const double ev_lb = (cb < s0) ? s0 : cb;
            const double ev_ub = (t[it] < ce) ? t[it] : ce;
            // The step's second segment has the second model slot; later
            // ones (short segments) are screened from their coefficients.
            segment_box_mixed<OP1>(coef_row<OP1>(pj, pj.seg_off[i] + it - 1, 0), inv_binom, ev_lb - s0,
                                   ev_ub - s0, radius, i, lb, ub, st,
                                   (it == tb + 1 && scr) ? scr + (uint64_t(b) * N + i) * 4 + 2 : nullptr);
        }
        o[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
        o[1] = make_float4(ub[0], ub[1], ub[2], ub[3]);
    }
}

// Global box of each step (aabbs.cpp:353-391): one block per step reduces
// the object boxes with ordered-integer min / max.
__global__ void k_gbox(uint32_t s_first, uint64_t N, float *__restrict__ aabbs, dev_status *st)
{
    __shared__ uint32_t red[8][32];
    const uint64_t s = uint64_t(s_first) + blockIdx.x;
    const float *base = aabbs + s * (N + 1) * 8;
    uint32_t olb[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu}, oub[4] = {0, 0, 0, 0};
    for (uint64_t i = threadIdx.x; i < N; i += blockDim.x) {
        const float4 l = reinterpret_cast<const float4 *>(base + i * 8)[0];
        const float4 u = reinterpret_cast<const float4 *>(base + i * 8)[1];
        olb[0] = min(olb[0], f2ord(l.x));
        olb[1] = min(olb[1], f2ord(l.y));
        olb[2] = min(olb[2], f2ord(l.z));
        olb[3] = min(olb[3], f2ord(l.w));
        oub[0] = max(oub[0], f2ord(u.x));
        oub[1] = max(oub[1], f2ord(u.y));
        oub[2] = max(oub[2], f2ord(u.z));
        oub[3] = max(oub[3], f2ord(u.w));
    }
#pragma unroll
    for (int d = 0; d < 4; ++d)
        for (int off = 16; off > 0; off >>= 1) {
            olb[d] = min(olb[d], __shfl_xor_sync(0xffffffffu, olb[d], off));
            oub[d] = max(oub[d], __shfl_xor_sync(0xffffffffu, oub[d], off));
        }
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0)
        for (int d = 0; d < 4; ++d) {
            red[d][warp] = olb[d];
            red[4 + d][warp] = oub[d];
        }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int r = threadIdx.x;
        uint32_t v = red[r][0];
        for (unsigned w = 1; w < nw; ++w) v = (r < 4) ? min(v, red[r][w]) : max(v, red[r][w]);
        float *row = aabbs + (s * (N + 1) + N) * 8;
        row[r] = ord2f(v);
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        const float *row = aabbs + (s * (N + 1) + N) * 8;
        const float l = row[threadIdx.x], u = row[4 + threadIdx.x];
        if (isfinite(l) && !isfinite(u - l)) set_error(st, ERR_GLOBAL_AABB, 0, 0, 0, 0);
    }
}

// 16 bits -> every 4th bit (bit k to bit 4k).
__device__ __forceinline__ uint64_t spread4(uint64_t x)
{
    x &= 0xffffull;
    x = (x | (x << 24)) & 0x000000ff000000ffull;
    x = (x | (x << 12)) & 0x000f000f000f000full;
    x = (x | (x << 6)) & 0x0303030303030303ull;
    x = (x | (x << 3)) & 0x1111111111111111ull;
    return x;
}

// disc_single_coord (morton.cpp:70-99).
__device__ __forceinline__ uint64_t disc(float x, float mn, float mx)
{
    const float isize = mx - mn;
    float rx = (x - mn) / isize;
    rx = rx >= 0.f ? rx : 0.f;
    rx *= 65536.f;
    const uint64_t v = static_cast<uint64_t>(rx);
    return v < 65535ull ? v : 65535ull;
}

// Morton codes of the box centres in the step's global box
// (morton.cpp:139-175); no-data objects get all ones.
__global__ void k_morton(const float *__restrict__ aabbs, uint32_t s_first, uint32_t n_batch, uint64_t N,
                         uint64_t *__restrict__ mcodes)
{
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (gid >= N * n_batch) return;
    const uint64_t s = s_first + gid / N, i = gid % N;
    const float4 *row = reinterpret_cast<const float4 *>(aabbs + (s * (N + 1) + i) * 8);
    const float4 *g = reinterpret_cast<const float4 *>(aabbs + (s * (N + 1) + N) * 8);
    const float4 lb = row[0], ub = row[1], gl = g[0], gu = g[1];
    uint64_t code;
    if (isfinite(lb.x)) {
        const uint64_t n0 = disc(lb.x / 2 + ub.x / 2, gl.x, gu.x);
        const uint64_t n1 = disc(lb.y / 2 + ub.y / 2, gl.y, gu.y);
        const uint64_t n2 = disc(lb.z / 2 + ub.z / 2, gl.z, gu.z);
        const uint64_t n3 = disc(lb.w / 2 + ub.w / 2, gl.w, gu.w);
        code = spread4(n0) | (spread4(n1) << 1) | (spread4(n2) << 2) | (spread4(n3) << 3);
    } else {
        code = ~0ull;
    }
    mcodes[s * N + i] = code;
}

// ------------------------------------------------------------------ launchers

void launch_relayout(const double *src, double *dst, uint64_t n_seg, int op1, unsigned long long *bad_seg,
                     cudaStream_t stream)
{
    if (n_seg == 0) return;
    k_relayout<<<148 * 8, 256, 0, stream>>>(src, dst, n_seg, op1, bad_seg);
}

template <int OP1>
static void aabb_t(const dev_pj &pj, const double2 *cdb, const double *inv_binom, uint32_t s_first, uint32_t nb,
                   double radius, float *aabbs, uint2 *more, unsigned long long *more_count, float4 *scr,
                   uint2 *srange, dev_status *st, cudaStream_t stream)
{
    const uint64_t n = pj.n_objs * nb;
    const unsigned bs = 128;
    if (inv_binom) {
        k_aabb_mixed<OP1><<<unsigned((n + bs - 1) / bs), bs, 0, stream>>>(pj, cdb, inv_binom, s_first, nb, radius,
                                                                          aabbs, more, more_count, scr, srange, st);
        k_aabb_mixed_more<OP1><<<148 * 5, bs, 0, stream>>>(pj, cdb, inv_binom, s_first, radius, aabbs, more,
                                                            more_count, scr, st);
    } else {
        k_aabb<OP1><<<unsigned((n + bs - 1) / bs), bs, 0, stream>>>(pj, cdb, s_first, nb, radius, aabbs, more,
                                                                    more_count, srange, st);
        k_aabb_more<OP1><<<148 * 4, bs, 0, stream>>>(pj, cdb, s_first, radius, aabbs, more, more_count, st);
    }
}

// inv_binom == nullptr selects the plain form; otherwise it points to
// 1 / C(order, i), i = 0..order, and selects the mixed form.
// scr (mixed form only): two 32-byte screen models per (step, object) of the
// batch, for the first and second segment overlapping the step.
// srange[b * N + i]: the segments of object i overlapping the batch's step b,
// as step_range gives them (time-point indices [tb, te); (0, 0) if none).
void launch_aabb(const dev_pj &pj, const double2 *cdb, const double *inv_binom, uint32_t s_first, uint32_t nb,
                 double radius, float *aabbs, uint2 *more, unsigned long long *more_count, float4 *scr,
                 uint2 *srange, dev_status *st, cudaStream_t stream)
{
    cudaMemsetAsync(more_count, 0, sizeof(unsigned long long), stream);
    switch (pj.op1) {
#define X(K)                                                                                                         \
    case K:                                                                                                            \
        aabb_t<K>(pj, cdb, inv_binom, s_first, nb, radius, aabbs, more, more_count, scr, srange, st, stream);         \
        break;
        MZB_FOR_EACH_OP1(X)
#undef X
    default:
        break;
    }
    k_gbox<<<nb, 512, 0, stream>>>(s_first, pj.n_objs, aabbs, st);
}

void launch_morton(const float *aabbs, uint32_t s_first, uint32_t nb, uint64_t N, uint64_t *mcodes, cudaStream_t stream)
{
    const uint64_t n = N * nb;
    k_morton<<<unsigned((n + 255) / 256), 256, 0, stream>>>(aabbs, s_first, nb, N, mcodes);
}

cudaError_t init_aabb_consts() { return upload_binom_table(); }

} // namespace mzb
