// Stage 5 of a conjunction step: narrow phase
// (mizuba/detect_conjunctions_narrow_phase.cpp:167-769).
//
// k_items: one thread per broad-phase pair walks the two objects' segment
//   boundaries (narrow.cpp:345-418) and appends every overlapping
//   sub-interval to a device queue of items.
// k_narrow: one thread per item (persistent grid pulling from that queue)
//   translates both position polynomials to the sub-interval start
//   (conjunctions_jit.cpp:68-140), evaluates them at the order+1 Chebyshev
//   nodes, interpolates the squared distance with Bjorck-Pereyra
//   (narrow.cpp:95-152, poly_utils.cpp:467-535) and encloses it with
//   Cargo-Shisha (narrow.cpp:502-517).  Sub-intervals whose enclosure does not
//   reach below threshold^2 are dropped; the others go to a device queue with
//   their distance polynomial.
// k_roots: one thread per queued sub-interval (persistent grid pulling from the
//   device queue) runs the minimum search on the
//   derivative (poly_utils.cpp:272-460): fast exclusion, Descartes/VCA
//   isolation with the reference's LIFO working list (in global scratch,
//   at most 251 entries as in the reference), TOMS 748 polishing, the
//   threshold test on the interpolant, the trajectory-boundary minima
//   (narrow.cpp:629-714) and the state vectors at TCA (narrow.cpp:542-575).
// k_conj_*: per-step ordering by (tca, record) (narrow.cpp:751-757).
#include "block.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

// ------------------------------------------------------------- k_narrow

__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; } // std::max(a, b)
__device__ __forceinline__ double dmin_ref(double a, double b) { return (b < a) ? b : a; } // std::min(a, b)

__device__ __forceinline__ void warp_add(unsigned long long *ctr, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr, v);
}

// Warp-aggregated append of one slot per active lane; returns this lane's
// slot.
__device__ __forceinline__ unsigned long long warp_append(unsigned long long *counter, bool want)
{
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (!want) return 0;
    const unsigned lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (int(lane) == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & lanemask_lt());
}

// One thread per broad-phase pair: the merge walk over both objects' segment
// boundaries (narrow.cpp:345-418) appends every overlapping sub-interval to
// the item queue.  Items are re-sorted per step at the end, so queue order is
// free.  With increasing time points every live iteration advances at least
// one cursor, so a walk ends within (ei - it_i) + (ej - it_j) iterations; a
// walk that reaches that bound (time points out of order on the device)
// stops and reports ERR_NP_INTERVAL instead of spinning.
__global__ void __launch_bounds__(128) k_items(const dev_pj pj, const double2 *__restrict__ cd_bounds,
                                               uint32_t s_first, uint32_t nb, const uint2 *__restrict__ pairs,
                                               const uint64_t *__restrict__ step_off,
                                               const uint2 *__restrict__ srange, np_item *__restrict__ items,
                                               uint64_t cap, unsigned long long *item_count,
                                               unsigned long long *counters, dev_status *st)
{
    const uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const uint64_t n_pairs = step_off[nb];
    bool active = p < n_pairs;
    uint32_t b = 0, i = 0, j = 0, it_i = 0, it_j = 0, ei = 0, ej = 0;
    const double *ti = nullptr, *tj = nullptr;
    double cb = 0, ce = 0;
    if (active) {
        uint32_t lo = 0, hi = nb;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (step_off[mid] <= p) lo = mid;
            else hi = mid;
        }
        b = lo;
        const double2 cbe = cd_bounds[s_first + b];
        cb = cbe.x;
        ce = cbe.y;
        const uint2 pr = pairs[p];
        i = pr.x;
        j = pr.y;
        ti = pj.time + pj.time_off[i];
        tj = pj.time + pj.time_off[j];
        // The segment ranges found by the AABB pass (step_range over the
        // same step bounds).
        const uint2 ri = srange[uint64_t(b) * pj.n_objs + i], rj = srange[uint64_t(b) * pj.n_objs + j];
        it_i = ri.x, ei = ri.y;
        it_j = rj.x, ej = rj.y;
    }
    unsigned long long n_cand = 0;
    uint32_t budget = (ei - it_i) + (ej - it_j);
    // Warp-synchronous loop: every lane iterates until all lanes are done.
    for (;;) {
        bool live = active && it_i != ei && it_j != ej;
        if (live && budget == 0) {
            set_error(st, ERR_NP_INTERVAL, i, j, 0.0, 0.0);
            live = false;
            active = false;
        }
        if (!__any_sync(0xffffffffu, live)) break;
        bool emit = false;
        double ti_e = 0, tj_e = 0;
        if (live) {
            const double si = ti[it_i - 1], sj = tj[it_j - 1];
            ti_e = ti[it_i];
            tj_e = tj[it_j];
            const double lb_i = dmax_ref(cb, si), ub_i = dmin_ref(ce, ti_e);
            const double lb_j = dmax_ref(cb, sj), ub_j = dmin_ref(ce, tj_e);
            emit = ub_i > lb_j && lb_i < ub_j;
        }
        const unsigned long long slot = warp_append(item_count, emit);
        if (emit) {
            ++n_cand;
            if (slot < cap) items[slot] = np_item{i, j, b, it_i, it_j, 0};
        }
        if (live) {
            it_i += (ti_e <= tj_e);
            it_j += (tj_e <= ti_e);
            --budget;
        }
    }
    warp_add(counters + 0, n_cand);
}

// One thread per item (persistent grid over the device-side item count).
// The per-item arithmetic is the reference's, operation for operation.
template <int OP1>
__global__ void __launch_bounds__(128, 3) k_narrow(dev_pj pj, cheb_nodes cheb, const double2 *__restrict__ cd_bounds,
                                                   uint32_t s_first, const np_item *__restrict__ items,
                                                   const unsigned long long *item_count, uint64_t item_cap,
                                                   double thresh2, root_item *__restrict__ rq, uint64_t rq_cap,
                                                   unsigned long long *rq_count, unsigned long long *counters,
                                                   dev_status *st)
{
    const uint64_t n_items = min(*item_count, (unsigned long long)item_cap);
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    unsigned long long n_pruned = 0;
    for (uint64_t base = blockIdx.x * uint64_t(blockDim.x); base < n_items; base += stride) {
        const uint64_t q_idx = base + threadIdx.x;
        const bool active = q_idx < n_items;
        bool push = false;
        np_item it{};
        double lb_rf = 0, rf_int = 0, di = 0, dj = 0;
        uint32_t flags = 0;
        uint64_t gsi = 0, gsj = 0;
        double f[OP1];
        if (active) {
            it = items[q_idx];
            const double2 cbe = cd_bounds[s_first + it.b];
            const double cb = cbe.x, ce = cbe.y;
            const double *ti = pj.time + pj.time_off[it.i];
            const double *tj = pj.time + pj.time_off[it.j];
            const double si = ti[it.it_i - 1], sj = tj[it.it_j - 1];
            const double ti_e = ti[it.it_i], tj_e = tj[it.it_j];
            const double lb_i = dmax_ref(cb, si), ub_i = dmin_ref(ce, ti_e);
            const double lb_j = dmax_ref(cb, sj), ub_j = dmin_ref(ce, tj_e);
            lb_rf = dmax_ref(lb_i, lb_j);
            const double ub_rf = dmin_ref(ub_i, ub_j);
            di = lb_rf - si;
            dj = lb_rf - sj;
            rf_int = ub_rf - lb_rf;
            if (!isfinite(di) || !isfinite(dj) || !isfinite(rf_int) || di < 0 || dj < 0 || rf_int < 0) {
                set_error(st, ERR_NP_INTERVAL, it.i, it.j, 0, 0);
            } else {
                gsi = pj.seg_off[it.i] + it.it_i - 1;
                gsj = pj.seg_off[it.j] + it.it_j - 1;
                const double *ci_base = coef_row<OP1>(pj, gsi, 0);
                const double *cj_base = coef_row<OP1>(pj, gsj, 0);
#pragma unroll 1
                for (int c = 0; c < 3; ++c) {
                    double cf[OP1], tr[OP1], vi[OP1];
                    load_row<OP1>(ci_base + c * row_ld(OP1), cf);
                    if (di != 0) translate<OP1>(cf, di, tr);
                    else
#pragma unroll
                        for (int k = 0; k < OP1; ++k) tr[k] = cf[k];
#pragma unroll
                    for (int m = 0; m < OP1; ++m) vi[m] = horner<OP1>(tr, cheb.v[m] * rf_int);
                    load_row<OP1>(cj_base + c * row_ld(OP1), cf);
                    if (dj != 0) translate<OP1>(cf, dj, tr);
                    else
#pragma unroll
                        for (int k = 0; k < OP1; ++k) tr[k] = cf[k];
#pragma unroll
                    for (int m = 0; m < OP1; ++m) {
                        const double d = vi[m] - horner<OP1>(tr, cheb.v[m] * rf_int);
                        f[m] = (c == 0) ? d * d : f[m] + d * d;
                    }
                }
                // Bjorck-Pereyra on the ascending nodes.
#pragma unroll
                for (int k = 0; k < OP1 - 1; ++k)
#pragma unroll
                    for (int jj = OP1 - 1; jj > k; --jj)
                        f[jj] = (f[jj] - f[jj - 1]) / (cheb.v[jj] * rf_int - cheb.v[jj - k - 1] * rf_int);
#pragma unroll
                for (int k = OP1 - 2; k >= 0; --k)
#pragma unroll
                    for (int jj = k; jj < OP1 - 1; ++jj) f[jj] = f[jj] - (cheb.v[k] * rf_int) * f[jj + 1];
                double e[OP1];
#pragma unroll
                for (int k = 0; k < OP1; ++k) e[k] = f[k];
                double emin, emax;
                cs_from_translated<OP1>(e, rf_int, emin, emax);
                if (!isfinite(emin) || !isfinite(emax)) {
                    set_error(st, ERR_NP_NONFINITE, it.i, it.j, 0, 0);
                } else if (emin < thresh2) {
                    push = true;
                    const uint32_t nsi = pj.nseg[it.i], nsj = pj.nseg[it.j];
                    if ((it.it_i == nsi && ti_e == ub_rf) || (it.it_j == nsj && tj_e == ub_rf)) flags |= 1u;
                    if ((it.it_i == 1 && lb_rf == ti[0]) || (it.it_j == 1 && lb_rf == tj[0])) flags |= 2u;
                } else {
                    ++n_pruned;
                }
            }
        }
        const unsigned long long slot = warp_append(rq_count, push);
        if (push && slot < rq_cap) {
            root_item &q = rq[slot];
            q.i = it.i;
            q.j = it.j;
            q.step = it.b;
            q.flags = flags;
            q.lb_rf = lb_rf;
            q.rf_int = rf_int;
            q.di = di;
            q.dj = dj;
            q.seg_i = gsi;
            q.seg_j = gsj;
#pragma unroll
            for (int k = 0; k < OP1; ++k) q.ptd2[k] = f[k];
        }
    }
    warp_add(counters + 1, n_pruned);
}

// ------------------------------------------------------------ mixed form
//
// A conservative FMA-native prefilter in front of k_narrow.  For each item
// the dist^2 interpolant is formed cheaply: each object's original segment
// polynomial is evaluated by FMA Horner at the shifted nodes delta + alpha_m
// (mathematically the translated polynomial at alpha_m, so the explicit
// translation is skipped), the squared distances are interpolated in the
// normalised time s = t / rf_int on the fixed nodes c_m with Bjorck-Pereyra
// using precomputed reciprocals 1 / (c_j - c_{j-k-1}), and the Cargo-Shisha
// enclosure over s in [0, 1] needs no powers of rf_int.  An item is dropped
// only if this enclosure clears threshold^2 by a margin (1e-8 of the largest
// sampled dist^2 plus 1e-12 of threshold^2) that covers the difference from
// the reference formulation; the survivors are queued and recomputed by
// k_narrow with the reference formulation, so every conjunction record comes
// from the reference arithmetic.  It runs on the items that the distance screen
// leaves.
//
// tab layout (doubles): [0, OP1) nodes c_m; [OP1, OP1 + OP1^2) inverse node
// differences, row k; then OP1 inverse binomials 1 / C(n, i).
template <int OP1>
__global__ void __launch_bounds__(128, 3) k_narrow_mixed(dev_pj pj, const double *__restrict__ tab,
                                                         const double2 *__restrict__ cd_bounds, uint32_t s_first,
                                                         const np_item *__restrict__ items,
                                                         const unsigned long long *item_count, uint64_t item_cap,
                                                         double thresh2, np_item *__restrict__ surv,
                                                         uint64_t surv_cap, unsigned long long *surv_count,
                                                         unsigned long long *counters, dev_status *st)
{
    constexpr int n = OP1 - 1;
    const double *cheb = tab;
    const double *inv_dd = tab + OP1;
    const double *inv_binom = tab + OP1 + OP1 * OP1;
    const uint64_t n_items = min(*item_count, (unsigned long long)item_cap);
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    unsigned long long n_pruned = 0;
    for (uint64_t base = blockIdx.x * uint64_t(blockDim.x); base < n_items; base += stride) {
        const uint64_t q_idx = base + threadIdx.x;
        const bool active = q_idx < n_items;
        bool push = false;
        np_item it{};
        double lb_rf = 0, rf_int = 0, di = 0, dj = 0;
        uint64_t gsi = 0, gsj = 0;
        double f[OP1];
        if (active) {
            it = items[q_idx];
            const double2 cbe = cd_bounds[s_first + it.b];
            const double cb = cbe.x, ce = cbe.y;
            const double *ti = pj.time + pj.time_off[it.i];
            const double *tj = pj.time + pj.time_off[it.j];
            const double si = ti[it.it_i - 1], sj = tj[it.it_j - 1];
            const double ti_e = ti[it.it_i], tj_e = tj[it.it_j];
            const double lb_i = dmax_ref(cb, si), ub_i = dmin_ref(ce, ti_e);
            const double lb_j = dmax_ref(cb, sj), ub_j = dmin_ref(ce, tj_e);
            lb_rf = dmax_ref(lb_i, lb_j);
            const double ub_rf = dmin_ref(ub_i, ub_j);
            (void)ti_e;
            (void)tj_e;
            di = lb_rf - si;
            dj = lb_rf - sj;
            rf_int = ub_rf - lb_rf;
            if (!isfinite(di) || !isfinite(dj) || !isfinite(rf_int) || di < 0 || dj < 0 || rf_int < 0) {
                push = true; // the exact recheck reports the invalid interval
            } else {
                gsi = pj.seg_off[it.i] + it.it_i - 1;
                gsj = pj.seg_off[it.j] + it.it_j - 1;
                const double *ci_base = coef_row<OP1>(pj, gsi, 0);
                const double *cj_base = coef_row<OP1>(pj, gsj, 0);
#pragma unroll 1
                for (int c = 0; c < 3; ++c) {
                    double ci[OP1], cj[OP1];
                    load_row<OP1>(ci_base + c * row_ld(OP1), ci);
                    load_row<OP1>(cj_base + c * row_ld(OP1), cj);
#pragma unroll
                    for (int m = 0; m < OP1; ++m) {
                        const double am = __ldg(cheb + m) * rf_int;
                        const double tii = di + am, tjj = dj + am;
                        double xi = ci[n], xj = cj[n];
#pragma unroll
                        for (int k = n - 1; k >= 0; --k) {
                            xi = fma(xi, tii, ci[k]);
                            xj = fma(xj, tjj, cj[k]);
                        }
                        const double d = xi - xj;
                        f[m] = (c == 0) ? d * d : fma(d, d, f[m]);
                    }
                }
                double fmax_s = f[0];
#pragma unroll
                for (int m = 1; m < OP1; ++m) fmax_s = fmax(fmax_s, f[m]);
                // Bjorck-Pereyra on the normalised nodes.
#pragma unroll
                for (int k = 0; k < n; ++k)
#pragma unroll
                    for (int jj = n; jj > k; --jj) f[jj] = (f[jj] - f[jj - 1]) * __ldg(inv_dd + k * OP1 + jj);
#pragma unroll
                for (int k = n - 1; k >= 0; --k) {
                    const double ck = __ldg(cheb + k);
#pragma unroll
                    for (int jj = k; jj < n; ++jj) f[jj] = fma(-ck, f[jj + 1], f[jj]);
                }
                // Cargo-Shisha over s in [0, 1].
                double e[OP1];
#pragma unroll
                for (int k = 0; k < OP1; ++k) e[k] = f[k] * __ldg(inv_binom + k);
                double emin = e[0], emax = e[0];
#pragma unroll
                for (int k = 1; k < OP1; ++k) {
#pragma unroll
                    for (int jj = 0; jj + k < OP1; ++jj) e[jj] = e[jj] + e[jj + 1];
                    emin = fmin(emin, e[0]);
                    emax = fmax(emax, e[0]);
                }
                const double margin = 1e-8 * fmax_s + 1e-12 * thresh2;
                if (!(emin >= thresh2 + margin)) {
                    // kept (non-finite values are left to the exact recheck,
                    // which reports them as the reference does)
                    push = true;
                } else {
                    ++n_pruned;
                }
            }
        }
        const unsigned long long slot = warp_append(surv_count, push);
        if (push && slot < surv_cap) surv[slot] = it;
    }
    warp_add(counters + 1, n_pruned);
}

// Screen ahead of the mixed prefilter: a rigorous lower bound on the
// distance over the item's sub-interval from linear models of both objects.
// For each object, on the portion of its segment inside the step, Taylor's
// theorem gives x(tm + s) = x(tm) + x'(tm) s + R(s) with |R(s)| <= |A| s^2 / 2,
// A_c = sum_k k (k - 1) |c_k| t_max^(k-2) bounding |x_c''| (t_max the portion
// end in the segment's own time).  The relative linear model over the item
// is D0 + Dv s, |s| <= h (half the sub-interval), so
//   min |dr(t)| >= min_{|s| <= h} |D0 + Dv s| - (|A_i| si^2 + |A_j| sj^2) / 2,
// si, sj the largest distance of the item from each model point; the first
// term is the closest approach of a straight line, in closed form.  Items
// whose bound clears the threshold (relative slack 1e-6) cannot hold a
// conjunction: they are dropped and counted as pruned by the distance
// check; the rest go on to k_narrow_mixed, compacted so its warps stay full.
//
// The models come from the mixed AABB pass (32 bytes each, FP32: position,
// velocity at the portion midpoint, |A| rounded up) for the first and second
// segments of each object in the step; their FP32 rounding is added to the
// margin.  Items on a later segment (objects with segments shorter than half
// a step) build the models here from the coefficients, at the item midpoint.
// The distance screen of one item (above): false when the item cannot hold
// a conjunction (then *pruned is set).
template <int OP1>
__device__ __forceinline__ bool screen_keeps(const dev_pj &pj, const double2 *__restrict__ cd_bounds,
                                             uint32_t s_first, const np_item &it, double thresh,
                                             const float4 *__restrict__ scr, bool &pruned)
{
    constexpr int n = OP1 - 1;
    const uint64_t N = pj.n_objs;
    bool push = false;
    const double2 cbe = cd_bounds[s_first + it.b];
    const double cb = cbe.x, ce = cbe.y;
    const double *ti = pj.time + pj.time_off[it.i];
    const double *tj = pj.time + pj.time_off[it.j];
    const double si = ti[it.it_i - 1], sj = tj[it.it_j - 1];
    const double ti_e = ti[it.it_i], tj_e = tj[it.it_j];
    const double lb_i = dmax_ref(cb, si), ub_i = dmin_ref(ce, ti_e);
    const double lb_j = dmax_ref(cb, sj), ub_j = dmin_ref(ce, tj_e);
    const double lb_rf = dmax_ref(lb_i, lb_j), ub_rf = dmin_ref(ub_i, ub_j);
    const double di = lb_rf - si, dj = lb_rf - sj, rf_int = ub_rf - lb_rf;
    push = true;
    if (isfinite(di) && isfinite(dj) && isfinite(rf_int) && di >= 0 && dj >= 0 && rf_int >= 0) {
        const double h = rf_int / 2;
        // Slot of each object's model: 0 for the step's first
        // overlapping segment, 1 for the second, none after that.
        int slot_i = -1, slot_j = -1;
        if (scr) {
            if (it.it_i == 1 || si <= cb) slot_i = 0;
            else if (it.it_i == 2 || ti[it.it_i - 2] <= cb) slot_i = 1;
            if (it.it_j == 1 || sj <= cb) slot_j = 0;
            else if (it.it_j == 2 || tj[it.it_j - 2] <= cb) slot_j = 1;
        }
        double P[2][3], V[2][3], A[2], off[2], emod = 0;
        if (slot_i >= 0 && slot_j >= 0) {
            const float4 *m[2] = {scr + (uint64_t(it.b) * N + it.i) * 4 + 2 * slot_i,
                                  scr + (uint64_t(it.b) * N + it.j) * 4 + 2 * slot_j};
            const double tm[2] = {((lb_i - si) + (ub_i - si)) / 2, ((lb_j - sj) + (ub_j - sj)) / 2};
            const double dd[2] = {di, dj};
#pragma unroll
            for (int o = 0; o < 2; ++o) {
                const float4 a = m[o][0], b = m[o][1];
                P[o][0] = a.x, P[o][1] = a.y, P[o][2] = a.z;
                V[o][0] = a.w, V[o][1] = b.x, V[o][2] = b.y;
                A[o] = b.z;
                off[o] = dd[o] + h - tm[o]; // item centre from the model point
                // FP32 storage: |fl(x) - x| <= 2^-24 |x| for each value.
                emod += 1.1920928955078125e-07
                        * (sqrt(P[o][0] * P[o][0] + P[o][1] * P[o][1] + P[o][2] * P[o][2])
                           + sqrt(V[o][0] * V[o][0] + V[o][1] * V[o][1] + V[o][2] * V[o][2])
                                 * (fabs(off[o]) + h));
            }
        } else {
            // Models at the item midpoint from the coefficients.
            const double tmi = di + h, tmj = dj + h, tei = di + rf_int, tej = dj + rf_int;
            const double *ci_base = coef_row<OP1>(pj, pj.seg_off[it.i] + it.it_i - 1, 0);
            const double *cj_base = coef_row<OP1>(pj, pj.seg_off[it.j] + it.it_j - 1, 0);
            double ai2 = 0, aj2 = 0;
#pragma unroll 1
            for (int c = 0; c < 3; ++c) {
                double ci[OP1], cj[OP1];
                load_row<OP1>(ci_base + c * row_ld(OP1), ci);
                load_row<OP1>(cj_base + c * row_ld(OP1), cj);
                double pi = ci[n], pj_ = cj[n], vi = 0, vj = 0;
                double ai = double(n) * (n - 1) * fabs(ci[n]), aj = double(n) * (n - 1) * fabs(cj[n]);
#pragma unroll
                for (int k = n - 1; k >= 0; --k) {
                    vi = fma(vi, tmi, pi);
                    vj = fma(vj, tmj, pj_);
                    pi = fma(pi, tmi, ci[k]);
                    pj_ = fma(pj_, tmj, cj[k]);
                    if (k >= 2) {
                        ai = fma(ai, tei, double(k) * (k - 1) * fabs(ci[k]));
                        aj = fma(aj, tej, double(k) * (k - 1) * fabs(cj[k]));
                    }
                }
                P[0][c] = pi, P[1][c] = pj_, V[0][c] = vi, V[1][c] = vj;
                ai2 = fma(ai, ai, ai2);
                aj2 = fma(aj, aj, aj2);
            }
            A[0] = sqrt(ai2) * (1.0 + 1e-12);
            A[1] = sqrt(aj2) * (1.0 + 1e-12);
            off[0] = off[1] = 0;
        }
        double d0[3], dv[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            d0[c] = fma(V[0][c], off[0], P[0][c]) - fma(V[1][c], off[1], P[1][c]);
            dv[c] = V[0][c] - V[1][c];
        }
        const double vv = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
        const double rv = d0[0] * dv[0] + d0[1] * dv[1] + d0[2] * dv[2];
        double sst = vv > 0 ? -rv / vv : 0;
        sst = fmin(fmax(sst, -h), h);
        const double e0 = fma(dv[0], sst, d0[0]), e1 = fma(dv[1], sst, d0[1]), e2 = fma(dv[2], sst, d0[2]);
        const double dlin = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        const double s_i = fabs(off[0]) + h, s_j = fabs(off[1]) + h;
        const double R = 0.5 * (A[0] * s_i * s_i + A[1] * s_j * s_j);
        const double slack =
            1e-6 * (thresh + sqrt(d0[0] * d0[0] + d0[1] * d0[1] + d0[2] * d0[2]) + sqrt(vv) * h + R) + emod;
        if (isfinite(dlin) && isfinite(R) && isfinite(slack) && dlin - R > thresh + slack) {
            push = false;
            pruned = true;
        }
    }
    return push;
}

// The mixed form's merge walk (k_items) with the distance screen inside: each item of the
// merge walk is screened as it is found and only the items the screen keeps
// are appended (to the prefilter's queue), so the day's 6.4 M items are
// never written out and read back.  Counters: every item (counter 0, and
// *item_count), the pruned ones (counter 1).
template <int OP1>
__global__ void __launch_bounds__(128, 6) k_items_screen(const dev_pj pj, const double2 *__restrict__ cd_bounds,
                                                         uint32_t s_first, uint32_t nb, const uint2 *__restrict__ pairs,
                                                         const uint64_t *__restrict__ step_off,
                                                         const uint2 *__restrict__ srange, double thresh,
                                                         const float4 *__restrict__ scr, np_item *__restrict__ cand,
                                                         uint64_t cand_cap, unsigned long long *cand_count,
                                                         unsigned long long *item_count,
                                                         unsigned long long *counters, dev_status *st)
{
    const uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const uint64_t n_pairs = step_off[nb];
    bool active = p < n_pairs;
    uint32_t b = 0, i = 0, j = 0, it_i = 0, it_j = 0, ei = 0, ej = 0;
    const double *ti = nullptr, *tj = nullptr;
    double cb = 0, ce = 0;
    if (active) {
        uint32_t lo = 0, hi = nb;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (step_off[mid] <= p) lo = mid;
            else hi = mid;
        }
        b = lo;
        const double2 cbe = cd_bounds[s_first + b];
        cb = cbe.x;
        ce = cbe.y;
        const uint2 pr = pairs[p];
        i = pr.x;
        j = pr.y;
        ti = pj.time + pj.time_off[i];
        tj = pj.time + pj.time_off[j];
        const uint2 ri = srange[uint64_t(b) * pj.n_objs + i], rj = srange[uint64_t(b) * pj.n_objs + j];
        it_i = ri.x, ei = ri.y;
        it_j = rj.x, ej = rj.y;
    }
    unsigned long long n_items = 0, n_pruned = 0;
    uint32_t budget = (ei - it_i) + (ej - it_j);
    // Warp-synchronous loop as in k_items (bounded the same way).
    for (;;) {
        bool live = active && it_i != ei && it_j != ej;
        if (live && budget == 0) {
            set_error(st, ERR_NP_INTERVAL, i, j, 0.0, 0.0);
            live = false;
            active = false;
        }
        if (!__any_sync(0xffffffffu, live)) break;
        bool emit = false;
        double ti_e = 0, tj_e = 0;
        if (live) {
            const double si = ti[it_i - 1], sj = tj[it_j - 1];
            ti_e = ti[it_i];
            tj_e = tj[it_j];
            const double lb_i = dmax_ref(cb, si), ub_i = dmin_ref(ce, ti_e);
            const double lb_j = dmax_ref(cb, sj), ub_j = dmin_ref(ce, tj_e);
            emit = ub_i > lb_j && lb_i < ub_j;
        }
        bool keep = false;
        const np_item it{i, j, b, it_i, it_j, 0};
        if (emit) {
            ++n_items;
            bool pruned = false;
            keep = screen_keeps<OP1>(pj, cd_bounds, s_first, it, thresh, scr, pruned);
            n_pruned += pruned;
        }
        const unsigned long long slot = warp_append(cand_count, keep);
        if (keep && slot < cand_cap) cand[slot] = it;
        if (live) {
            it_i += (ti_e <= tj_e);
            it_j += (tj_e <= ti_e);
            --budget;
        }
    }
    warp_add(counters + 0, n_items);
    warp_add(item_count, n_items);
    warp_add(counters + 1, n_pruned);
}

template <int OP1>
static void items_screen_t(const dev_pj &pj, const double2 *cdb, uint32_t s_first, uint32_t nb, const uint2 *pairs,
                           const uint64_t *step_off, const uint2 *srange, uint64_t n_pairs, double thresh,
                           const float4 *scr, np_item *cand, uint64_t cand_cap, unsigned long long *cand_count,
                           unsigned long long *item_count, unsigned long long *counters, dev_status *st,
                           cudaStream_t stream)
{
    const unsigned bs = 128;
    const unsigned g = unsigned((n_pairs + bs - 1) / bs);
    if (g == 0) return;
    k_items_screen<OP1><<<g, bs, 0, stream>>>(pj, cdb, s_first, nb, pairs, step_off, srange, thresh, scr, cand,
                                               cand_cap, cand_count, item_count, counters, st);
}

void launch_items_screen(const dev_pj &pj, const double2 *cdb, uint32_t s_first, uint32_t nb, const uint2 *pairs,
                         const uint64_t *step_off, const uint2 *srange, uint64_t n_pairs, double thresh,
                         const float4 *scr, np_item *cand, uint64_t cand_cap, unsigned long long *cand_count,
                         unsigned long long *item_count, unsigned long long *counters, dev_status *st,
                         cudaStream_t stream)
{
    switch (pj.op1) {
#define X(K)                                                                                                         \
    case K:                                                                                                            \
        items_screen_t<K>(pj, cdb, s_first, nb, pairs, step_off, srange, n_pairs, thresh, scr, cand, cand_cap,        \
                          cand_count, item_count, counters, st, stream);                                               \
        break;
        MZB_FOR_EACH_OP1(X)
#undef X
    default:
        break;
    }
}

// -------------------------------------------------------------- k_roots

constexpr int WL_CAP = 251; // the reference throws once its list exceeds 250

__device__ __forceinline__ int sgn(double v) { return (0. < v) - (v < 0.); }

__device__ __forceinline__ bool tol_ok(double a, double b)
{
    return fabs(a - b) <= (4 * 2.220446049250313e-16) * fmin(fabs(a), fabs(b));
}

__device__ double secant_step(double a, double b, double fa, double fb)
{
    const double e5 = 5 * 2.220446049250313e-16;
    const double c = a - (fa / (fb - fa)) * (b - a);
    if (c <= a + fabs(a) * e5 || c >= b - fabs(b) * e5) return (a + b) / 2;
    return c;
}

__device__ double guarded_div(double num, double den, double fallback)
{
    if (fabs(den) < 1 && fabs(den * 1.7976931348623157e308) <= fabs(num)) return fallback;
    return num / den;
}

__device__ double newton_quadratic(double a, double b, double d, double fa, double fb, double fd, int k)
{
    const double big = 1.7976931348623157e308;
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

__device__ double inverse_cubic(double a, double b, double d, double e, double fa, double fb, double fd, double fe)
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

__device__ bool near_equal_values(double fa, double fb, double fd, double fe)
{
    const double m = 2.2250738585072014e-308 * 32;
    return fabs(fa - fb) < m || fabs(fa - fd) < m || fabs(fa - fe) < m || fabs(fb - fd) < m || fabs(fb - fe) < m
           || fabs(fd - fe) < m;
}

constexpr int MAX_ROOTS = 2 * MAX_OP1;

// ---- Compile-time-order building blocks of the minimum search.

// Taylor shift by 1 (heyoka poly_translate_1): out_I = sum_{k >= I} C(k, I) in_k,
// pairwise summed in k order.
template <int OP1, int I>
__device__ __forceinline__ double shift1_coef(const double (&in)[OP1])
{
    constexpr int M = OP1 - I;
    double t[M];
#pragma unroll
    for (int k = 0; k < M; ++k) t[k] = c_binom[I + k][I] * in[I + k];
    return pw<M>::reduce(t, add_op{});
}
template <int OP1, int... I>
__device__ __forceinline__ void shift1_impl(const double (&in)[OP1], double (&out)[OP1],
                                            std::integer_sequence<int, I...>)
{
    ((out[I] = shift1_coef<OP1, I>(in)), ...);
}
template <int OP1>
__device__ __forceinline__ void shift1(const double (&in)[OP1], double (&out)[OP1])
{
    shift1_impl<OP1>(in, out, std::make_integer_sequence<int, OP1>{});
}

// Descartes sign changes of the coefficients, zeros skipped.
template <int OP1>
__device__ __forceinline__ int sign_changes_t(const double (&c)[OP1])
{
    int cnt = 0, prev = 0;
#pragma unroll
    for (int k = 0; k < OP1; ++k) {
        const int s = sgn(c[k]);
        cnt += (s != 0 && prev != 0 && s != prev);
        prev = (s != 0) ? s : prev;
    }
    return cnt;
}

// First derivative of a (poly_utils.cpp poly_eval_1).
template <int OP1>
__device__ __forceinline__ double poly_eval_1_t(const double (&a)[OP1], double x)
{
    constexpr int n = OP1 - 1;
    double r = a[n] * n;
#pragma unroll
    for (int i = 1; i < n; ++i) r = a[n - i] * (n - i) + r * x;
    return r;
}

// Fast exclusion: interval Horner over [0, h]; true = no root there.
template <int OP1>
__device__ __forceinline__ bool fex_excludes_t(const double (&p)[OP1], double h)
{
    constexpr int n = OP1 - 1;
    double lo = p[n], hi = p[n];
#pragma unroll
    for (int o = 1; o <= n; ++o) {
        const double a = lo * h, b = hi * h;
        const double plo = fmin(0., fmin(a, b)), phi = fmax(0., fmax(a, b));
        lo = p[n - o] + plo;
        hi = p[n - o] + phi;
    }
    return lo > 0 || hi < 0;
}

// ---- TOMS 748 (Alefeld, Potra, Shi 1995, Algorithm 4.2) on horner(p, .).
template <int OP1>
struct toms_t {
    const double (&p)[OP1];
    int evals;
    __device__ double f(double x)
    {
        ++evals;
        return horner<OP1>(p, x);
    }
};

// Shrink [a, b] around c (paper: BRACKT), keeping c off the endpoints.
template <typename ST>
__device__ void bracket_at_t(ST &st, double &a, double &b, double c, double &fa, double &fb, double &d, double &fd)
{
    const double t = 2 * 2.220446049250313e-16;
    if ((b - a) < 2 * t * a) c = a + (b - a) / 2;
    else if (c <= a + fabs(a) * t) c = a + fabs(a) * t;
    else if (c >= b - fabs(b) * t) c = b - fabs(b) * t;
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

// Returns the flag (0 ok, 33 = EDOM for a non-bracketing interval, -1 for an
// exhausted budget of 100 evaluations) and the root in *root.
template <int OP1>
__device__ int toms748_t(const double (&p)[OP1], double lo, double hi, double *root)
{
    constexpr int budget = 100;
    toms_t<OP1> st{p, 0};
    double a = lo, b = hi;
    double fa = st.f(a), fb = st.f(b);
    if (!(a < b)) return 33;
    if (tol_ok(a, b) || fa == 0 || fb == 0) {
        if (fa == 0) b = a;
        else if (fb == 0) a = b;
        *root = a / 2 + b / 2;
        return 0;
    }
    if (sgn(fa) * sgn(fb) > 0) return 33;
    double d = 0, fd = 0, e = 1e5, fe = 1e5;
#define MZB_DONE() (st.evals >= budget || fa == 0 || tol_ok(a, b))
    bracket_at_t(st, a, b, secant_step(a, b, fa, fb), fa, fb, d, fd);
    if (!MZB_DONE()) {
        const double c = newton_quadratic(a, b, d, fa, fb, fd, 2);
        e = d;
        fe = fd;
        bracket_at_t(st, a, b, c, fa, fb, d, fd);
    }
    while (!MZB_DONE()) {
        const double a0 = a, b0 = b;
        double c = near_equal_values(fa, fb, fd, fe) ? newton_quadratic(a, b, d, fa, fb, fd, 2)
                                                     : inverse_cubic(a, b, d, e, fa, fb, fd, fe);
        e = d;
        fe = fd;
        bracket_at_t(st, a, b, c, fa, fb, d, fd);
        if (MZB_DONE()) break;
        c = near_equal_values(fa, fb, fd, fe) ? newton_quadratic(a, b, d, fa, fb, fd, 3)
                                              : inverse_cubic(a, b, d, e, fa, fb, fd, fe);
        bracket_at_t(st, a, b, c, fa, fb, d, fd);
        if (MZB_DONE()) break;
        double u, fu;
        if (fabs(fa) < fabs(fb)) u = a, fu = fa;
        else u = b, fu = fb;
        c = u - 2 * (fu / (fb - fa)) * (b - a);
        if (fabs(c - u) > (b - a) / 2) c = a + (b - a) / 2;
        e = d;
        fe = fd;
        bracket_at_t(st, a, b, c, fa, fb, d, fd);
        if (MZB_DONE()) break;
        if ((b - a) < 0.5 * (b0 - a0)) continue;
        e = d;
        fe = fd;
        bracket_at_t(st, a, b, a + (b - a) / 2, fa, fb, d, fd);
    }
#undef MZB_DONE
    if (fa == 0) b = a;
    else if (fb == 0) a = b;
    *root = a / 2 + b / 2;
    if (st.evals >= budget && !(fa == 0 || tol_ok(a, b))) return -1;
    return 0;
}

// State vectors at tm for one object's segment translated by delta
// (add_conjunction, narrow.cpp:542-575).
template <int OP1>
__device__ void states_at_t(const dev_pj &pj, uint64_t gseg, double delta, double tm, double *r, double *v)
{
#pragma unroll 1
    for (int var = 0; var < 6; ++var) {
        double c[OP1], t[OP1];
        load_row<OP1>(coef_row<OP1>(pj, gseg, var), c);
        double x;
        if (delta != 0) {
            translate<OP1>(c, delta, t);
            x = horner<OP1>(t, tm);
        } else {
            x = horner<OP1>(c, tm);
        }
        if (var < 3) r[var] = x;
        else v[var - 3] = x;
    }
}

// wl_cap: working-list entries available per thread.  With wl_cap < 251 an
// item whose list would outgrow it is deferred to `retry` untouched and is
// run again with the full 251-entry list by a second, smaller launch.  The
// item count is read on the device (persistent grid).
template <int OP1>
__global__ void __launch_bounds__(128) k_roots(dev_pj pj, const root_item *__restrict__ rq,
                                               const unsigned long long *rq_count, uint64_t rq_cap,
                                               const uint32_t *__restrict__ item_list,
                                               const unsigned long long *item_list_count, double thresh2,
                                               double *__restrict__ wl_scratch, int wl_cap,
                                               uint32_t *__restrict__ retry, unsigned long long *retry_count,
                                               conj_out *__restrict__ cq, uint64_t cq_cap,
                                               unsigned long long *cq_count, unsigned long long *counters,
                                               dev_status *st)
{
    constexpr int n = OP1 - 1;
    constexpr int ENT = OP1 + 2; // (lb, ub, q[0..n])
    const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const uint64_t nthreads = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t n_items = item_list ? *item_list_count : min(*rq_count, (unsigned long long)rq_cap);
    double *wl = wl_scratch + tid * uint64_t(wl_cap) * ENT;
    unsigned long long n_roots = 0, n_fex = 0, n_noroot = 0, n_minima = 0, n_disc = 0;
    for (uint64_t it = tid; it < n_items; it += nthreads) {
        const uint32_t item = item_list ? item_list[it] : uint32_t(it);
        const root_item &q = rq[item];
        const double rf_int = q.rf_int;
        double d2p[OP1];
#pragma unroll
        for (int k = 0; k < n; ++k) d2p[k] = (k + 1u) * q.ptd2[k + 1];
        d2p[n] = 0;
        double roots[MAX_ROOTS];
        int nroots = 0;
        bool failed = false, deferred = false;
        auto add_root = [&](double root) {
            if (!isfinite(root)) {
                set_error(st, ERR_ROOT_NONFINITE, q.i, q.j, root, 0);
                failed = true;
                return;
            }
            const double der = poly_eval_1_t<OP1>(d2p, root);
            if (!isfinite(der)) {
                set_error(st, ERR_ROOT_DER, q.i, q.j, root, der);
                failed = true;
                return;
            }
            if (sgn(der) == 1) {
                if (nroots < MAX_ROOTS) roots[nroots++] = root;
                else {
                    set_error(st, ERR_ISOLATION, q.i, q.j, MAX_ROOTS, 0);
                    failed = true;
                }
            }
        };
        const bool fex = fex_excludes_t<OP1>(d2p, rf_int);
        if (!fex) {
            // VCA isolation with a LIFO working list of (lb, ub, q[0..n]).
            {
                double fct = 1;
                wl[0] = 0;
                wl[1] = 1;
#pragma unroll
                for (int k = 0; k < OP1; ++k) {
                    wl[2 + k] = fct * d2p[k];
                    fct *= rf_int;
                }
            }
            int wsz = 1;
            double isol_lb[OP1 + 1], isol_ub[OP1 + 1];
            int nisol = 0;
            do {
                --wsz;
                const double *ent = wl + uint64_t(wsz) * ENT;
                const double lb = ent[0], ub = ent[1];
                double cur[OP1], r1[OP1], r2[OP1];
#pragma unroll
                for (int k = 0; k < OP1; ++k) cur[k] = ent[2 + k];
                bool tail_finite = true;
#pragma unroll
                for (int k = 1; k < OP1; ++k) tail_finite = tail_finite && isfinite(cur[k]);
                if (cur[0] == 0 && tail_finite) add_root(lb * rf_int);
#pragma unroll
                for (int k = 0; k < OP1; ++k) r1[k] = cur[n - k];
                shift1<OP1>(r1, r2);
                const int nsc = sign_changes_t<OP1>(r2);
                if (nsc == 1) {
                    if (nisol < OP1 + 1) {
                        isol_lb[nisol] = lb;
                        isol_ub[nisol] = ub;
                    }
                    ++nisol;
                } else if (nsc > 1) {
                    if (wsz + 2 > wl_cap) {
                        if (wl_cap < WL_CAP) {
                            const unsigned long long r = atomicAdd(retry_count, 1ull);
                            retry[r] = item;
                            deferred = true;
                        } else {
                            set_error(st, ERR_ISOLATION, q.i, q.j, wsz + 2, nisol);
                            failed = true;
                        }
                        break;
                    }
                    double L[OP1], R[OP1];
                    double fct = 1;
#pragma unroll
                    for (int k = 0; k < OP1; ++k) {
                        L[n - k] = fct * cur[n - k];
                        fct *= 2;
                    }
                    shift1<OP1>(L, R);
                    const double mid = lb / 2 + ub / 2;
                    double *El = wl + uint64_t(wsz) * ENT;
                    double *Er = El + ENT;
                    El[0] = lb;
                    El[1] = mid;
                    Er[0] = mid;
                    Er[1] = ub;
#pragma unroll
                    for (int k = 0; k < OP1; ++k) {
                        El[2 + k] = L[k];
                        Er[2 + k] = R[k];
                    }
                    wsz += 2;
                }
                if (wsz > 250 || nisol > n) {
                    set_error(st, ERR_ISOLATION, q.i, q.j, wsz, nisol);
                    failed = true;
                    break;
                }
            } while (wsz > 0 && !failed);
            if (deferred) continue;
            if (!failed && nisol > 0) {
                double sp[OP1];
                double fct = 1;
#pragma unroll
                for (int k = 0; k < OP1; ++k) {
                    sp[k] = fct * d2p[k];
                    fct *= rf_int;
                }
                for (int r = 0; r < nisol && !failed; ++r) {
                    double lb = isol_lb[r], ub = isol_ub[r];
                    if (isfinite(lb) && isfinite(ub) && ub > lb) ub = nextafter(ub, lb);
                    double root = 0;
                    const int flag = toms748_t<OP1>(sp, lb, ub, &root);
                    if (flag == -1) {
                        set_error(st, ERR_TOMS_ITER, q.i, q.j, 0, 0);
                        failed = true;
                    } else if (flag != 0) {
                        set_error(st, ERR_TOMS_ERRNO, q.i, q.j, flag, 0);
                        failed = true;
                    } else {
                        add_root(root * rf_int);
                    }
                }
            }
        }
        if (failed) continue;
        ++n_roots;
        n_fex += fex;
        n_noroot += (nroots == 0);
        n_minima += nroots;

        double ptd2[OP1];
#pragma unroll
        for (int k = 0; k < OP1; ++k) ptd2[k] = q.ptd2[k];
        auto emit = [&](double tm) {
            conj_out o;
            o.c.i = q.i;
            o.c.j = q.j;
            states_at_t<OP1>(pj, q.seg_i, q.di, tm, o.c.ri, o.c.vi);
            states_at_t<OP1>(pj, q.seg_j, q.dj, tm, o.c.rj, o.c.vj);
            const double dx = o.c.ri[0] - o.c.rj[0], dy = o.c.ri[1] - o.c.rj[1], dz = o.c.ri[2] - o.c.rj[2];
            o.c.dca = sqrt((dx * dx) + (dy * dy) + (dz * dz));
            o.c.tca = q.lb_rf + tm;
            o.step = q.step;
            const unsigned long long slot = atomicAdd(cq_count, 1ull);
            if (slot < cq_cap) cq[slot] = o;
        };
        for (int r = 0; r < nroots; ++r) {
            const double tm = roots[r];
            const double d2 = horner<OP1>(ptd2, tm);
            if (!isfinite(d2)) {
                set_error(st, ERR_CONJ_D2, q.i, q.j, d2, 0);
                continue;
            }
            if (d2 < thresh2) emit(tm);
            else ++n_disc;
        }
        if (q.flags & 1u) {
            const double tm = nextafter(rf_int, -1.);
            const double dv = horner<OP1>(d2p, tm);
            if (!isfinite(dv)) set_error(st, ERR_UB_DER, q.i, q.j, dv, 0);
            else if (dv < 0) {
                const double d2 = horner<OP1>(ptd2, tm);
                if (!isfinite(d2)) set_error(st, ERR_UB_D2, q.i, q.j, d2, 0);
                else if (d2 < thresh2) emit(tm);
            }
        }
        if (q.flags & 2u) {
            const double dv = horner<OP1>(d2p, 0.);
            if (!isfinite(dv)) set_error(st, ERR_LB_DER, q.i, q.j, dv, 0);
            else if (dv > 0) {
                const double d2 = horner<OP1>(ptd2, 0.);
                if (!isfinite(d2)) set_error(st, ERR_LB_D2, q.i, q.j, d2, 0);
                else if (d2 < thresh2) emit(0.);
            }
        }
    }
    warp_add(counters + 2, n_roots);
    warp_add(counters + 3, n_fex);
    warp_add(counters + 4, n_noroot);
    warp_add(counters + 5, n_minima);
    warp_add(counters + 6, n_disc);
}

// ------------------------------------------------------------- conj order

__device__ __forceinline__ bool conj_less(const conj_rec &a, const conj_rec &b)
{
    if (a.tca != b.tca) return a.tca < b.tca;
    if (a.i != b.i) return a.i < b.i;
    if (a.j != b.j) return a.j < b.j;
    if (a.dca != b.dca) return a.dca < b.dca;
    const double *pa[4] = {a.ri, a.vi, a.rj, a.vj}, *pb[4] = {b.ri, b.vi, b.rj, b.vj};
    for (int v = 0; v < 4; ++v)
        for (int k = 0; k < 3; ++k)
            if (pa[v][k] != pb[v][k]) return pa[v][k] < pb[v][k];
    return false;
}

__global__ void k_conj_count(const conj_out *cq, uint64_t n, uint32_t *cnt)
{
    const uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (g < n) atomicAdd(cnt + cq[g].step, 1u);
}

// One block: exclusive scan of the per-step counts (also resets cursors).
__global__ void k_conj_offsets(const uint32_t *cnt, uint32_t nb, uint32_t *off, uint32_t *cursor)
{
    __shared__ uint32_t sm[33];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += blockDim.x) {
        const uint32_t k = base + threadIdx.x;
        const uint32_t v = k < nb ? cnt[k] : 0;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(v, sm, &tot);
        if (k < nb) {
            off[k] = carry + ex;
            cursor[k] = 0;
        }
        carry += tot;
    }
    if (threadIdx.x == 0) off[nb] = carry;
}

__global__ void k_conj_group(const conj_out *cq, uint64_t n, const uint32_t *off, uint32_t *cursor, conj_out *grp)
{
    const uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (g >= n) return;
    const uint32_t s = cq[g].step;
    const uint32_t pos = atomicAdd(cursor + s, 1u);
    grp[off[s] + pos] = cq[g];
}

// Steps with at most CONJ_SORT_MAX conjunctions are ordered by one block
// each (k_conj_sort_step); larger groups by k_conj_rank.
constexpr uint32_t CONJ_SORT_MAX = 16384;
constexpr size_t CONJ_SORT_SMEM = size_t(CONJ_SORT_MAX) * (sizeof(uint64_t) + sizeof(uint32_t));

// Order-preserving integer image of a double (the TCAs are finite).
__device__ __forceinline__ uint64_t tca_key(double x)
{
    const uint64_t b = uint64_t(__double_as_longlong(x));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// One block per step: bitonic sort of the step's (TCA, slot) keys in shared
// memory, then each run of equal TCAs ordered by the whole record
// (detect_conjunctions_narrow_phase.cpp:751-757: by tca, ties by the
// record's three-way comparison), then the records written in order.
__global__ void __launch_bounds__(1024) k_conj_sort_step(const conj_out *__restrict__ grp,
                                                         const uint32_t *__restrict__ off, conj_rec *__restrict__ out)
{
    extern __shared__ __align__(16) unsigned char conj_smem[];
    uint64_t *key = reinterpret_cast<uint64_t *>(conj_smem);
    uint32_t *idx = reinterpret_cast<uint32_t *>(key + CONJ_SORT_MAX);
    const uint32_t s = blockIdx.x;
    const uint32_t b0 = off[s], n = off[s + 1] - b0;
    if (n == 0 || n > CONJ_SORT_MAX) return;
    uint32_t P = 1;
    while (P < n) P <<= 1;
    for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) {
        key[k] = k < n ? tca_key(grp[b0 + k].c.tca) : ~0ull;
        idx[k] = k < n ? k : 0xffffffffu;
    }
    __syncthreads();
    for (uint32_t size = 2; size <= P; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const uint32_t i = 2 * t - (t & (stride - 1)), j = i + stride;
                const bool asc = (i & size) == 0;
                const uint64_t ki = key[i], kj = key[j];
                const uint32_t ii = idx[i], ij = idx[j];
                const bool gt = ki > kj || (ki == kj && ii > ij);
                if (gt == asc) {
                    key[i] = kj;
                    key[j] = ki;
                    idx[i] = ij;
                    idx[j] = ii;
                }
            }
            __syncthreads();
        }
    // Runs of equal TCA (rare, short): insertion sort by the whole record.
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        if ((k == 0 || key[k - 1] != key[k]) && k + 1 < n && key[k + 1] == key[k]) {
            uint32_t e = k + 1;
            while (e < n && key[e] == key[k]) ++e;
            for (uint32_t a = k + 1; a < e; ++a)
                for (uint32_t c = a; c > k && conj_less(grp[b0 + idx[c]].c, grp[b0 + idx[c - 1]].c); --c) {
                    const uint32_t t2 = idx[c];
                    idx[c] = idx[c - 1];
                    idx[c - 1] = t2;
                }
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) out[b0 + k] = grp[b0 + idx[k]].c;
}

// Rank within the step's group (groups larger than CONJ_SORT_MAX); equal
// records are ordered by group slot.
__global__ void k_conj_rank(const conj_out *grp, uint64_t n, const uint32_t *off, conj_rec *out)
{
    const uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (g >= n) return;
    const conj_out me = grp[g];
    const uint32_t b0 = off[me.step], b1 = off[me.step + 1];
    if (b1 - b0 <= CONJ_SORT_MAX) return;
    uint32_t rank = 0;
    for (uint32_t k = b0; k < b1; ++k) {
        if (k == g) continue;
        const conj_rec &o = grp[k].c;
        if (conj_less(o, me.c) || (k < g && !conj_less(me.c, o))) ++rank;
    }
    out[b0 + rank] = me.c;
}

// ------------------------------------------------------------- launchers

void launch_items(const dev_pj &pj, const double2 *cdb, uint32_t s_first, uint32_t nb, const uint2 *pairs,
                  const uint64_t *step_off, const uint2 *srange, uint64_t n_pairs, np_item *items, uint64_t cap,
                  unsigned long long *item_count, unsigned long long *counters, dev_status *st, cudaStream_t stream)
{
    const unsigned bs = 128;
    const unsigned g = unsigned((n_pairs + bs - 1) / bs);
    if (g == 0) return;
    k_items<<<g, bs, 0, stream>>>(pj, cdb, s_first, nb, pairs, step_off, srange, items, cap, item_count, counters,
                                  st);
}

template <int OP1>
static void narrow_t(const dev_pj &pj, const double2 *cdb, uint32_t s_first, const np_item *items,
                     const unsigned long long *item_count, uint64_t item_cap, double thresh2, root_item *rq,
                     uint64_t rq_cap, unsigned long long *rq_count, unsigned long long *counters, dev_status *st,
                     unsigned grid, cudaStream_t stream)
{
    k_narrow<OP1><<<grid, 128, 0, stream>>>(pj, make_cheb_nodes(OP1), cdb, s_first, items, item_count, item_cap,
                                             thresh2, rq, rq_cap, rq_count, counters, st);
}

void launch_narrow(const dev_pj &pj, const double2 *cdb, uint32_t s_first, const np_item *items,
                   const unsigned long long *item_count, uint64_t item_cap, double thresh2, root_item *rq,
                   uint64_t rq_cap, unsigned long long *rq_count, unsigned long long *counters, dev_status *st,
                   unsigned grid, cudaStream_t stream)
{
    switch (pj.op1) {
#define X(K)                                                                                                         \
    case K:                                                                                                            \
        narrow_t<K>(pj, cdb, s_first, items, item_count, item_cap, thresh2, rq, rq_cap, rq_count, counters, st, grid, \
                    stream);                                                                                           \
        break;
        MZB_FOR_EACH_OP1(X)
#undef X
    default:
        break;
    }
}

template <int OP1>
static void prefilter_t(const dev_pj &pj, const double *tab, const double2 *cdb, uint32_t s_first,
                        const np_item *items, const unsigned long long *item_count, uint64_t item_cap, double thresh2,
                        np_item *surv, uint64_t surv_cap, unsigned long long *surv_count,
                        unsigned long long *counters, dev_status *st, unsigned grid, cudaStream_t stream)
{
    k_narrow_mixed<OP1><<<grid, 128, 0, stream>>>(pj, tab, cdb, s_first, items, item_count, item_cap, thresh2, surv,
                                                   surv_cap, surv_count, counters, st);
}

void launch_narrow_prefilter(const dev_pj &pj, const double *tab, const double2 *cdb, uint32_t s_first,
                             const np_item *items, const unsigned long long *item_count, uint64_t item_cap,
                             double thresh2, np_item *surv, uint64_t surv_cap, unsigned long long *surv_count,
                             unsigned long long *counters, dev_status *st, unsigned grid, cudaStream_t stream)
{
    switch (pj.op1) {
#define X(K)                                                                                                         \
    case K:                                                                                                            \
        prefilter_t<K>(pj, tab, cdb, s_first, items, item_count, item_cap, thresh2, surv, surv_cap, surv_count,       \
                       counters, st, grid, stream);                                                                    \
        break;
        MZB_FOR_EACH_OP1(X)
#undef X
    default:
        break;
    }
}

template <int OP1>
static void roots_t(const dev_pj &pj, const root_item *rq, const unsigned long long *rq_count, uint64_t rq_cap,
                    const uint32_t *item_list, const unsigned long long *item_list_count, double thresh2,
                    double *wl_scratch, int wl_cap, unsigned grid, uint32_t *retry, unsigned long long *retry_count,
                    conj_out *cq, uint64_t cq_cap, unsigned long long *cq_count, unsigned long long *counters,
                    dev_status *st, cudaStream_t stream)
{
    k_roots<OP1><<<grid, 128, 0, stream>>>(pj, rq, rq_count, rq_cap, item_list, item_list_count, thresh2, wl_scratch,
                                            wl_cap, retry, retry_count, cq, cq_cap, cq_count, counters, st);
}

void launch_roots(const dev_pj &pj, const root_item *rq, const unsigned long long *rq_count, uint64_t rq_cap,
                  const uint32_t *item_list, const unsigned long long *item_list_count, double thresh2,
                  double *wl_scratch, int wl_cap, unsigned grid, uint32_t *retry, unsigned long long *retry_count,
                  conj_out *cq, uint64_t cq_cap, unsigned long long *cq_count, unsigned long long *counters,
                  dev_status *st, cudaStream_t stream)
{
    switch (pj.op1) {
#define X(K)                                                                                                         \
    case K:                                                                                                            \
        roots_t<K>(pj, rq, rq_count, rq_cap, item_list, item_list_count, thresh2, wl_scratch, wl_cap, grid, retry,    \
                   retry_count, cq, cq_cap, cq_count, counters, st, stream);                                          \
        break;
        MZB_FOR_EACH_OP1(X)
#undef X
    default:
        break;
    }
}

void launch_conj_sort(const conj_out *cq, uint64_t n, uint32_t nb, uint32_t *cnt, uint32_t *off, uint32_t *cursor,
                      conj_out *grp, conj_rec *out, cudaStream_t stream)
{
    cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * nb, stream);
    if (n > 0) k_conj_count<<<unsigned((n + 255) / 256), 256, 0, stream>>>(cq, n, cnt);
    k_conj_offsets<<<1, 1024, 0, stream>>>(cnt, nb, off, cursor);
    if (n == 0) return;
    k_conj_group<<<unsigned((n + 255) / 256), 256, 0, stream>>>(cq, n, off, cursor, grp);
    k_conj_sort_step<<<nb, 1024, CONJ_SORT_SMEM, stream>>>(grp, off, out);
    k_conj_rank<<<unsigned((n + 255) / 256), 256, 0, stream>>>(grp, n, off, out);
}

cudaError_t init_narrow_consts()
{
    const cudaError_t e = cudaFuncSetAttribute(k_conj_sort_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(CONJ_SORT_SMEM));
    if (e != cudaSuccess) return e;
    return upload_binom_table();
}

} // namespace mzb
