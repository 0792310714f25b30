// State evaluation of a polyjectory at arbitrary times: polyjectory::state_eval
// and polyjectory::state_meval (mizuba/polyjectory.cpp:1162-1366), whose
// per-(object, time) work is pj_eval_obj_state (mizuba/polyjectory.cpp:1092-1159).
//
// One thread per (object, time) evaluation.  The segment holding the time is
// found by binary search for the first segment end after it (upper_bound over
// the object's time points 1 .. n_steps), and the seven state variables are
// evaluated by Horner's scheme in the reference's operation order
// (c[n-o] + res * h, no fused multiply-add: the library is compiled without
// contraction).  Objects without data, and times before the first time point
// or at / after the last one, give NaN in all seven outputs.  Consecutive
// threads evaluate consecutive times of one object (state_meval), so they
// read the same segment coefficients through L1/L2.
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

__global__ void __launch_bounds__(128) k_state_eval(dev_pj pj, const double *__restrict__ tm, uint64_t tm_stride_obj,
                                                    uint64_t tm_stride_t, const uint64_t *__restrict__ sel,
                                                    uint64_t n_eval, uint64_t n_t, double *__restrict__ out)
{
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (gid >= n_eval * n_t) return;
    const uint64_t e = gid / n_t, j = gid % n_t;
    const uint64_t obj = sel ? sel[e] : e;
    const double t = tm[e * tm_stride_obj + j * tm_stride_t];
    double *o = out + gid * 7;
    const uint32_t ns = pj.nseg[obj];
    const double *times = pj.time + pj.time_off[obj];
    if (ns == 0 || t < times[0] || t >= times[ns]) {
#pragma unroll
        for (int v = 0; v < 7; ++v) o[v] = NAN;
        return;
    }
    // First k in [1, ns] with times[k] > t (exists because t < times[ns]).
    uint32_t lo = 1, hi = ns;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (times[mid] > t) hi = mid;
        else lo = mid + 1;
    }
    const uint32_t seg = lo - 1;
    const double h = t - times[seg];
    const int n = pj.order, op1 = pj.op1;
    const int ld = row_ld(op1);
    const double *cf = pj.coef + (pj.seg_off[obj] + seg) * uint64_t(7 * ld);
#pragma unroll
    for (int v = 0; v < 7; ++v) {
        const double *c = cf + v * ld;
        double res = c[n];
        for (int k = n - 1; k >= 0; --k) res = __dadd_rn(c[k], __dmul_rn(res, h));
        o[v] = res;
    }
}

void launch_state_eval(const dev_pj &pj, const double *tm, uint64_t tm_stride_obj, uint64_t tm_stride_t,
                       const uint64_t *sel, uint64_t n_eval, uint64_t n_t, double *out, cudaStream_t stream)
{
    const uint64_t n = n_eval * n_t;
    if (n == 0) return;
    k_state_eval<<<unsigned((n + 127) / 128), 128, 0, stream>>>(pj, tm, tm_stride_obj, tm_stride_t, sel, n_eval, n_t,
                                                                 out);
}

} // namespace mzb
