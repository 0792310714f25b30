// Stage 1 and 2 of a conjunction step: per-object AABBs (Cargo-Shisha
// enclosures of the segment polynomials, rounded outward to float) with the
// step's global box, then 64-bit Morton codes of the box centres.
//
// Reference: mizuba/detect_conjunctions_aabbs.cpp:64-398 and
// mizuba/detect_conjunctions_morton.cpp:70-175.
#include <utility>

#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

// mizuba layout [gseg][k][7] -> working layout [gseg][7][op1], so that one
// variable's coefficients are contiguous.
__global__ void k_relayout(const double *__restrict__ src, double *__restrict__ dst, uint64_t n_seg, int op1)
{
    const uint64_t per = uint64_t(op1) * 7;
    const uint64_t total = n_seg * per;
    for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < total; g += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t seg = g / per, r = g % per;
        const uint64_t v = r / op1, k = r % op1;
        dst[g] = src[seg * per + k * 7 + v];
    }
}

// One thread per (step, object).  For each trajectory segment overlapping the
// step, the x, y, z and r polynomials are translated to the start of the
// overlap and enclosed with Cargo-Shisha (aabbs.cpp:146-244); the enclosure is
// widened by the conjunction radius and rounded outward to float
// (aabbs.cpp:206-231); the per-object box is the union over segments.
template <int OP1>
__global__ void __launch_bounds__(128) k_aabb(dev_pj pj, const double2 *__restrict__ cd_bounds, uint32_t s_first,
                                              uint32_t n_batch, double radius, float *__restrict__ aabbs,
                                              uint32_t *__restrict__ gbox, dev_status *st)
{
    const uint64_t N = pj.n_objs;
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const bool active = gid < N * n_batch;
    const uint32_t b = active ? uint32_t(gid / N) : 0;
    const uint64_t i = active ? gid % N : 0;

    float lb[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    float ub[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    if (active) {
        const double2 cbe = cd_bounds[s_first + b];
        const double cb = cbe.x, ce = cbe.y;
        const uint32_t ns = pj.nseg[i];
        if (ns > 0) {
            const double *t = pj.time + pj.time_off[i];
            if (!(t[0] >= ce || t[ns] <= cb)) {
                uint32_t tb, te;
                step_range(t, ns, cb, ce, tb, te);
                for (uint32_t it = tb; it != te; ++it) {
                    const double s0 = t[it - 1];
                    const double ev_lb = (cb < s0) ? s0 : cb;       // std::max(cb, s0)
                    const double ev_ub = (t[it] < ce) ? t[it] : ce; // std::min(ce, t[it])
                    const double h_lb = ev_lb - s0, h_ub = ev_ub - s0;
                    const double *cf = pj.coef + (pj.seg_off[i] + it - 1) * (7 * OP1);
#pragma unroll 1
                    for (int d = 0; d < 4; ++d) {
                        const int v = (d == 3) ? 6 : d;
                        double c[OP1], tr[OP1];
#pragma unroll
                        for (int k = 0; k < OP1; ++k) c[k] = __ldg(cf + v * OP1 + k);
                        translate<OP1>(c, h_lb, tr);
                        double mn, mx;
                        cs_from_translated<OP1>(tr, h_ub - h_lb, mn, mx);
                        mn = mn - radius;
                        mx = mx + radius;
                        const float fl = next_down(__double2float_rn(mn));
                        const float fu = next_up(__double2float_rn(mx));
                        if (!isfinite(fl)) set_error(st, ERR_AABB_LB, uint32_t(i), 0, fl, 0);
                        if (!isfinite(fu)) set_error(st, ERR_AABB_UB, uint32_t(i), 0, fu, 0);
                        lb[d] = fmin_ref(lb[d], fl);
                        ub[d] = fmax_ref(ub[d], fu);
                    }
                }
            }
        }
        float4 *o = reinterpret_cast<float4 *>(aabbs + ((uint64_t(s_first) + b) * (N + 1) + i) * 8);
        o[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
        o[1] = make_float4(ub[0], ub[1], ub[2], ub[3]);
    }
    // Global box of the step: ordered-integer atomics, warp-aggregated when
    // the whole warp works on one step.
    const unsigned lane = threadIdx.x & 31;
    const uint32_t b0 = __shfl_sync(0xffffffffu, b, 0);
    const bool uniform = __all_sync(0xffffffffu, !active || b == b0);
    const bool any_active = __any_sync(0xffffffffu, active);
    uint32_t olb[4], oub[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        olb[d] = active ? f2ord(lb[d]) : 0xffffffffu;
        oub[d] = active ? f2ord(ub[d]) : 0u;
    }
    if (uniform) {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            for (int off = 16; off > 0; off >>= 1) {
                olb[d] = min(olb[d], __shfl_xor_sync(0xffffffffu, olb[d], off));
                oub[d] = max(oub[d], __shfl_xor_sync(0xffffffffu, oub[d], off));
            }
        }
        if (lane == 0 && any_active) {
            // Inactive lanes carry neutral sentinels; lane 0 is active
            // whenever any lane is (inactive threads are the grid's tail).
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                atomicMin(gbox + b0 * 8 + d, olb[d]);
                atomicMax(gbox + b0 * 8 + 4 + d, oub[d]);
            }
        }
    } else if (active) {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            atomicMin(gbox + b * 8 + d, olb[d]);
            atomicMax(gbox + b * 8 + 4 + d, oub[d]);
        }
    }
}

__global__ void k_gbox_init(uint32_t *gbox, uint32_t n_batch)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n_batch * 8) gbox[g] = (g % 8 < 4) ? f2ord(INFINITY) : f2ord(-INFINITY);
}

// Writes the global box into row N of each step (aabbs.cpp:353-391).
__global__ void k_gbox_finalize(const uint32_t *gbox, uint32_t s_first, uint32_t n_batch, uint64_t N, float *aabbs,
                                dev_status *st)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_batch) return;
    float *row = aabbs + ((uint64_t(s_first) + b) * (N + 1) + N) * 8;
    for (int d = 0; d < 4; ++d) {
        const float l = ord2f(gbox[b * 8 + d]), u = ord2f(gbox[b * 8 + 4 + d]);
        if (isfinite(l) && !isfinite(u - l)) set_error(st, ERR_GLOBAL_AABB, 0, 0, 0, 0);
        row[d] = l;
        row[4 + d] = u;
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

void launch_relayout(const double *src, double *dst, uint64_t n_seg, int op1, cudaStream_t stream)
{
    if (n_seg == 0) return;
    k_relayout<<<148 * 8, 256, 0, stream>>>(src, dst, n_seg, op1);
}

template <int OP1>
static void aabb_t(const dev_pj &pj, const double2 *cdb, uint32_t s_first, uint32_t nb, double radius, float *aabbs,
                   uint32_t *gbox, dev_status *st, cudaStream_t stream)
{
    const uint64_t n = pj.n_objs * nb;
    const unsigned bs = 128;
    k_aabb<OP1><<<unsigned((n + bs - 1) / bs), bs, 0, stream>>>(pj, cdb, s_first, nb, radius, aabbs, gbox, st);
}

void launch_aabb(const dev_pj &pj, const double2 *cdb, uint32_t s_first, uint32_t nb, double radius, float *aabbs,
                 uint32_t *gbox, dev_status *st, cudaStream_t stream)
{
    k_gbox_init<<<(nb * 8 + 255) / 256, 256, 0, stream>>>(gbox, nb);
    switch (pj.op1) {
#define X(K)                                                                                                         \
    case K:                                                                                                            \
        aabb_t<K>(pj, cdb, s_first, nb, radius, aabbs, gbox, st, stream);                                            \
        break;
        MZB_FOR_EACH_OP1(X)
#undef X
    default:
        break;
    }
    k_gbox_finalize<<<(nb + 127) / 128, 128, 0, stream>>>(gbox, s_first, nb, pj.n_objs, aabbs, st);
}

void launch_morton(const float *aabbs, uint32_t s_first, uint32_t nb, uint64_t N, uint64_t *mcodes, cudaStream_t stream)
{
    const uint64_t n = N * nb;
    k_morton<<<unsigned((n + 255) / 256), 256, 0, stream>>>(aabbs, s_first, nb, N, mcodes);
}

cudaError_t init_aabb_consts() { return upload_binom_table(); }

} // namespace mzb
