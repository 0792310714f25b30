// Stage 4 of a conjunction step: broad phase, i.e. every object's box tested
// against the step's BVH (mizuba/detect_conjunctions_broad_phase.cpp:153-339).
//
// The reference walks the tree once per object in Morton order with an
// explicit stack and emits (orig_p, orig_q) for every member q of every
// overlapped leaf with orig_p < orig_q and otype[p] + otype[q] <= 3, then sorts
// the step's pairs lexicographically.  Here one thread handles one Morton
// position p (so a warp's boxes are neighbours in space and its traversals
// stay coherent), walks the tree without a stack by following ropes, and
// files its pairs under the object's original index a = srt_idx[p]: a count
// pass, an exclusive scan over (step, original index), a write pass at the
// scanned offsets and an in-place insertion sort of each object's short list
// of partners produce the lexicographic order directly.  Overlap is the
// reference's closed-interval test on the four dimensions
// (broad_phase.cpp:269-271).
#include "block.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

// `aabbs` here are the Morton-sorted boxes (srt_aabbs).
template <bool WRITE>
__global__ void __launch_bounds__(128) k_broad(const float *__restrict__ aabbs, const bvh_node *__restrict__ trees,
                                               uint64_t cap, const int32_t *__restrict__ ropes,
                                               const uint32_t *__restrict__ srt_idx,
                                               const uint32_t *__restrict__ tree_size,
                                               const int32_t *__restrict__ otypes, uint32_t s_first, uint32_t nb,
                                               uint64_t N, uint32_t *__restrict__ counts,
                                               const uint64_t *__restrict__ offs, uint2 *__restrict__ pairs)
{
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (gid >= N * nb) return;
    const uint32_t b = uint32_t(gid / N);
    const uint32_t p = uint32_t(gid % N);
    const uint64_t s = uint64_t(s_first) + b;
    const uint32_t *sidx = srt_idx + s * N;
    const uint32_t a = sidx[p];
    const uint64_t slot = uint64_t(b) * N + a;
    const float4 *row = reinterpret_cast<const float4 *>(aabbs + (s * (N + 1) + p) * 8);
    const float4 lb = row[0], ub = row[1];
    uint32_t cnt = 0;
    if (isfinite(lb.x) && tree_size[s] > 0) {
        const bvh_node *tree = trees + s * cap;
        const int32_t *rope = ropes + uint64_t(b) * cap;
        const int32_t ota = otypes[a];
        uint2 *out = WRITE ? pairs + offs[slot] : nullptr;
        int32_t cur = 0;
        while (cur >= 0) {
            const float4 *np = reinterpret_cast<const float4 *>(tree + cur);
            const float4 h = np[0], nl = np[1], nu = np[2]; // {begin,end,left,right}, lb, ub
            const bool ov = (ub.x >= nl.x && lb.x <= nu.x) && (ub.y >= nl.y && lb.y <= nu.y)
                            && (ub.z >= nl.z && lb.z <= nu.z) && (ub.w >= nl.w && lb.w <= nu.w);
            const int32_t left = __float_as_int(h.z);
            if (ov && left != -1) {
                cur = left;
                continue;
            }
            if (ov) {
                const uint32_t qb = __float_as_uint(h.x), qe = __float_as_uint(h.y);
                for (uint32_t q = qb; q < qe; ++q) {
                    const uint32_t o = sidx[q];
                    if (a < o && ota + otypes[o] <= 3) {
                        if (WRITE) out[cnt] = make_uint2(a, o);
                        ++cnt;
                    }
                }
            }
            cur = rope[cur];
        }
        if (WRITE) {
            // Partners of a in ascending order.
            for (uint32_t x = 1; x < cnt; ++x) {
                const uint2 v = out[x];
                uint32_t y = x;
                while (y > 0 && out[y - 1].y > v.y) {
                    out[y] = out[y - 1];
                    --y;
                }
                out[y] = v;
            }
        }
    }
    if (!WRITE) counts[slot] = cnt;
}

// ---- exclusive scan of uint32 counts into uint64 offsets (3 kernels).
constexpr int SCAN_T = 1024;

__global__ void k_scan_blocks(const uint32_t *in, uint64_t n, uint64_t *out, uint64_t *block_sums)
{
    __shared__ uint32_t sm[33];
    const uint64_t i = blockIdx.x * uint64_t(SCAN_T) + threadIdx.x;
    const uint32_t v = i < n ? in[i] : 0;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(v, sm, &tot);
    if (i < n) out[i] = ex;
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// One block: exclusive scan of the per-block totals, chunk by chunk.  The
// per-block totals are 32-bit (block_excl_scan); a batch is limited on the
// host to fewer than 2^32 pairs, so every partial sum here fits in 32 bits.
__global__ void k_scan_sums(uint64_t *block_sums, uint64_t nblocks, uint64_t *total)
{
    __shared__ uint32_t sm[33];
    uint64_t carry = 0;
    for (uint64_t base = 0; base < nblocks; base += SCAN_T) {
        const uint64_t k = base + threadIdx.x;
        const uint32_t v = k < nblocks ? uint32_t(block_sums[k]) : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(v, sm, &tot);
        if (k < nblocks) block_sums[k] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(uint64_t *out, uint64_t n, const uint64_t *block_sums)
{
    const uint64_t i = blockIdx.x * uint64_t(SCAN_T) + threadIdx.x;
    if (i < n) out[i] += block_sums[blockIdx.x];
}

// Per-step pair offsets: off[b] = scanned offset of (step b, object 0).
__global__ void k_step_offsets(const uint64_t *offs, uint64_t N, uint32_t nb, const uint64_t *total, uint64_t *step_off)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb) step_off[b] = offs[uint64_t(b) * N];
    if (b == nb) step_off[nb] = *total;
}

void launch_broad(bool write, const float *aabbs, const bvh_node *trees, uint64_t cap, const int32_t *ropes,
                  const uint32_t *srt_idx, const uint32_t *tree_size, const int32_t *otypes, uint32_t s_first,
                  uint32_t nb, uint64_t N, uint32_t *counts, const uint64_t *offs, uint2 *pairs, cudaStream_t stream)
{
    const uint64_t n = N * nb;
    const unsigned bs = 128, g = unsigned((n + bs - 1) / bs);
    if (write)
        k_broad<true><<<g, bs, 0, stream>>>(aabbs, trees, cap, ropes, srt_idx, tree_size, otypes, s_first, nb, N,
                                            counts, offs, pairs);
    else
        k_broad<false><<<g, bs, 0, stream>>>(aabbs, trees, cap, ropes, srt_idx, tree_size, otypes, s_first, nb, N,
                                             counts, offs, pairs);
}

void launch_scan(const uint32_t *counts, uint64_t n, uint64_t *offs, uint64_t *block_sums, uint64_t *total,
                 cudaStream_t stream)
{
    const uint64_t nbk = (n + SCAN_T - 1) / SCAN_T;
    k_scan_blocks<<<unsigned(nbk), SCAN_T, 0, stream>>>(counts, n, offs, block_sums);
    k_scan_sums<<<1, SCAN_T, 0, stream>>>(block_sums, nbk, total);
    k_scan_add<<<unsigned(nbk), SCAN_T, 0, stream>>>(offs, n, block_sums);
}

void launch_step_offsets(const uint64_t *offs, uint64_t N, uint32_t nb, const uint64_t *total, uint64_t *step_off,
                         cudaStream_t stream)
{
    k_step_offsets<<<(nb + 1 + 127) / 128, 128, 0, stream>>>(offs, N, nb, total, step_off);
}

} // namespace mzb
