// Stage 4 of a conjunction step: broad phase, i.e. every object's box tested
// against the step's BVH (mizuba/detect_conjunctions_broad_phase.cpp:153-339).
//
// The reference walks the tree once per object in Morton order with an
// explicit stack and emits (orig_p, orig_q) for every member q of every
// overlapped leaf with orig_p < orig_q and otype[p] + otype[q] <= 3, then sorts
// the step's pairs lexicographically.  Here one thread handles one Morton
// position (so a warp's boxes are neighbours in space and its walks stay
// coherent) and walks the tree without a stack by following ropes.  Each
// pair is examined once (the half traversal below); partners are counted per
// (step, original index), an exclusive scan gives every object its offset in
// the step's list, and a copy pass writes each object's sorted partners, so
// the lexicographic order comes out directly.  Overlap is the reference's
// closed-interval test on the four dimensions (broad_phase.cpp:269-271).
#include "block.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

// ---- Half traversal (one pass).
//
// Every pair is considered once, from the object x with the lower Morton
// position p.  x's query box is Q = box of x's leaf (equal to x's own box
// unless x sits in a multi-object leaf).  The walk starts at x's own leaf,
// whose members after p are tested first, and then follows the ropes: in
// the depth-first order of the tree the subtrees reached from a leaf by its
// rope chain hold exactly the positions after that leaf, so the walk never
// visits the root-to-leaf path or anything at or before p.  At a leaf L it
// tests each member y at a position q > p with the reference's rule for the
// pair (a, b) = (min, max) of the two indices, "box(a) overlaps the box of
// b's leaf": box(x) vs box(L) when x < y, box(y) vs Q when y < x.  A pair of
// the reference's set is reached by this walk because Q contains box(x) and
// b's leaf box contains box(b), so the exact rule gives the reference's pair
// set with half the node visits.  Partners are filed under a = min(x, y):
// the count by atomics, the first K partners into a small per-object buffer.
constexpr int BP_K = BROAD_STAGE_K;

__device__ __forceinline__ bool overlap4(float4 al, float4 au, float4 bl, float4 bu)
{
    return (au.x >= bl.x && al.x <= bu.x) && (au.y >= bl.y && al.y <= bu.y) && (au.z >= bl.z && al.z <= bu.z)
           && (au.w >= bl.w && al.w <= bu.w);
}

// The member tests of one leaf of a half walk (reached about 1.5 times per
// walk).
__device__ __forceinline__ void half_leaf(const float *__restrict__ srt_aabbs, const bvh_node *__restrict__ tree,
                                       const uint32_t *__restrict__ sidx, const int32_t *__restrict__ otypes,
                                       uint64_t s, uint64_t N, uint32_t b, uint32_t p, uint32_t x, int32_t own,
                                       int32_t cur, uint32_t qb, uint32_t qe, uint32_t *__restrict__ counts,
                                       uint32_t *__restrict__ stage, ulonglong2 *__restrict__ spill,
                                       uint64_t spill_cap, unsigned long long *spill_count)
{
    const float4 *row = reinterpret_cast<const float4 *>(srt_aabbs + (s * (N + 1) + p) * 8);
    const float4 *ln = reinterpret_cast<const float4 *>(tree + cur);
    const float4 *lq = reinterpret_cast<const float4 *>(tree + own);
    const int32_t otx = otypes[x];
    for (uint32_t q = (qb > p + 1 ? qb : p + 1); q < qe; ++q) {
        const uint32_t y = sidx[q];
        bool ok;
        if (x < y) {
            ok = overlap4(row[0], row[1], ln[1], ln[2]);
        } else {
            const float4 *ry = reinterpret_cast<const float4 *>(srt_aabbs + (s * (N + 1) + q) * 8);
            ok = overlap4(ry[0], ry[1], lq[1], lq[2]);
        }
        if (ok && otx + otypes[y] <= 3) {
            const uint32_t a = x < y ? x : y, o = x < y ? y : x;
            const uint64_t slot = uint64_t(b) * N + a;
            const uint32_t k = atomicAdd(counts + slot, 1u);
            if (k < BP_K) {
                stage[slot * BP_K + k] = o;
            } else {
                const unsigned long long w = atomicAdd(spill_count, 1ull);
                if (w < spill_cap) spill[w] = make_ulonglong2(slot, o);
            }
        }
    }
}

// The half walk of position gid % N of batch step gid / N (see above).
__device__ __forceinline__ void walk_half(const float *__restrict__ srt_aabbs, const bvh_node *__restrict__ trees,
                                          uint64_t cap, const walk_node *__restrict__ walks,
                                          const uint32_t *__restrict__ leaf_of, const uint32_t *__restrict__ srt_idx,
                                          const uint32_t *__restrict__ tree_size, const int32_t *__restrict__ otypes,
                                          uint32_t s_first, uint64_t N, uint32_t *__restrict__ counts,
                                          uint32_t *__restrict__ stage, ulonglong2 *__restrict__ spill,
                                          uint64_t spill_cap, unsigned long long *spill_count, uint64_t gid,
                                          uint32_t &n_visits)
{
    const uint32_t b = uint32_t(gid / N);
    const uint32_t p = uint32_t(gid % N);
    const uint64_t s = uint64_t(s_first) + b;
    const float4 *row = reinterpret_cast<const float4 *>(srt_aabbs + (s * (N + 1) + p) * 8);
    if (!isfinite(row[0].x) || tree_size[s] == 0) return;
    const bvh_node *tree = trees + s * cap;
    const walk_node *wk = walks + uint64_t(b) * cap;
    const uint32_t *sidx = srt_idx + s * N;
    const uint32_t x = sidx[p];
    const int32_t own = int32_t(leaf_of[uint64_t(b) * N + p]);
    // The walk prunes with the quantised query box; the exact query box and
    // x's own box are read at leaves only (about 1.5 leaves per walk).
    const uint4 qq = reinterpret_cast<const uint4 *>(wk + own)[0];
    int32_t cur = own;
    while (cur >= 0) {
        // One 32-byte sector per visit: quantised box, left child, rope and
        // member range.
        const uint4 nq = reinterpret_cast<const uint4 *>(wk + cur)[0];
        const int4 m = reinterpret_cast<const int4 *>(wk + cur)[1];
        ++n_visits;
        if (!walk_overlap(qq, nq)) {
            cur = m.y;
            continue;
        }
        if (m.x != -1) {
            cur = m.x;
            continue;
        }
        // Leaf: the reference's exact rule on each member after p (the
        // member tests imply the exact query-box / leaf-box overlap, so the
        // conservative test above changes no pair).
        half_leaf(srt_aabbs, tree, sidx, otypes, s, N, b, p, x, own, cur, uint32_t(m.z), uint32_t(m.w), counts,
                  stage, spill, spill_cap, spill_count);
        cur = m.y;
    }
}

__global__ void __launch_bounds__(128) k_broad_half(const float *__restrict__ srt_aabbs,
                                                    const bvh_node *__restrict__ trees, uint64_t cap,
                                                    const walk_node *__restrict__ walks,
                                                    const uint32_t *__restrict__ leaf_of,
                                                    const uint32_t *__restrict__ srt_idx,
                                                    const uint32_t *__restrict__ tree_size,
                                                    const int32_t *__restrict__ otypes, uint32_t s_first,
                                                    uint32_t nb, uint64_t N, uint32_t *__restrict__ counts,
                                                    uint32_t *__restrict__ stage, ulonglong2 *__restrict__ spill,
                                                    uint64_t spill_cap, unsigned long long *spill_count,
                                                    unsigned long long *visits)
{
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    uint32_t n_visits = 0;
    if (gid < N * nb) walk_half(srt_aabbs, trees, cap, walks, leaf_of, srt_idx, tree_size, otypes, s_first, N,
                                counts, stage, spill, spill_cap, spill_count, gid, n_visits);
    // Node visits of the block's walks, one atomic per warp (the walk's
    // work unit for the roofline).
    const unsigned long long w = __reduce_add_sync(0xffffffffu, n_visits);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(visits, w);
}

// ---- Half traversal with work refill.
//
// The walk and pair rule of k_broad_half, but a lane whose walk has ended
// takes the next position at once instead of waiting for the slowest walk of
// its warp (walk lengths vary several-fold between neighbours, so a warp
// with fixed positions spends most of its time with a third of its lanes
// active).  Each warp draws pools of WALK_POOL consecutive positions from a
// global counter with one atomic; every loop iteration hands the pool's next
// positions to the lanes without a walk and advances every other lane by one
// node.  The set of live lanes is kept explicitly and the warp reconverges on
// it at the top of each iteration, so the pool bookkeeping is warp-uniform.
// On the 20k-object catalogue it loses to fixed positions (3.57 ms against
// 2.81 ms for a day): the per-visit reconvergence and ballot cost more than
// the idle lanes did.  It is kept for inputs with more skewed walks and is
// measured by the autotuner.
constexpr uint32_t WALK_POOL = 64;

__global__ void __launch_bounds__(128) k_broad_pool(const float *__restrict__ srt_aabbs,
                                                    const bvh_node *__restrict__ trees, uint64_t cap,
                                                    const walk_node *__restrict__ walks,
                                                    const uint32_t *__restrict__ leaf_of,
                                                    const uint32_t *__restrict__ srt_idx,
                                                    const uint32_t *__restrict__ tree_size,
                                                    const int32_t *__restrict__ otypes, uint32_t s_first,
                                                    uint32_t nb, uint64_t N, uint32_t *__restrict__ counts,
                                                    uint32_t *__restrict__ stage, ulonglong2 *__restrict__ spill,
                                                    uint64_t spill_cap, unsigned long long *spill_count,
                                                    unsigned long long *next)
{
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const uint64_t total = N * nb;
    unsigned alive = 0xffffffffu;
    uint64_t pool = 0, pool_end = 0; // warp-uniform
    int32_t cur = -1, own = 0;
    uint32_t b = 0, p = 0, x = 0;
    uint64_t s = 0;
    uint4 qq = make_uint4(0, 0, 0, 0);
    for (;;) {
        __syncwarp(alive);
        const unsigned need = __ballot_sync(alive, cur < 0);
        if (need) {
            if (pool == pool_end) {
                const int leader = __ffs(alive) - 1;
                unsigned long long base = 0;
                if (int(lane) == leader) base = atomicAdd(next, (unsigned long long)WALK_POOL);
                base = __shfl_sync(alive, base, leader);
                pool = base < total ? base : total;
                pool_end = base + WALK_POOL < total ? base + WALK_POOL : total;
            }
            const uint64_t avail = pool_end - pool;
            if (avail == 0) { // every position has been handed out
                alive &= ~need;
                if (cur < 0) break;
                continue;
            }
            if (cur < 0) {
                const uint32_t rank = __popc(need & lt);
                if (rank < avail) {
                    const uint64_t gid = pool + rank;
                    b = uint32_t(gid / N);
                    p = uint32_t(gid % N);
                    s = uint64_t(s_first) + b;
                    const float *row = srt_aabbs + (s * (N + 1) + p) * 8;
                    if (isfinite(row[0]) && tree_size[s] != 0) {
                        x = srt_idx[s * N + p];
                        own = int32_t(leaf_of[uint64_t(b) * N + p]);
                        qq = reinterpret_cast<const uint4 *>(walks + uint64_t(b) * cap + own)[0];
                        cur = own;
                    }
                }
            }
            const uint32_t k = __popc(need);
            pool += (k < avail) ? k : avail;
            continue; // lanes given a position start walking next iteration
        }
        // Every live lane has a walk: advance it by one node.
        const walk_node *wk = walks + uint64_t(b) * cap;
        const uint4 nq = reinterpret_cast<const uint4 *>(wk + cur)[0];
        const int4 m = reinterpret_cast<const int4 *>(wk + cur)[1];
        if (!walk_overlap(qq, nq)) {
            cur = m.y;
        } else if (m.x != -1) {
            cur = m.x;
        } else {
            half_leaf(srt_aabbs, trees + s * cap, srt_idx + s * N, otypes, s, N, b, p, x, own, cur, uint32_t(m.z),
                      uint32_t(m.w), counts, stage, spill, spill_cap, spill_count);
            cur = m.y;
        }
    }
}

// ---- Warp-coherent half traversal.
//
// The same walk and pair rule as k_broad_half, made warp-uniform.  A warp
// holds 32 consecutive Morton positions p of one step (warps never straddle
// two steps), i.e. 32 spatial neighbours whose walks largely coincide.  The
// warp starts at the leaf of its first position and follows the ropes; it
// descends into a node when any lane wants it (an overlap of the lane's
// query box with the node box, and positions after the lane's own in the
// node), otherwise it takes the rope.  Every lane's own leaf and every
// subtree holding positions after it come after the first lane's leaf in
// the depth-first order, so each lane meets every node its own walk would;
// at a leaf each interested lane tests only the members after its own
// position, with the exact rule of k_broad_half, so the pairs are the same.
// Node and rope loads are the same address across the warp (broadcasts) and
// the loop has no divergence except inside leaves.
__global__ void __launch_bounds__(128) k_broad_warp(const float *__restrict__ srt_aabbs,
                                                    const bvh_node *__restrict__ trees, uint64_t cap,
                                                    const int32_t *__restrict__ ropes,
                                                    const uint32_t *__restrict__ leaf_of,
                                                    const uint32_t *__restrict__ srt_idx,
                                                    const uint32_t *__restrict__ tree_size,
                                                    const int32_t *__restrict__ otypes, uint32_t s_first,
                                                    uint32_t nb, uint64_t N, uint32_t *__restrict__ counts,
                                                    uint32_t *__restrict__ stage, ulonglong2 *__restrict__ spill,
                                                    uint64_t spill_cap, unsigned long long *spill_count)
{
    const uint64_t warps_per_step = (N + 31) / 32;
    const uint64_t gw = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) / 32;
    const unsigned lane = threadIdx.x & 31;
    if (gw >= warps_per_step * nb) return; // whole warps only
    const uint32_t b = uint32_t(gw / warps_per_step);
    const uint64_t p64 = (gw % warps_per_step) * 32 + lane;
    const uint64_t s = uint64_t(s_first) + b;
    if (tree_size[s] == 0) return; // uniform over the warp
    bool active = p64 < N;
    const uint32_t p = uint32_t(p64);
    float4 xl = make_float4(0, 0, 0, 0), xu = xl, ql = xl, qu = xl;
    uint32_t x = 0;
    int32_t otx = 0;
    int32_t own = -1;
    if (active) {
        const float4 *row = reinterpret_cast<const float4 *>(srt_aabbs + (s * (N + 1) + p) * 8);
        xl = row[0];
        xu = row[1];
        active = isfinite(xl.x);
    }
    const bvh_node *tree = trees + s * cap;
    const int32_t *rope = ropes + uint64_t(b) * cap;
    const uint32_t *sidx = srt_idx + s * N;
    if (active) {
        x = sidx[p];
        otx = otypes[x];
        own = int32_t(leaf_of[uint64_t(b) * N + p]);
        const float4 *lq = reinterpret_cast<const float4 *>(tree + own);
        ql = lq[1];
        qu = lq[2];
    }
    // No-data boxes sort last: the active lanes are a prefix of the warp.
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (act == 0) return;
    int32_t cur = __shfl_sync(0xffffffffu, own, __ffs(act) - 1);
    while (cur >= 0) {
        const float4 *np = reinterpret_cast<const float4 *>(tree + cur);
        const float4 h = np[0], nl = np[1], nu = np[2];
        const int32_t next = rope[cur];
        const uint32_t qb = __float_as_uint(h.x), qe = __float_as_uint(h.y);
        const bool want = active && qe > p + 1 && overlap4(ql, qu, nl, nu);
        const int32_t left = __float_as_int(h.z);
        if (left != -1) {
            cur = __any_sync(0xffffffffu, want) ? left : next;
            continue;
        }
        if (want) {
            for (uint32_t q = (qb > p + 1 ? qb : p + 1); q < qe; ++q) {
                const uint32_t y = sidx[q];
                bool ok;
                if (x < y) {
                    ok = overlap4(xl, xu, nl, nu);
                } else {
                    const float4 *ry = reinterpret_cast<const float4 *>(srt_aabbs + (s * (N + 1) + q) * 8);
                    ok = overlap4(ry[0], ry[1], ql, qu);
                }
                if (ok && otx + otypes[y] <= 3) {
                    const uint32_t a = x < y ? x : y, o = x < y ? y : x;
                    const uint64_t slot = uint64_t(b) * N + a;
                    const uint32_t k = atomicAdd(counts + slot, 1u);
                    if (k < BP_K) {
                        stage[slot * BP_K + k] = o;
                    } else {
                        const unsigned long long w = atomicAdd(spill_count, 1ull);
                        if (w < spill_cap) spill[w] = make_ulonglong2(slot, o);
                    }
                }
            }
        }
        cur = next;
    }
}

// Writes each object's partners (sorted) at its scanned offset; objects with
// more than BP_K partners are listed for the full walk below.
__global__ void k_broad_copy(uint32_t *__restrict__ counts, const uint64_t *__restrict__ offs,
                             const uint32_t *__restrict__ stage, uint32_t nb, uint64_t N, uint2 *__restrict__ pairs,
                             uint64_t *__restrict__ overflow, unsigned long long *overflow_count)
{
    const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (gid >= N * nb) return;
    const uint32_t cnt = counts[gid];
    if (cnt == 0) return;
    const uint32_t a = uint32_t(gid % N);
    if (cnt > BP_K) {
        // The first BP_K partners now; the spilled ones are scattered behind
        // them (the count becomes the scatter cursor) and the list is sorted
        // afterwards, or the full walk below rewrites it.
        overflow[atomicAdd(overflow_count, 1ull)] = gid;
        uint2 *out = pairs + offs[gid];
#pragma unroll
        for (int k = 0; k < BP_K; ++k) out[k] = make_uint2(a, stage[gid * BP_K + k]);
        counts[gid] = BP_K;
        return;
    }
    uint32_t v[BP_K];
#pragma unroll
    for (int k = 0; k < BP_K; ++k) v[k] = (uint32_t(k) < cnt) ? stage[gid * BP_K + k] : 0xffffffffu;
#pragma unroll
    for (int x = 1; x < BP_K; ++x)
#pragma unroll
        for (int y = x; y > 0; --y)
            if (v[y - 1] > v[y]) {
                const uint32_t t = v[y - 1];
                v[y - 1] = v[y];
                v[y] = t;
            }
    uint2 *out = pairs + offs[gid];
#pragma unroll
    for (int k = 0; k < BP_K; ++k)
        if (uint32_t(k) < cnt) out[k] = make_uint2(a, v[k]);
}

// Spilled partners to their places behind the staged ones.
__global__ void __launch_bounds__(256) k_broad_spill(const ulonglong2 *__restrict__ spill,
                                                     const unsigned long long *spill_count, uint64_t N,
                                                     const uint64_t *__restrict__ offs, uint32_t *__restrict__ cursor,
                                                     uint2 *__restrict__ pairs)
{
    const uint64_t n = *spill_count;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n;
         k += uint64_t(gridDim.x) * blockDim.x) {
        const ulonglong2 e = spill[k];
        const uint32_t pos = atomicAdd(cursor + e.x, 1u);
        pairs[offs[e.x] + pos] = make_uint2(uint32_t(e.x % N), uint32_t(e.y));
    }
}

// Sorts each overflowing object's partner list by partner index (one thread
// per object; the lists are short except in dense clusters).
__global__ void __launch_bounds__(128) k_broad_sort_lists(const uint64_t *__restrict__ overflow,
                                                          const unsigned long long *overflow_count,
                                                          const uint64_t *__restrict__ offs,
                                                          const uint32_t *__restrict__ cnts, uint2 *__restrict__ pairs)
{
    const uint64_t n = *overflow_count;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n;
         k += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t gid = overflow[k];
        uint2 *out = pairs + offs[gid];
        const uint32_t cnt = cnts[gid];
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

// Full walk for the objects with more than BP_K partners: the reference's own
// per-object rule (box(a) against the leaf boxes of its partners b > a),
// written at the object's offset and sorted.
__global__ void __launch_bounds__(128) k_broad_full(const float *__restrict__ aabbs,
                                                    const bvh_node *__restrict__ trees, uint64_t cap,
                                                    const int32_t *__restrict__ ropes,
                                                    const uint32_t *__restrict__ srt_idx,
                                                    const int32_t *__restrict__ otypes, uint32_t s_first, uint64_t N,
                                                    const uint64_t *__restrict__ overflow,
                                                    const unsigned long long *overflow_count,
                                                    const uint64_t *__restrict__ offs, uint2 *__restrict__ pairs)
{
    const uint64_t n = *overflow_count;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n;
         k += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t gid = overflow[k];
        const uint32_t b = uint32_t(gid / N), a = uint32_t(gid % N);
        const uint64_t s = uint64_t(s_first) + b;
        const float4 *row = reinterpret_cast<const float4 *>(aabbs + (s * (N + 1) + a) * 8);
        const float4 lb = row[0], ub = row[1];
        const bvh_node *tree = trees + s * cap;
        const int32_t *rope = ropes + uint64_t(b) * cap;
        const uint32_t *sidx = srt_idx + s * N;
        const int32_t ota = otypes[a];
        uint2 *out = pairs + offs[gid];
        uint32_t cnt = 0;
        int32_t cur = 0;
        while (cur >= 0) {
            const float4 *np = reinterpret_cast<const float4 *>(tree + cur);
            const float4 h = np[0], nl = np[1], nu = np[2];
            const int32_t next = rope[cur];
            const bool ov = overlap4(lb, ub, nl, nu);
            const int32_t left = __float_as_int(h.z);
            if (ov && left != -1) {
                cur = left;
                continue;
            }
            if (ov) {
                const uint32_t qb = __float_as_uint(h.x), qe = __float_as_uint(h.y);
                for (uint32_t q = qb; q < qe; ++q) {
                    const uint32_t o = sidx[q];
                    if (a < o && ota + otypes[o] <= 3) out[cnt++] = make_uint2(a, o);
                }
            }
            cur = next;
        }
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

void launch_broad_half(const float *srt_aabbs, const bvh_node *trees, uint64_t cap, const int32_t *ropes,
                       const walk_node *walks, const uint32_t *leaf_of, const uint32_t *srt_idx,
                       const uint32_t *tree_size, const int32_t *otypes, uint32_t s_first, uint32_t nb, uint64_t N,
                       uint32_t *counts, uint32_t *stage, ulonglong2 *spill, uint64_t spill_cap,
                       unsigned long long *spill_count, unsigned long long *walk_next, int walk,
                       unsigned long long *visits, cudaStream_t stream)
{
    const uint64_t n = N * nb;
    cudaMemsetAsync(counts, 0, n * sizeof(uint32_t), stream);
    cudaMemsetAsync(spill_count, 0, sizeof(unsigned long long), stream);
    if (walk == 2) {
        cudaMemsetAsync(walk_next, 0, sizeof(unsigned long long), stream);
        // Enough warps to fill every SM; each keeps drawing positions.
        k_broad_pool<<<148 * 16, 128, 0, stream>>>(srt_aabbs, trees, cap, walks, leaf_of, srt_idx, tree_size, otypes,
                                                   s_first, nb, N, counts, stage, spill, spill_cap, spill_count,
                                                   walk_next);
    } else if (walk == 0) {
        k_broad_half<<<unsigned((n + 127) / 128), 128, 0, stream>>>(srt_aabbs, trees, cap, walks, leaf_of, srt_idx,
                                                                    tree_size, otypes, s_first, nb, N, counts, stage,
                                                                    spill, spill_cap, spill_count, visits);
    } else {
        const uint64_t threads = (N + 31) / 32 * 32 * nb;
        k_broad_warp<<<unsigned((threads + 127) / 128), 128, 0, stream>>>(srt_aabbs, trees, cap, ropes, leaf_of,
                                                                          srt_idx, tree_size, otypes, s_first, nb, N,
                                                                          counts, stage, spill, spill_cap,
                                                                          spill_count);
    }
}

// spilled_ok: every spilled partner was kept (the spill list did not
// overflow), so the lists are completed by scatter and sort; otherwise the
// overflowing objects are walked again in full.
void launch_broad_copy(const float *aabbs, const bvh_node *trees, uint64_t cap, const int32_t *ropes,
                       const uint32_t *srt_idx, const int32_t *otypes, uint32_t s_first, uint32_t nb, uint64_t N,
                       uint32_t *counts, const uint64_t *offs, const uint32_t *stage, uint2 *pairs,
                       uint64_t *overflow, unsigned long long *overflow_count, const ulonglong2 *spill,
                       const unsigned long long *spill_count, bool spilled_ok, cudaStream_t stream)
{
    const uint64_t n = N * nb;
    cudaMemsetAsync(overflow_count, 0, sizeof(unsigned long long), stream);
    k_broad_copy<<<unsigned((n + 255) / 256), 256, 0, stream>>>(counts, offs, stage, nb, N, pairs, overflow,
                                                                overflow_count);
    if (spilled_ok) {
        k_broad_spill<<<148 * 8, 256, 0, stream>>>(spill, spill_count, N, offs, counts, pairs);
        k_broad_sort_lists<<<148 * 4, 128, 0, stream>>>(overflow, overflow_count, offs, counts, pairs);
    } else {
        k_broad_full<<<148 * 4, 128, 0, stream>>>(aabbs, trees, cap, ropes, srt_idx, otypes, s_first, N, overflow,
                                                  overflow_count, offs, pairs);
    }
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
