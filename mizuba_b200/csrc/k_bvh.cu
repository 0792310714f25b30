// Stage 3 of a conjunction step: the BVH over the Morton-sorted boxes
// (mizuba/detect_conjunctions_bvh.cpp:267-699).
//
// One 1024-thread CTA per step builds the tree level by level exactly as the
// reference numbers it: a node [begin, end) with more than one object splits
// at the first bit (from the MSB) where its codes differ, i.e.
// clz(code[begin] ^ code[end - 1]), at the first position whose code has that
// bit set (binary search); equal codes make a multi-object leaf.  Children of
// the level's internal nodes are appended in parent order (left child index =
// level end + exclusive prefix of child counts, bvh.cpp:572-580), so the
// array is in breadth-first order with adjacent siblings.  Leaf boxes are the
// min/max over members; internal boxes come from a bottom-up pass over the
// levels.  A rope (escape index) per node is produced for the stackless
// broad-phase traversal: rope(left) = right sibling, rope(right) =
// rope(parent), rope(root) = -1.
#include "block.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

constexpr int BVH_T = 1024;
constexpr int MAX_LEVELS = 160;

__global__ void __launch_bounds__(BVH_T, 2) k_bvh(const float *__restrict__ srt_aabbs,
                                               const uint64_t *__restrict__ srt_mcodes, uint32_t s_first,
                                               uint64_t N, bvh_node *__restrict__ trees, uint64_t cap,
                                               int32_t *__restrict__ ropes, uint32_t *__restrict__ aux,
                                               uint32_t *__restrict__ leaf_of, uint32_t *__restrict__ tree_size,
                                               dev_status *st)
{
    __shared__ uint32_t scan_smem[33];
    __shared__ uint32_t lvl[MAX_LEVELS + 1];
    __shared__ uint32_t s_neff, s_nlev;

    const uint32_t b = blockIdx.x;
    const uint64_t s = uint64_t(s_first) + b;
    const unsigned tid = threadIdx.x;
    const float *sa = srt_aabbs + s * (N + 1) * 8;
    const uint64_t *mc = srt_mcodes + s * N;
    bvh_node *tree = trees + s * cap;
    int32_t *rope = ropes + uint64_t(b) * cap;
    // aux[2 * node]: split index; aux[2 * node + 1]: child count / scratch.
    uint32_t *ax = aux + uint64_t(b) * cap * 2;
    // leaf_of[p]: the leaf holding Morton position p (for the broad phase).
    uint32_t *lof = leaf_of + uint64_t(b) * N;

    if (tid == 0) {
        // Number of finite boxes: they precede the no-data ones.
        uint64_t lo = 0, hi = N;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) / 2;
            if (!isinf(sa[mid * 8])) lo = mid + 1;
            else hi = mid;
        }
        s_neff = uint32_t(lo);
    }
    __syncthreads();
    const uint32_t neff = s_neff;
    if (neff == 0) {
        if (tid == 0) tree_size[s] = 0;
        return;
    }
    if (tid == 0) {
        bvh_node r;
        r.begin = 0;
        r.end = neff;
        r.left = r.right = -1;
        for (int d = 0; d < 4; ++d) r.lb[d] = INFINITY, r.ub[d] = -INFINITY;
        tree[0] = r;
        rope[0] = -1;
        ax[0] = 0;
    }
    __syncthreads();

    uint32_t lbeg = 0, lend = 1, nlev = 0;
    while (lbeg < lend) {
        if (nlev >= MAX_LEVELS) { // unreachable: depth <= 65 + 1
            if (tid == 0) set_error(st, ERR_CAPACITY, 0, 0, 0, 0);
            return;
        }
        if (tid == 0) lvl[nlev] = lbeg;
        ++nlev;
        // Phase 1: classify the level's nodes.
        for (uint32_t nd = lbeg + tid; nd < lend; nd += BVH_T) {
            bvh_node node = tree[nd];
            const uint32_t sp0 = ax[2 * nd];
            bool leaf = true;
            uint32_t nolc = 0, sp = sp0;
            if (node.end - node.begin > 1 && sp0 < 64) {
                const uint64_t x = mc[node.begin] ^ mc[node.end - 1];
                if (x != 0) {
                    sp = __clzll(x);
                    const uint64_t mask = 1ull << (63 - sp);
                    uint32_t lo = node.begin, hi = node.end;
                    while (lo < hi) {
                        const uint32_t mid = lo + (hi - lo) / 2;
                        if ((mc[mid] & mask) == 0) lo = mid + 1;
                        else hi = mid;
                    }
                    nolc = lo - node.begin;
                    leaf = false;
                } else {
                    sp = 64;
                }
            }
            if (leaf) {
                for (uint32_t o = node.begin; o < node.end; ++o) {
                    lof[o] = nd;
                    const float4 l = *reinterpret_cast<const float4 *>(sa + uint64_t(o) * 8);
                    const float4 u = *reinterpret_cast<const float4 *>(sa + uint64_t(o) * 8 + 4);
                    node.lb[0] = fmin_ref(node.lb[0], l.x);
                    node.lb[1] = fmin_ref(node.lb[1], l.y);
                    node.lb[2] = fmin_ref(node.lb[2], l.z);
                    node.lb[3] = fmin_ref(node.lb[3], l.w);
                    node.ub[0] = fmax_ref(node.ub[0], u.x);
                    node.ub[1] = fmax_ref(node.ub[1], u.y);
                    node.ub[2] = fmax_ref(node.ub[2], u.z);
                    node.ub[3] = fmax_ref(node.ub[3], u.w);
                }
                tree[nd] = node;
                ax[2 * nd + 1] = 0;
            } else {
                ax[2 * nd] = sp;
                ax[2 * nd + 1] = (nolc << 1) | 1u; // internal marker in bit 0
            }
        }
        __syncthreads();
        // Phase 2: children placement (exclusive scan of child counts).
        uint32_t carry = 0;
        for (uint32_t base = lbeg; base < lend; base += BVH_T) {
            const uint32_t nd = base + tid;
            const uint32_t info = (nd < lend) ? ax[2 * nd + 1] : 0;
            const uint32_t nc = (info & 1u) ? 2u : 0u;
            uint32_t tot;
            const uint32_t ex = block_excl_scan(nc, scan_smem, &tot);
            if (nc) {
                const uint32_t lc = lend + carry + ex;
                if (uint64_t(lc) + 1 >= cap) {
                    set_error(st, ERR_CAPACITY, 0, 0, 0, 0);
                } else {
                    bvh_node node = tree[nd];
                    const uint32_t nolc = info >> 1;
                    node.left = int32_t(lc);
                    node.right = int32_t(lc + 1);
                    tree[nd] = node;
                    bvh_node c;
                    c.left = c.right = -1;
                    for (int d = 0; d < 4; ++d) c.lb[d] = INFINITY, c.ub[d] = -INFINITY;
                    c.begin = node.begin;
                    c.end = node.begin + nolc;
                    tree[lc] = c;
                    c.begin = node.begin + nolc;
                    c.end = node.end;
                    tree[lc + 1] = c;
                    const uint32_t sp = ax[2 * nd];
                    ax[2 * lc] = sp + 1;
                    ax[2 * (lc + 1)] = sp + 1;
                    rope[lc] = int32_t(lc + 1);
                    rope[lc + 1] = rope[nd];
                }
            }
            carry += tot;
        }
        __syncthreads();
        lbeg = lend;
        lend = lend + carry;
        if (uint64_t(lend) > cap) { // unreachable: a radix tree has 2 n - 1 nodes
            if (tid == 0) set_error(st, ERR_CAPACITY, 0, 0, 0, 0);
            return;
        }
    }
    if (tid == 0) {
        lvl[nlev] = lend;
        s_nlev = nlev;
        tree_size[s] = lend;
    }
    __syncthreads();
    // Bottom-up boxes of internal nodes, level by level.
    for (int l = int(s_nlev) - 2; l >= 0; --l) {
        for (uint32_t nd = lvl[l] + tid; nd < lvl[l + 1]; nd += BVH_T) {
            bvh_node node = tree[nd];
            if (node.left == -1) continue;
            const bvh_node L = tree[node.left], R = tree[node.right];
            for (int d = 0; d < 4; ++d) {
                node.lb[d] = fmin_ref(L.lb[d], R.lb[d]);
                node.ub[d] = fmax_ref(L.ub[d], R.ub[d]);
            }
            tree[nd] = node;
        }
        __syncthreads();
    }
}

// Packs the per-step trees (stored at a fixed capacity per step) into one
// contiguous array at the given node offsets.
__global__ void k_tree_gather(const bvh_node *__restrict__ trees, uint64_t cap, const uint64_t *__restrict__ offs,
                              const uint32_t *__restrict__ sizes, bvh_node *__restrict__ out)
{
    const uint64_t s = blockIdx.x;
    const uint32_t n = sizes[s];
    const float4 *src = reinterpret_cast<const float4 *>(trees + s * cap);
    float4 *dst = reinterpret_cast<float4 *>(out + offs[s]);
    for (uint32_t k = threadIdx.x; k < 3 * n; k += blockDim.x) dst[k] = src[k];
}

void launch_tree_gather(const bvh_node *trees, uint64_t cap, const uint64_t *offs, const uint32_t *sizes,
                        uint64_t n_steps, bvh_node *out, cudaStream_t stream)
{
    if (n_steps) k_tree_gather<<<unsigned(n_steps), 256, 0, stream>>>(trees, cap, offs, sizes, out);
}

void launch_bvh(const float *srt_aabbs, const uint64_t *srt_mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                bvh_node *trees, uint64_t cap, int32_t *ropes, uint32_t *aux, uint32_t *leaf_of, uint32_t *tree_size,
                dev_status *st, cudaStream_t stream)
{
    k_bvh<<<nb, BVH_T, 0, stream>>>(srt_aabbs, srt_mcodes, s_first, N, trees, cap, ropes, aux, leaf_of, tree_size,
                                    st);
}

} // namespace mzb
