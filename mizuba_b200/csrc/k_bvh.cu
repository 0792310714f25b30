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

constexpr int MAX_LEVELS = 160;
// Dynamic shared memory for staged codes (216 KiB: 27,648 objects).
constexpr size_t BVH_SMEM_CODES = size_t(216) << 10;

// Nodes are 48 bytes at 16-byte-aligned addresses: move them as three
// 16-byte vectors instead of twelve 4-byte words.
__device__ __forceinline__ bvh_node load_node(const bvh_node *p)
{
    const float4 *v = reinterpret_cast<const float4 *>(p);
    const float4 a = v[0], b = v[1], c = v[2];
    bvh_node n;
    n.begin = __float_as_uint(a.x);
    n.end = __float_as_uint(a.y);
    n.left = __float_as_int(a.z);
    n.right = __float_as_int(a.w);
    n.lb[0] = b.x, n.lb[1] = b.y, n.lb[2] = b.z, n.lb[3] = b.w;
    n.ub[0] = c.x, n.ub[1] = c.y, n.ub[2] = c.z, n.ub[3] = c.w;
    return n;
}
__device__ __forceinline__ void store_node(bvh_node *p, const bvh_node &n)
{
    float4 *v = reinterpret_cast<float4 *>(p);
    v[0] = make_float4(__uint_as_float(n.begin), __uint_as_float(n.end), __int_as_float(n.left),
                       __int_as_float(n.right));
    v[1] = make_float4(n.lb[0], n.lb[1], n.lb[2], n.lb[3]);
    v[2] = make_float4(n.ub[0], n.ub[1], n.ub[2], n.ub[3]);
}

template <int BVH_T>
__global__ void __launch_bounds__(BVH_T, 1024 / BVH_T) k_bvh(const float *__restrict__ srt_aabbs,
                                               const uint64_t *__restrict__ srt_mcodes, uint32_t s_first,
                                               uint64_t N, bvh_node *__restrict__ trees, uint64_t cap,
                                               int32_t *__restrict__ ropes, uint32_t *__restrict__ aux,
                                               uint32_t *__restrict__ leaf_of, uint32_t *__restrict__ tree_size,
                                               dev_status *st, bool codes_in_smem)
{
    // With codes_in_smem the step's sorted codes are staged in dynamic shared
    // memory, so the split searches of every level read shared memory
    // instead of L2.
    extern __shared__ uint64_t smc[];
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
    const uint64_t *codes = mc;
    if (codes_in_smem) {
        for (uint32_t k = tid; k < neff; k += BVH_T) smc[k] = mc[k];
        codes = smc; // made visible by the barrier below
    }
    if (tid == 0) {
        bvh_node r;
        r.begin = 0;
        r.end = neff;
        r.left = r.right = -1;
        for (int d = 0; d < 4; ++d) r.lb[d] = INFINITY, r.ub[d] = -INFINITY;
        store_node(tree, r);
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
            bvh_node node = load_node(tree + nd);
            const uint32_t sp0 = ax[2 * nd];
            bool leaf = true;
            uint32_t nolc = 0, sp = sp0;
            if (node.end - node.begin > 1 && sp0 < 64) {
                const uint64_t x = codes[node.begin] ^ codes[node.end - 1];
                if (x != 0) {
                    sp = __clzll(x);
                    const uint64_t mask = 1ull << (63 - sp);
                    uint32_t lo = node.begin, hi = node.end;
                    while (lo < hi) {
                        const uint32_t mid = lo + (hi - lo) / 2;
                        if ((codes[mid] & mask) == 0) lo = mid + 1;
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
                store_node(tree + nd, node);
                ax[2 * nd + 1] = 0;
            } else {
                reinterpret_cast<uint2 *>(ax)[nd] = make_uint2(sp, (nolc << 1) | 1u); // internal marker in bit 0
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
                    const uint2 be = reinterpret_cast<const uint2 *>(tree + nd)[0];
                    const uint32_t nolc = info >> 1;
                    reinterpret_cast<int2 *>(tree + nd)[1] = make_int2(int32_t(lc), int32_t(lc + 1));
                    bvh_node c;
                    c.left = c.right = -1;
                    for (int d = 0; d < 4; ++d) c.lb[d] = INFINITY, c.ub[d] = -INFINITY;
                    c.begin = be.x;
                    c.end = be.x + nolc;
                    store_node(tree + lc, c);
                    c.begin = be.x + nolc;
                    c.end = be.y;
                    store_node(tree + lc + 1, c);
                    const uint32_t sp = ax[2 * nd];
                    reinterpret_cast<uint2 *>(ax)[lc] = make_uint2(sp + 1, 0);
                    reinterpret_cast<uint2 *>(ax)[lc + 1] = make_uint2(sp + 1, 0);
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
            const int2 lr = reinterpret_cast<const int2 *>(tree + nd)[1];
            if (lr.x == -1) continue;
            const float4 *Lv = reinterpret_cast<const float4 *>(tree + lr.x);
            const float4 *Rv = reinterpret_cast<const float4 *>(tree + lr.y);
            const float4 ll = Lv[1], lu = Lv[2], rl = Rv[1], ru = Rv[2];
            float4 *v = reinterpret_cast<float4 *>(tree + nd);
            v[1] = make_float4(fmin_ref(ll.x, rl.x), fmin_ref(ll.y, rl.y), fmin_ref(ll.z, rl.z), fmin_ref(ll.w, rl.w));
            v[2] = make_float4(fmax_ref(lu.x, ru.x), fmax_ref(lu.y, ru.y), fmax_ref(lu.z, ru.z), fmax_ref(lu.w, ru.w));
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

// threads: the CTA size, 256, 512 or 1024 (anything else: 1024).  Smaller
// CTAs fit several per SM, so more steps build at once, at the cost of more
// iterations on the wide levels of each tree.
void launch_bvh(const float *srt_aabbs, const uint64_t *srt_mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                bvh_node *trees, uint64_t cap, int32_t *ropes, uint32_t *aux, uint32_t *leaf_of, uint32_t *tree_size,
                dev_status *st, int threads, cudaStream_t stream)
{
    if (threads == 256)
        k_bvh<256><<<nb, 256, 0, stream>>>(srt_aabbs, srt_mcodes, s_first, N, trees, cap, ropes, aux, leaf_of,
                                           tree_size, st, false);
    else if (threads == 512)
        k_bvh<512><<<nb, 512, 0, stream>>>(srt_aabbs, srt_mcodes, s_first, N, trees, cap, ropes, aux, leaf_of,
                                           tree_size, st, false);
    else {
        // The 1,024-thread build runs one CTA per SM anyway: give it the
        // step's codes in shared memory when they fit.
        const size_t bytes = N * sizeof(uint64_t);
        const bool smem = bytes <= BVH_SMEM_CODES;
        k_bvh<1024><<<nb, 1024, smem ? bytes : 0, stream>>>(srt_aabbs, srt_mcodes, s_first, N, trees, cap, ropes,
                                                             aux, leaf_of, tree_size, st, smem);
    }
}

// Once per device (before any stream capture): allows the 1,024-thread build
// its dynamic shared memory for staged codes.
cudaError_t init_bvh_attrs()
{
    return cudaFuncSetAttribute(k_bvh<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(BVH_SMEM_CODES));
}

} // namespace mzb
