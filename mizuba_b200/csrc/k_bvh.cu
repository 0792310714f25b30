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
#include <algorithm>

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

// ---------------------------------------------------------------------------
// One-pass build.  The same tree, numbered the same way, without walking the
// levels top-down.  Over the sorted codes of a step, a "split" sits at every
// position i with code[i] != code[i + 1]; its bit is d(i) = clz(code[i] ^
// code[i + 1]).  Every internal node of the tree is the node split at one
// such position, its range being all positions whose codes share code[i]'s
// top d(i) bits (found by galloping searches); every leaf is a maximal run
// of equal codes.  The parent of a node [b, e) is the split at b - 1 or at
// e - 1, whichever has the larger d (the tighter prefix); the node is the
// parent's left child iff the parent splits at e - 1.
//
// The reference numbers nodes breadth first, siblings adjacent, each level
// in range order.  A split's depth is the number of splits whose range holds
// its own two positions, i.e. one less than the count of split ranges
// [b, e - 2] covering it: a difference array over positions and one block
// prefix sum.  A leaf sits one level below its parent.  The breadth-first
// index of an item is then its level's offset plus its rank among the
// level's items in position order (leaf at p before split at p): a stable
// multisplit by depth, each warp ranking a contiguous block of positions
// with bit ballots.  Children register with their parent, ropes follow from
// the ranges (the rope of [b, e) is the right child of the split at e - 1,
// or -1 when e is the end), leaf boxes fold their members, and internal
// boxes are the bottom-up union of their children's, one level at a time.
// std::min / std::max keep the first of equal values, so the union of a
// node equals the left-to-right fold over its range whatever the grouping,
// and the boxes are bit-identical to the reference's.
constexpr int FLAT_T = 1024;
constexpr int FLAT_W = FLAT_T / 32;
constexpr int FLAT_LEVELS = 66; // 64 split levels below the root at most, then leaves
constexpr int FLAT_G = 4;       // positions whose loads a thread issues together
constexpr uint32_t NOT_ITEM = 0xFFFFFFFEu, ROOT_PARENT = 0xFFFFFFFFu;

// Words of per-step scratch the one-pass build uses.
__host__ __device__ constexpr uint64_t flat_aux_words(uint64_t N) { return 12 * N + 16; }

__device__ __forceinline__ uint32_t split_bit(const uint64_t *c, uint32_t k) { return __clzll(c[k] ^ c[k + 1]); }

// Parent word of the node with range [b, e): ROOT_PARENT, or the parent split
// position shifted left by one with bit 0 set for a right child.
__device__ __forceinline__ uint32_t parent_word(const uint64_t *c, uint32_t b, uint32_t e, uint32_t neff)
{
    if (b == 0 && e == neff) return ROOT_PARENT;
    if (b == 0) return (e - 1) << 1;
    if (e == neff) return ((b - 1) << 1) | 1u;
    return split_bit(c, b - 1) > split_bit(c, e - 1) ? (((b - 1) << 1) | 1u) : ((e - 1) << 1);
}

__global__ void __launch_bounds__(FLAT_T, 1)
    k_bvh_flat(const float *__restrict__ srt_aabbs, const uint64_t *__restrict__ srt_mcodes, uint32_t s_first,
               uint64_t N, bvh_node *__restrict__ trees, uint64_t cap, int32_t *__restrict__ ropes,
               uint32_t *__restrict__ aux, uint32_t *__restrict__ leaf_of, uint32_t *__restrict__ tree_size,
               dev_status *st, bool codes_in_smem, bool depth_in_smem)
{
    extern __shared__ __align__(16) unsigned char fsm[];
    __shared__ uint32_t cnt[FLAT_W][FLAT_LEVELS];
    __shared__ uint32_t lvl_off[FLAT_LEVELS + 1];
    __shared__ uint32_t scan_smem[33];
    __shared__ uint32_t s_neff, s_bad;

    const uint32_t b = blockIdx.x;
    const uint64_t s = uint64_t(s_first) + b;
    const unsigned tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float *sa = srt_aabbs + s * (N + 1) * 8;
    const uint64_t *mc = srt_mcodes + s * N;
    bvh_node *tree = trees + s * cap;
    int32_t *rope = ropes + uint64_t(b) * cap;
    uint32_t *lof = leaf_of + uint64_t(b) * N;
    uint32_t *ax = aux + uint64_t(b) * flat_aux_words(N);
    uint32_t *par_s = ax, *par_l = ax + N, *rb = ax + 2 * N, *re = ax + 3 * N, *le = ax + 4 * N;
    int32_t *diff = reinterpret_cast<int32_t *>(ax + 5 * N);
    uint32_t *bfs_s = ax + 6 * N, *bfs_l = ax + 7 * N, *lc = ax + 8 * N;

    if (tid == 0) {
        uint64_t lo = 0, hi = N;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) / 2;
            if (!isinf(sa[mid * 8])) lo = mid + 1;
            else hi = mid;
        }
        s_neff = uint32_t(lo);
        s_bad = 0;
    }
    for (uint32_t k = tid; k < FLAT_W * FLAT_LEVELS; k += FLAT_T) (&cnt[0][0])[k] = 0;
    __syncthreads();
    const uint32_t neff = s_neff;
    if (neff == 0) {
        if (tid == 0) tree_size[s] = 0;
        return;
    }
    const uint64_t *codes = mc;
    if (codes_in_smem) {
        uint64_t *sc = reinterpret_cast<uint64_t *>(fsm);
        for (uint32_t k = tid; k < neff; k += FLAT_T) sc[k] = mc[k];
        codes = sc;
    }
    for (uint32_t k = tid; k < neff; k += FLAT_T) diff[k] = 0;
    __syncthreads();

    // Ranges and parents of every split and every leaf (run of equal codes).
    for (uint32_t p = tid; p < neff; p += FLAT_T) {
        const uint64_t cp = codes[p];
        // Leaf starting at p.
        if (p == 0 || codes[p - 1] != cp) {
            // End of the run: first k > p with a different code (galloping).
            uint32_t good = p, step = 1, bad = neff;
            while (good + step < neff) {
                if (codes[good + step] == cp) {
                    good += step;
                    step <<= 1;
                } else {
                    bad = good + step;
                    break;
                }
            }
            uint32_t lo = good + 1, hi = bad;
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo) / 2;
                if (codes[mid] == cp) lo = mid + 1;
                else hi = mid;
            }
            le[p] = lo;
            par_l[p] = parent_word(codes, p, lo, neff);
        } else {
            par_l[p] = NOT_ITEM;
        }
        // Split between p and p + 1.
        if (p + 1 < neff && codes[p + 1] != cp) {
            const int d = __clzll(cp ^ codes[p + 1]);
            uint32_t rbeg = 0, rend = neff;
            if (d > 0) {
                const uint64_t P = cp >> (64 - d);
                // First position with the prefix: gallop left from p.
                uint32_t good = p, step = 1;
                int64_t bad = -1;
                while (step <= good) {
                    if ((codes[good - step] >> (64 - d)) == P) {
                        good -= step;
                        step <<= 1;
                    } else {
                        bad = int64_t(good - step);
                        break;
                    }
                }
                uint32_t lo = uint32_t(bad + 1), hi = good;
                while (lo < hi) {
                    const uint32_t mid = lo + (hi - lo) / 2;
                    if ((codes[mid] >> (64 - d)) == P) hi = mid;
                    else lo = mid + 1;
                }
                rbeg = lo;
                // One past the last position with the prefix: gallop right
                // from p + 1 (which shares it).
                good = p + 1, step = 1;
                uint32_t badr = neff;
                while (good + step < neff) {
                    if ((codes[good + step] >> (64 - d)) == P) {
                        good += step;
                        step <<= 1;
                    } else {
                        badr = good + step;
                        break;
                    }
                }
                lo = good + 1, hi = badr;
                while (lo < hi) {
                    const uint32_t mid = lo + (hi - lo) / 2;
                    if ((codes[mid] >> (64 - d)) == P) lo = mid + 1;
                    else hi = mid;
                }
                rend = lo;
            }
            rb[p] = rbeg;
            re[p] = rend;
            par_s[p] = parent_word(codes, rbeg, rend, neff);
            // The split covers the split positions [rbeg, rend - 2].
            atomicAdd(diff + rbeg, 1);
            atomicAdd(diff + (rend - 1), -1);
        } else {
            par_s[p] = NOT_ITEM;
        }
    }
    __syncthreads(); // codes no longer read: the shared region is reused

    // Depths: prefix sum of the difference array (each thread a contiguous
    // chunk), split depth = cover - 1, leaf depth = parent's + 1.
    int32_t *dep = depth_in_smem ? reinterpret_cast<int32_t *>(fsm) : diff;
    unsigned char *ld = depth_in_smem ? fsm + 4 * uint64_t(N) : reinterpret_cast<unsigned char *>(ax + 9 * N);
    unsigned char *sd = ld + N;
    if (depth_in_smem)
        for (uint32_t k = tid; k < neff; k += FLAT_T) dep[k] = diff[k];
    __syncthreads();
    {
        const uint32_t chunk = (neff + FLAT_T - 1) / FLAT_T;
        const uint32_t c0 = min(neff, tid * chunk), c1 = min(neff, c0 + chunk);
        int32_t sum = 0;
        for (uint32_t k = c0; k < c1; ++k) sum += dep[k];
        uint32_t tot;
        int32_t run = int32_t(block_excl_scan(uint32_t(sum), scan_smem, &tot));
        for (uint32_t k = c0; k < c1; ++k) {
            run += dep[k];
            dep[k] = run - 1;
        }
    }
    __syncthreads();
    const uint32_t blk = (neff + FLAT_W - 1) / FLAT_W; // positions ranked by each warp
    for (uint32_t p = tid; p < neff; p += FLAT_T) {
        const uint32_t ws = par_s[p], wl = par_l[p];
        uint32_t ds = 0xFF, dl = 0xFF;
        if (ws != NOT_ITEM) ds = uint32_t(dep[p]);
        if (wl != NOT_ITEM) dl = (wl == ROOT_PARENT) ? 0u : uint32_t(dep[wl >> 1]) + 1;
        if ((ds != 0xFF && ds >= FLAT_LEVELS) || (dl != 0xFF && dl >= FLAT_LEVELS)) {
            s_bad = 1; // unreachable: codes have 64 bits
            ds = dl = 0xFF;
        }
        sd[p] = (unsigned char)ds;
        ld[p] = (unsigned char)dl;
        const uint32_t w = p / blk;
        if (ds != 0xFF) atomicAdd(&cnt[w][ds], 1u);
        if (dl != 0xFF) atomicAdd(&cnt[w][dl], 1u);
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0) set_error(st, ERR_CAPACITY, 0, 0, 0, 0);
        return;
    }
    // Level sizes, level offsets, and each warp's base within every level.
    if (tid < FLAT_LEVELS) {
        uint32_t t = 0;
        for (int w = 0; w < FLAT_W; ++w) t += cnt[w][tid];
        lvl_off[tid + 1] = t;
    }
    __syncthreads();
    if (tid == 0) {
        lvl_off[0] = 0;
        for (int l = 1; l <= FLAT_LEVELS; ++l) lvl_off[l] += lvl_off[l - 1];
    }
    __syncthreads();
    if (tid < FLAT_LEVELS) {
        uint32_t run = lvl_off[tid];
        for (int w = 0; w < FLAT_W; ++w) {
            const uint32_t c = cnt[w][tid];
            cnt[w][tid] = run;
            run += c;
        }
    }
    __syncthreads();
    const uint32_t total = lvl_off[FLAT_LEVELS];
    if (uint64_t(total) > cap) { // unreachable: a radix tree has 2 n - 1 nodes
        if (tid == 0) set_error(st, ERR_CAPACITY, 0, 0, 0, 0);
        return;
    }
    // Stable ranking: warp w walks positions [w blk, (w + 1) blk) 32 at a
    // time; an item's rank counts the earlier items of its level (leaf at p
    // before split at p) found by bit ballots over both kinds.
    {
        const uint32_t pb = min(neff, warp * blk), pe = min(neff, pb + blk);
        const unsigned lt = lanemask_lt(), gt = ~lt & ~(1u << lane);
        for (uint32_t c0 = pb; c0 < pe; c0 += 32) {
            const uint32_t p = c0 + lane;
            const bool in = p < pe;
            const uint32_t dl = in ? ld[p] : 0xFFu, ds = in ? sd[p] : 0xFFu;
            uint32_t bl[7], bs[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                bl[k] = __ballot_sync(0xffffffffu, (dl >> k) & 1u);
                bs[k] = __ballot_sync(0xffffffffu, (ds >> k) & 1u);
            }
            const uint32_t vl = __ballot_sync(0xffffffffu, dl != 0xFFu), vs = __ballot_sync(0xffffffffu, ds != 0xFFu);
            auto same = [&](uint32_t d, const uint32_t *bb, uint32_t m) {
#pragma unroll
                for (int k = 0; k < 7; ++k) m &= ((d >> k) & 1u) ? bb[k] : ~bb[k];
                return m;
            };
            uint32_t xl = 0, xs = 0;
            bool last_l = false, last_s = false;
            if (dl != 0xFFu) {
                const uint32_t mL = same(dl, bl, vl), mS = same(dl, bs, vs);
                xl = cnt[warp][dl] + __popc(mL & lt) + __popc(mS & lt);
                last_l = ((mL | mS) & gt) == 0 && ds != dl;
            }
            if (ds != 0xFFu) {
                const uint32_t mL = same(ds, bl, vl), mS = same(ds, bs, vs);
                xs = cnt[warp][ds] + __popc(mL & lt) + __popc(mS & lt) + (dl == ds ? 1u : 0u);
                last_s = ((mL | mS) & gt) == 0;
            }
            __syncwarp();
            if (last_l) cnt[warp][dl] = xl + 1;
            if (last_s) cnt[warp][ds] = xs + 1;
            __syncwarp();
            if (dl != 0xFFu) bfs_l[p] = xl;
            if (ds != 0xFFu) bfs_s[p] = xs;
        }
    }
    __syncthreads();
    // Left children register with their parents (right = left + 1).  Each
    // thread loads FLAT_G positions' inputs before using any of them, so that
    // many L2 round trips are in flight.
    for (uint32_t p0 = tid; p0 < neff; p0 += FLAT_T * FLAT_G) {
        uint32_t ws[FLAT_G], wl[FLAT_G], xs[FLAT_G], xl[FLAT_G];
#pragma unroll
        for (int g = 0; g < FLAT_G; ++g) {
            const uint32_t p = p0 + g * FLAT_T;
            ws[g] = wl[g] = NOT_ITEM;
            if (p < neff) ws[g] = par_s[p], wl[g] = par_l[p], xs[g] = bfs_s[p], xl[g] = bfs_l[p];
        }
#pragma unroll
        for (int g = 0; g < FLAT_G; ++g) {
            if (ws[g] < ROOT_PARENT - 1 && !(ws[g] & 1u)) lc[ws[g] >> 1] = xs[g];
            if (wl[g] < ROOT_PARENT - 1 && !(wl[g] & 1u)) lc[wl[g] >> 1] = xl[g];
        }
    }
    __syncthreads();
    // Nodes, ropes, leaf boxes and the leaf of every position; up[left
    // child] = node for the bottom-up pass (in shared memory when the codes
    // were).  One pass over the positions: under a full grid this phase is
    // bound by the L2 traffic of the node stores, and splitting it into
    // grouped passes measured slower.
    uint32_t *up = codes_in_smem ? reinterpret_cast<uint32_t *>(fsm) : ax + 10 * N;
    for (uint32_t p = tid; p < neff; p += FLAT_T) {
        if (par_s[p] != NOT_ITEM) {
            const uint32_t x = bfs_s[p], e = re[p], l = lc[p];
            // The box of an internal node is written by the bottom-up pass.
            reinterpret_cast<uint4 *>(tree + x)[0] = make_uint4(rb[p], e, l, l + 1);
            rope[x] = (e == neff) ? -1 : int32_t(lc[e - 1] + 1);
            up[l] = x;
        }
        if (par_l[p] != NOT_ITEM) {
            const uint32_t x = bfs_l[p], e = le[p];
            bvh_node n;
            n.begin = p;
            n.end = e;
            n.left = n.right = -1;
            for (int d = 0; d < 4; ++d) n.lb[d] = INFINITY, n.ub[d] = -INFINITY;
            for (uint32_t o = p; o < e; ++o) {
                lof[o] = x;
                const float4 lo = *reinterpret_cast<const float4 *>(sa + uint64_t(o) * 8);
                const float4 u = *reinterpret_cast<const float4 *>(sa + uint64_t(o) * 8 + 4);
                n.lb[0] = fmin_ref(n.lb[0], lo.x);
                n.lb[1] = fmin_ref(n.lb[1], lo.y);
                n.lb[2] = fmin_ref(n.lb[2], lo.z);
                n.lb[3] = fmin_ref(n.lb[3], lo.w);
                n.ub[0] = fmax_ref(n.ub[0], u.x);
                n.ub[1] = fmax_ref(n.ub[1], u.y);
                n.ub[2] = fmax_ref(n.ub[2], u.z);
                n.ub[3] = fmax_ref(n.ub[3], u.w);
            }
            store_node(tree + x, n);
            rope[x] = (e == neff) ? -1 : int32_t(lc[e - 1] + 1);
        }
    }
    if (tid == 0) tree_size[s] = total;
    __syncthreads();
    // Bottom-up boxes of internal nodes, level by level.  The children of
    // level l's internal nodes are level l + 1, pair by pair in parent order,
    // and up[] names each pair's parent: one round trip per level.
    int top = FLAT_LEVELS - 1;
    while (top > 0 && lvl_off[top] == lvl_off[top + 1]) --top;
    for (int l = top - 1; l >= 0; --l) {
        const uint32_t c0 = lvl_off[l + 1], npairs = (lvl_off[l + 2] - c0) / 2;
        for (uint32_t k = tid; k < npairs; k += FLAT_T) {
            const uint32_t j = c0 + 2 * k;
            const uint32_t x = up[j];
            const float4 *Lv = reinterpret_cast<const float4 *>(tree + j);
            const float4 *Rv = reinterpret_cast<const float4 *>(tree + j + 1);
            const float4 ll = Lv[1], lu = Lv[2], rl = Rv[1], ru = Rv[2];
            float4 *v = reinterpret_cast<float4 *>(tree + x);
            v[1] = make_float4(fmin_ref(ll.x, rl.x), fmin_ref(ll.y, rl.y), fmin_ref(ll.z, rl.z), fmin_ref(ll.w, rl.w));
            v[2] = make_float4(fmax_ref(lu.x, ru.x), fmax_ref(lu.y, ru.y), fmax_ref(lu.z, ru.z), fmax_ref(lu.w, ru.w));
        }
        __syncthreads();
    }
}

// Walk nodes from the finished trees: one thread per (step, node), so the
// 32-byte records are written whole and in order (written from inside the
// one-pass build, scattered and in two halves, they cost that kernel more
// than this pass takes).
__global__ void k_walk_nodes(const float *__restrict__ srt_aabbs, const bvh_node *__restrict__ trees, uint64_t cap,
                             const int32_t *__restrict__ ropes, const uint32_t *__restrict__ tree_size,
                             uint32_t s_first, uint64_t N, walk_node *__restrict__ walks)
{
    const uint32_t b = blockIdx.y;
    const uint64_t s = uint64_t(s_first) + b;
    const uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (k >= tree_size[s]) return;
    const walk_grid wg = make_walk_grid(srt_aabbs + (s * (N + 1) + N) * 8);
    const bvh_node nd = load_node(trees + s * cap + k);
    walk_node *w = walks + uint64_t(b) * cap + k;
    reinterpret_cast<uint4 *>(w)[0] = walk_box(nd.lb, nd.ub, wg);
    reinterpret_cast<int4 *>(w)[1] = make_int4(nd.left, ropes[uint64_t(b) * cap + k], int32_t(nd.begin), int32_t(nd.end));
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

// The level-by-level build with a CTA of 256, 512 or 1,024 threads.
void launch_bvh_levels(const float *srt_aabbs, const uint64_t *srt_mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                       bvh_node *trees, uint64_t cap, int32_t *ropes, uint32_t *aux, uint32_t *leaf_of,
                       uint32_t *tree_size, dev_status *st, int threads, cudaStream_t stream)
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

// threads: 256, 512 or 1024 select the level-by-level build with that CTA
// size (smaller CTAs fit several per SM, so more steps build at once, at the
// cost of more iterations on the wide levels of each tree); anything else
// selects the one-pass build.  Either way walks[b * cap + k] receives the
// walk node of node k of the batch's step b.
void launch_bvh(const float *srt_aabbs, const uint64_t *srt_mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                bvh_node *trees, uint64_t cap, int32_t *ropes, uint32_t *aux, uint32_t *leaf_of, uint32_t *tree_size,
                walk_node *walks, dev_status *st, int threads, cudaStream_t stream)
{
    if (threads == 256 || threads == 512 || threads == 1024) {
        launch_bvh_levels(srt_aabbs, srt_mcodes, s_first, nb, N, trees, cap, ropes, aux, leaf_of, tree_size, st,
                          threads, stream);
        k_walk_nodes<<<dim3(unsigned((cap + 255) / 256), nb), 256, 0, stream>>>(srt_aabbs, trees, cap, ropes,
                                                                                tree_size, s_first, N, walks);
        return;
    }
    // Codes (8 B per object) while ranges are searched, then depths (4 B)
    // and the two per-position level bytes, in shared memory when they fit;
    // global scratch otherwise.
    const bool csm = N * 8 <= BVH_SMEM_CODES, dsm = N * 6 <= BVH_SMEM_CODES;
    const size_t bytes = std::max(csm ? N * 8 : 0, dsm ? N * 6 : 0);
    k_bvh_flat<<<nb, FLAT_T, bytes, stream>>>(srt_aabbs, srt_mcodes, s_first, N, trees, cap, ropes, aux, leaf_of,
                                              tree_size, st, csm, dsm);
    k_walk_nodes<<<dim3(unsigned((cap + 255) / 256), nb), 256, 0, stream>>>(srt_aabbs, trees, cap, ropes, tree_size,
                                                                            s_first, N, walks);
}

// Scratch words per step of the batch that launch_bvh needs.
uint64_t bvh_aux_words(uint64_t N, uint64_t cap) { return std::max<uint64_t>(2 * cap, flat_aux_words(N)); }

// Once per device (before any stream capture): allows the 1,024-thread build
// its dynamic shared memory for staged codes.
cudaError_t init_bvh_attrs()
{
    const cudaError_t e =
        cudaFuncSetAttribute(k_bvh<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(BVH_SMEM_CODES));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_bvh_flat, cudaFuncAttributeMaxDynamicSharedMemorySize, int(BVH_SMEM_CODES));
}

} // namespace mzb
