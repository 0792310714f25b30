// Stage 2b of a conjunction step: order the objects by Morton code, objects
// without trajectory data last, ties by object index, then gather the sorted
// boxes and codes (mizuba/detect_conjunctions_morton.cpp:177-223).
//
// One 512-thread CTA per conjunction step.  The comparator of the reference
// (no-data boxes after every finite box, then by code) is realised as a
// stable partition (finite first, each group in index order) followed by a
// stable LSD radix sort on the code; boxes without data carry the code
// 2^64 - 1, so they stay behind every finite box.  Bits that are equal in
// every code of the step do not affect the order, so the codes are first
// compacted to their varying bits (passes whose digit is constant over the
// step are skipped; the 20,000-object catalogue varies in all 64 bits).  The
// prologue counts the finite boxes, finds the varying bits, stores every
// compacted key by original index and builds the histograms of every pass;
// each pass then moves original indices only, reading each one's digit from
// the stored keys, and ranks tiles of 4,096 (8 per thread, warp-striped so a
// warp's are consecutive) with bit ballots and per-warp digit counters in
// shared memory.  Scratch: the compacted keys (8 bytes per object and step)
// and the index ping-pong (2 x 4 bytes).  Moving indices alone keeps a step's
// working set at 320 KB, so under a full grid the resident steps' buffers fit
// the L2 (the key + index ping-pong took 480 KB and 1.62 against 1.34 ms for
// the day's sorts).
#include <mutex>

#include "block.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

constexpr int SORT_KPT = 8;

// SORT_T: 256 or 512 threads (the per-digit sections need at least 256).
template <int SORT_T>
__global__ void __launch_bounds__(SORT_T, 1024 / SORT_T) k_sort_step(const float *__restrict__ aabbs,
                                                         const uint64_t *__restrict__ mcodes, uint32_t s_first,
                                                         uint64_t N, uint64_t *keys_a,
                                                         uint32_t *vals_a, uint32_t *vals_b,
                                                         uint32_t *__restrict__ srt_idx,
                                                         uint64_t *__restrict__ srt_mcodes,
                                                         float *__restrict__ srt_aabbs)
{
    constexpr int SORT_W = SORT_T / 32;
    constexpr uint64_t SORT_TILE = uint64_t(SORT_T) * SORT_KPT;
    // Per-digit, per-warp counts of the current tile, digit-major; rows are
    // padded to an odd number of words so the per-digit scans are
    // conflict-free.
    __shared__ uint32_t wcnt[256][SORT_W + 1];
    __shared__ uint32_t hist[8][256];
    __shared__ uint8_t ctab[8][256]; // varying bits of each code byte, packed
    __shared__ uint32_t cshift[8];   // where each byte's packed bits go
    __shared__ uint32_t base[256], tilecnt[256], bscan[8], wtot[SORT_W];
    __shared__ unsigned long long vmask;
    __shared__ uint32_t nfin_s, skipmask;

    const uint32_t b = blockIdx.x;
    const uint64_t s = uint64_t(s_first) + b;
    const unsigned tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t *mc = mcodes + s * N;
    const float *ab = aabbs + s * (N + 1) * 8;
    // The passes move original indices only; each reads its key's digit from
    // the compacted keys stored by original index (a smaller working set per
    // step: under a full grid the resident steps' buffers then fit the L2).
    uint64_t *ckey = keys_a + uint64_t(b) * N;
    uint32_t *vin = vals_a + uint64_t(b) * N, *vout = vals_b + uint64_t(b) * N;

    // ---- Prologue 1: finite count and the mask of varying code bits.
    if (tid == 0) {
        vmask = 0;
        nfin_s = 0;
        skipmask = 0;
    }
    for (unsigned z = tid; z < 8u * 256u; z += SORT_T) (&hist[0][0])[z] = 0;
    __syncthreads();
    {
        const uint64_t c0 = N ? mc[0] : 0;
        uint64_t vm = 0;
        uint32_t nf = 0;
        for (uint64_t i = tid; i < N; i += SORT_T) {
            vm |= mc[i] ^ c0;
            nf += isfinite(ab[i * 8]) ? 1u : 0u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            vm |= __shfl_xor_sync(0xffffffffu, vm, o);
            nf += __shfl_xor_sync(0xffffffffu, nf, o);
        }
        if (lane == 0) {
            atomicOr(&vmask, (unsigned long long)vm);
            atomicAdd(&nfin_s, nf);
        }
    }
    __syncthreads();
    const uint64_t mask = vmask;
    const uint32_t n_fin = nfin_s;
    const int npass = (__popcll(mask) + 7) / 8;
    for (unsigned z = tid; z < 8u * 256u; z += SORT_T) {
        const unsigned j = z >> 8, v = z & 255u;
        const unsigned mb = unsigned(mask >> (8 * j)) & 255u;
        unsigned out = 0, k = 0;
        for (unsigned bit = 0; bit < 8; ++bit)
            if ((mb >> bit) & 1u) out |= ((v >> bit) & 1u) << k++;
        ctab[j][v] = uint8_t(out);
    }
    if (tid < 8) cshift[tid] = __popcll(mask & ((1ull << (8 * tid)) - 1ull));
    __syncthreads();

    // ---- Prologue 2: stable partition (finite first), compacted keys, and
    // the digit histograms of every pass.
    {
        uint32_t carry = 0;
        for (uint64_t t0 = 0; t0 < N; t0 += SORT_TILE) {
            const uint64_t wbase = t0 + uint64_t(warp) * 32 * SORT_KPT;
            uint32_t fcnt = 0, pre[SORT_KPT];
            uint64_t ck[SORT_KPT];
            unsigned fin = 0;
#pragma unroll
            for (int k = 0; k < SORT_KPT; ++k) {
                const uint64_t i = wbase + uint64_t(k) * 32 + lane;
                const bool valid = i < N;
                const bool f = valid && isfinite(ab[i * 8]);
                const unsigned bal = __ballot_sync(0xffffffffu, f);
                pre[k] = fcnt + __popc(bal & lanemask_lt());
                fcnt += __popc(bal);
                fin |= (f ? 1u : 0u) << k;
                uint64_t c = 0;
                if (valid) {
                    const uint64_t code = mc[i];
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        c |= uint64_t(ctab[j][unsigned(code >> (8 * j)) & 255u]) << cshift[j];
                    for (int ps = 0; ps < npass; ++ps) atomicAdd(&hist[ps][unsigned(c >> (8 * ps)) & 255u], 1u);
                }
                ck[k] = c;
            }
            if (lane == 0) wtot[warp] = fcnt;
            __syncthreads();
            uint32_t wpre = 0, ttot = 0;
#pragma unroll
            for (int w = 0; w < SORT_W; ++w) {
                const uint32_t v = wtot[w];
                wpre += (unsigned(w) < warp) ? v : 0u;
                ttot += v;
            }
#pragma unroll
            for (int k = 0; k < SORT_KPT; ++k) {
                const uint64_t i = wbase + uint64_t(k) * 32 + lane;
                if (i < N) {
                    const uint64_t fin_before = carry + wpre + pre[k];
                    const uint64_t pos = ((fin >> k) & 1u) ? fin_before : n_fin + (i - fin_before);
                    ckey[i] = ck[k]; // by original index: read back by the passes
                    vin[pos] = uint32_t(i);
                }
            }
            carry += ttot;
            __syncthreads();
        }
    }
    for (unsigned z = tid; z < 8u * 256u; z += SORT_T)
        if ((&hist[0][0])[z] == N) atomicOr(&skipmask, 1u << (z >> 8));
    __syncthreads();

    // ---- LSD radix passes over the compacted keys.
    for (int ps = 0; ps < npass; ++ps) {
        if ((skipmask >> ps) & 1u) continue; // digit constant: the pass is the identity
        const int shift = 8 * ps;
        if (tid < 256) {
            const uint32_t v = hist[ps][tid];
            uint32_t x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= unsigned(o)) x += y;
            }
            if (lane == 31) bscan[warp] = x;
            base[tid] = x - v;
        }
        __syncthreads();
        if (tid < 256) {
            uint32_t add = 0;
            for (unsigned w = 0; w < warp; ++w) add += bscan[w];
            base[tid] += add;
        }
        for (uint64_t t0 = 0; t0 < N; t0 += SORT_TILE) {
            for (unsigned z = tid; z < 256u * (SORT_W + 1); z += SORT_T) (&wcnt[0][0])[z] = 0;
            __syncthreads();
            const uint64_t wbase = t0 + uint64_t(warp) * 32 * SORT_KPT;
            uint64_t key[SORT_KPT];
            uint32_t val[SORT_KPT], rk[SORT_KPT];
            // All of the tile's loads first: the ranking below has a
            // __syncwarp per key, which loads cannot be moved across, so
            // loading inside it serialised one L2 round trip per key.
#pragma unroll
            for (int k = 0; k < SORT_KPT; ++k) {
                const uint64_t i = wbase + uint64_t(k) * 32 + lane;
                val[k] = (i < N) ? vin[i] : 0;
            }
#pragma unroll
            for (int k = 0; k < SORT_KPT; ++k) {
                const uint64_t i = wbase + uint64_t(k) * 32 + lane;
                key[k] = (i < N) ? ckey[val[k]] : 0;
            }
#pragma unroll
            for (int k = 0; k < SORT_KPT; ++k) {
                const uint64_t i = wbase + uint64_t(k) * 32 + lane;
                const bool valid = i < N;
                const unsigned d = valid ? unsigned(key[k] >> shift) & 255u : 256u;
                // Lanes holding the same digit, from one ballot per digit bit
                // (constant cost, where __match_any_sync slows down with the
                // number of distinct digits in the warp).
                const unsigned vb = __ballot_sync(0xffffffffu, valid);
                unsigned peers = valid ? vb : ~vb;
#pragma unroll
                for (int bit = 0; bit < 8; ++bit) {
                    const unsigned bb = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
                    peers &= ((d >> bit) & 1u) ? bb : ~bb;
                }
                const unsigned leader = __ffs(peers) - 1;
                uint32_t old = 0;
                if (valid && lane == leader) {
                    old = wcnt[d][warp];
                    wcnt[d][warp] = old + __popc(peers);
                }
                old = __shfl_sync(0xffffffffu, old, leader);
                rk[k] = old + __popc(peers & lanemask_lt());
                __syncwarp();
            }
            __syncthreads();
            // Exclusive scan over the warps of every digit row.
            if (tid < 256) {
                uint32_t run = 0;
#pragma unroll
                for (int w = 0; w < SORT_W; ++w) {
                    const uint32_t c = wcnt[tid][w];
                    wcnt[tid][w] = run;
                    run += c;
                }
                tilecnt[tid] = run;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < SORT_KPT; ++k) {
                const uint64_t i = wbase + uint64_t(k) * 32 + lane;
                if (i < N) {
                    const unsigned d = unsigned(key[k] >> shift) & 255u;
                    const uint32_t pos = base[d] + wcnt[d][warp] + rk[k];
                    vout[pos] = val[k];
                }
            }
            __syncthreads();
            if (tid < 256) base[tid] += tilecnt[tid];
        }
        __syncthreads();
        uint32_t *vt = vin;
        vin = vout;
        vout = vt;
    }

    // Outputs: sorted indices and codes, gathered boxes, global box row.
    for (uint64_t p = tid; p < N; p += SORT_T) {
        const uint32_t o = vin[p];
        srt_idx[s * N + p] = o;
        srt_mcodes[s * N + p] = mc[o];
        const float4 *src = reinterpret_cast<const float4 *>(ab + uint64_t(o) * 8);
        float4 *dst = reinterpret_cast<float4 *>(srt_aabbs + (s * (N + 1) + p) * 8);
        dst[0] = src[0];
        dst[1] = src[1];
    }
    if (tid < 2) {
        const float4 *src = reinterpret_cast<const float4 *>(ab + N * 8);
        float4 *dst = reinterpret_cast<float4 *>(srt_aabbs + (s * (N + 1) + N) * 8);
        dst[tid] = src[tid];
    }
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the step sort.
//
// Some callers cannot allocate device memory at the point where they sort:
// hosts that reserve all device memory for their own allocator at start-up
// and forbid cudaMalloc afterwards, or services whose hot loop must not call
// into the allocator at all.  For them the key and index buffers of the sort
// live in the file-scope array below: sized for NOALLOC_MAX_OBJS objects
// (16 bytes each: one 64-bit key and two 32-bit indices, 8 MiB), it is part
// of this library's device image, so every GPU that loads the library holds
// it until the process exits.  All calls share it; calls whose kernels
// overlap on the GPU race on it.
constexpr uint64_t NOALLOC_MAX_OBJS = uint64_t(1) << 19;
constexpr uint64_t NOALLOC_BYTES_PER_OBJ = sizeof(uint64_t) + 2 * sizeof(uint32_t);
static __device__ __align__(256) unsigned char g_sort_scratch[NOALLOC_MAX_OBJS * NOALLOC_BYTES_PER_OBJ];

// Device address of g_sort_scratch on each device, looked up once per device
// with that device current (in host code the array's name is only a
// stand-in, not a device address).  std::call_once makes the first calls of
// concurrent host threads on one device safe.
static unsigned char *g_sort_scratch_addr[64];
static cudaError_t g_sort_scratch_err[64];
static std::once_flag g_sort_scratch_once[64];

cudaError_t sort_step_noalloc(const float *aabbs, const uint64_t *mcodes, uint64_t n_objs, uint32_t *srt_idx,
                              uint64_t *srt_mcodes, float *srt_aabbs, cudaStream_t stream)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::call_once(g_sort_scratch_once[dev], [dev]() {
        void *ptr = nullptr;
        g_sort_scratch_err[dev] = cudaGetSymbolAddress(&ptr, g_sort_scratch);
        g_sort_scratch_addr[dev] = static_cast<unsigned char *>(ptr);
    });
    if (g_sort_scratch_err[dev] != cudaSuccess) return g_sort_scratch_err[dev];
    unsigned char *base = g_sort_scratch_addr[dev];
    // Layout: keys [n] u64 | vals_a [n] u32 | vals_b [n] u32.  Every element
    // of these buffers is written before it is read, so nothing needs
    // clearing between calls.
    uint64_t *keys_a = reinterpret_cast<uint64_t *>(base);
    uint32_t *vals_a = reinterpret_cast<uint32_t *>(keys_a + n_objs);
    uint32_t *vals_b = vals_a + n_objs;
    k_sort_step<512><<<1, 512, 0, stream>>>(aabbs, mcodes, 0, n_objs, keys_a, vals_a, vals_b, srt_idx,
                                          srt_mcodes, srt_aabbs);
    return cudaGetLastError();
}

uint64_t sort_noalloc_max_objs() { return NOALLOC_MAX_OBJS; }

// threads: the CTA size, 256 or 512 (anything else: 512).  Four 256-thread
// CTAs fit on an SM against two of 512, which matters when the batch holds
// between one and two waves of steps.
void launch_sort(const float *aabbs, const uint64_t *mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                 uint64_t *keys_a, uint32_t *vals_a, uint32_t *vals_b, uint32_t *srt_idx,
                 uint64_t *srt_mcodes, float *srt_aabbs, int threads, cudaStream_t stream)
{
    if (threads == 256)
        k_sort_step<256><<<nb, 256, 0, stream>>>(aabbs, mcodes, s_first, N, keys_a, vals_a, vals_b, srt_idx,
                                                 srt_mcodes, srt_aabbs);
    else
        k_sort_step<512><<<nb, 512, 0, stream>>>(aabbs, mcodes, s_first, N, keys_a, vals_a, vals_b, srt_idx,
                                                 srt_mcodes, srt_aabbs);
}

} // namespace mzb
