// Stage 2b of a conjunction step: order the objects by Morton code, objects
// without trajectory data last, ties by object index, then gather the sorted
// boxes and codes (mizuba/detect_conjunctions_morton.cpp:177-223).
//
// One 1024-thread CTA per conjunction step.  The comparator of the reference
// (no-data boxes after every finite box, then by code) is a 65-bit key; it is
// realised as a stable partition (finite first) followed by a stable LSD
// radix sort on the 64-bit code, so equal keys keep index order.  Each radix
// pass ranks a 1024-key tile with __match_any_sync on the 8-bit digit and a
// per-warp digit table in shared memory; passes whose digit is constant over
// the step are skipped.  The key/value ping-pong buffers are scratch memory
// of 2 x 12 bytes per object and step, resident in L2 for the CTA's lifetime.
#include "block.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace mzb
{

constexpr int SORT_T = 1024;

__global__ void __launch_bounds__(SORT_T) k_sort_step(const float *__restrict__ aabbs,
                                                      const uint64_t *__restrict__ mcodes, uint32_t s_first,
                                                      uint64_t N, uint64_t *keys_a, uint64_t *keys_b,
                                                      uint32_t *vals_a, uint32_t *vals_b, uint32_t *__restrict__ srt_idx,
                                                      uint64_t *__restrict__ srt_mcodes, float *__restrict__ srt_aabbs)
{
    // Per-digit, per-warp counts of the current tile, digit-major; the row is
    // padded to 33 words so the column scans below are conflict-free.
    __shared__ uint32_t wcnt[256][33];
    __shared__ uint32_t base[256], tilecnt[256], hist[256];
    __shared__ uint32_t scan_smem[33];
    __shared__ int skip;

    const uint32_t b = blockIdx.x;
    const uint64_t s = uint64_t(s_first) + b;
    const unsigned tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t *mc = mcodes + s * N;
    const float *ab = aabbs + s * (N + 1) * 8;
    uint64_t *kin = keys_a + uint64_t(b) * N, *kout = keys_b + uint64_t(b) * N;
    uint32_t *vin = vals_a + uint64_t(b) * N, *vout = vals_b + uint64_t(b) * N;

    // Stable partition: finite boxes first, each group in index order.
    uint32_t n_fin = 0;
    {
        uint32_t carry = 0;
        for (uint64_t t0 = 0; t0 < N; t0 += SORT_T) {
            const uint64_t i = t0 + tid;
            const uint32_t f = (i < N && isfinite(ab[i * 8])) ? 1u : 0u;
            uint32_t tot;
            block_excl_scan(f, scan_smem, &tot);
            carry += tot;
        }
        n_fin = carry;
        carry = 0;
        for (uint64_t t0 = 0; t0 < N; t0 += SORT_T) {
            const uint64_t i = t0 + tid;
            const uint32_t f = (i < N && isfinite(ab[i * 8])) ? 1u : 0u;
            uint32_t tot;
            const uint32_t ex = block_excl_scan(f, scan_smem, &tot);
            if (i < N) {
                const uint64_t fin_before = carry + ex;
                const uint64_t pos = f ? fin_before : n_fin + (i - fin_before);
                kin[pos] = mc[i];
                vin[pos] = uint32_t(i);
            }
            carry += tot;
        }
    }
    __syncthreads();

    for (int shift = 0; shift < 64; shift += 8) {
        if (tid < 256) hist[tid] = 0;
        __syncthreads();
        for (uint64_t i = tid; i < N; i += SORT_T) atomicAdd(&hist[(kin[i] >> shift) & 255u], 1u);
        __syncthreads();
        if (tid == 0) {
            int sk = 0;
            for (int d = 0; d < 256; ++d) sk |= (hist[d] == N);
            skip = sk;
        }
        __syncthreads();
        if (skip) continue; // digit constant: the pass is the identity
        // Exclusive scan of the 256-bin histogram (first 8 warps).
        if (tid < 256) {
            uint32_t x = hist[tid];
            const uint32_t v = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= unsigned(o)) x += y;
            }
            if (lane == 31) scan_smem[warp] = x;
            base[tid] = x - v;
        }
        __syncthreads();
        if (tid < 256) {
            uint32_t add = 0;
            for (unsigned w = 0; w < warp; ++w) add += scan_smem[w];
            base[tid] += add;
        }
        __syncthreads();
        for (uint64_t t0 = 0; t0 < N; t0 += SORT_T) {
            const uint64_t i = t0 + tid;
            const bool valid = i < N;
            const uint64_t key = valid ? kin[i] : 0;
            const uint32_t val = valid ? vin[i] : 0;
            const uint32_t d = valid ? uint32_t((key >> shift) & 255u) : 256u;
            uint32_t *wflat = &wcnt[0][0];
            for (unsigned z = tid; z < 256u * 33u; z += SORT_T) wflat[z] = 0;
            __syncthreads();
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const uint32_t rank = __popc(peers & lanemask_lt());
            if (valid && lane == unsigned(__ffs(peers) - 1)) wcnt[d][warp] = __popc(peers);
            __syncthreads();
            // Exclusive scan over the 32 warps of every digit column: warp w
            // takes digits 8w .. 8w + 7, lane l holds warp l's count.
#pragma unroll
            for (int z = 0; z < 8; ++z) {
                const unsigned dd = warp * 8 + z;
                const uint32_t c = wcnt[dd][lane];
                uint32_t x = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= unsigned(o)) x += y;
                }
                wcnt[dd][lane] = x - c;
                if (lane == 31) tilecnt[dd] = x;
            }
            __syncthreads();
            if (valid) {
                const uint32_t pos = base[d] + wcnt[d][warp] + rank;
                kout[pos] = key;
                vout[pos] = val;
            }
            __syncthreads();
            if (tid < 256) base[tid] += tilecnt[tid];
        }
        __syncthreads();
        uint64_t *kt = kin;
        kin = kout;
        kout = kt;
        uint32_t *vt = vin;
        vin = vout;
        vout = vt;
    }

    // Outputs: sorted indices and codes, gathered boxes, global box row.
    for (uint64_t p = tid; p < N; p += SORT_T) {
        const uint32_t o = vin[p];
        srt_idx[s * N + p] = o;
        srt_mcodes[s * N + p] = kin[p];
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
// into the allocator at all.  For them the key/value ping-pong buffers of the
// sort live in the file-scope array below: sized for NOALLOC_MAX_OBJS objects
// (24 bytes each, 12 MiB), it is part of this library's device image, so
// every GPU that loads the library holds it until the process exits.  All
// calls share it; calls whose kernels overlap on the GPU race on it.
constexpr uint64_t NOALLOC_MAX_OBJS = uint64_t(1) << 19;
static __device__ __align__(256) unsigned char g_sort_scratch[NOALLOC_MAX_OBJS * 24];

// Host-side address of g_sort_scratch on each device, set once per device
// (the name itself is only a host-side stand-in, not a device address).
static unsigned char *g_sort_scratch_addr[64];
static bool g_sort_scratch_init[64];

cudaError_t sort_step_noalloc(const float *aabbs, const uint64_t *mcodes, uint64_t n_objs, uint32_t *srt_idx,
                              uint64_t *srt_mcodes, float *srt_aabbs, cudaStream_t stream)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!g_sort_scratch_init[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_sort_scratch);
        if (e != cudaSuccess) return e;
        g_sort_scratch_addr[dev] = static_cast<unsigned char *>(ptr);
        g_sort_scratch_init[dev] = true;
    }
    unsigned char *base = g_sort_scratch_addr[dev];
    // Layout: keys_a [n] u64 | keys_b [n] u64 | vals_a [n] u32 | vals_b [n] u32.
    // Every element of these buffers is written before it is read, so nothing
    // needs clearing between calls.
    uint64_t *keys_a = reinterpret_cast<uint64_t *>(base);
    uint64_t *keys_b = keys_a + n_objs;
    uint32_t *vals_a = reinterpret_cast<uint32_t *>(keys_b + n_objs);
    uint32_t *vals_b = vals_a + n_objs;
    k_sort_step<<<1, SORT_T, 0, stream>>>(aabbs, mcodes, 0, n_objs, keys_a, keys_b, vals_a, vals_b, srt_idx,
                                          srt_mcodes, srt_aabbs);
    return cudaGetLastError();
}

uint64_t sort_noalloc_max_objs() { return NOALLOC_MAX_OBJS; }

void launch_sort(const float *aabbs, const uint64_t *mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                 uint64_t *keys_a, uint64_t *keys_b, uint32_t *vals_a, uint32_t *vals_b, uint32_t *srt_idx,
                 uint64_t *srt_mcodes, float *srt_aabbs, cudaStream_t stream)
{
    k_sort_step<<<nb, SORT_T, 0, stream>>>(aabbs, mcodes, s_first, N, keys_a, keys_b, vals_a, vals_b, srt_idx,
                                           srt_mcodes, srt_aabbs);
}

} // namespace mzb
