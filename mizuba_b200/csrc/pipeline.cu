// Host pipeline and C ABI (include/mizuba_b200.h).
//
// The reference driver (mizuba/detect_conjunctions.cpp:53-537) runs the five
// stages per conjunction step on CPU threads, chunked by 128 steps, and
// streams variable-size outputs to files through a writer thread.  Here the
// steps are processed in batches (all of a batch's steps in every launch):
//   aabb -> global box -> morton -> sort/gather -> bvh -> broad count ->
//   scan -> broad write -> narrow -> roots -> per-step conj order
// on one CUDA stream, with three host synchronisations per batch (to size the
// pair list, the root queue and the conjunction list).  All outputs stay in
// HBM until the caller copies them out.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

using namespace mzb;

namespace
{

thread_local std::string g_err;

struct invalid_arg : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
struct out_of_range_err : std::out_of_range {
    using std::out_of_range::out_of_range;
};

[[noreturn]] void cuda_fail(cudaError_t e, const char *what)
{
    throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
#define CK(x)                                                                                                        \
    do {                                                                                                               \
        const cudaError_t e_ = (x);                                                                                    \
        if (e_ != cudaSuccess) cuda_fail(e_, #x);                                                                      \
    } while (0)

// Device buffers come from the device's stream-ordered memory pool, whose
// release threshold is raised once so that freed blocks stay cached: repeated
// screening calls then allocate without going back to the driver.  A buffer
// is allocated and freed on one stream (stream-ordered); result buffers are
// switched to stream 0 once the call's own stream has drained.
void ensure_pool()
{
    static std::once_flag flags[64];
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::call_once(flags[dev & 63], [dev]() {
        cudaMemPool_t pool;
        CK(cudaDeviceGetDefaultMemPool(&pool, dev));
        uint64_t thr = ~0ull;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    });
}

// Batch scratch kept between screening calls, one set of blocks per device.
// Every call allocates the same few dozen scratch buffers of a few GB in
// total; drawn from the stream-ordered pool afresh each time, their changing
// mix (plain and mixed form, different batch sizes) fragments the pool, and
// a call that finds no cached block that fits waits for the driver to map
// new memory (measured at 0.5 to 1 s per call).  Cached per role instead,
// each block only grows, so steady-state calls allocate nothing.  A call
// holds the device's set for its whole duration; a concurrent call on the
// same device finds it taken and uses private buffers.
struct scratch_slot {
    void *p = nullptr;
    size_t bytes = 0;
};
constexpr int SCRATCH_SLOTS = 64;
struct scratch_cache {
    std::mutex m;
    scratch_slot slots[SCRATCH_SLOTS];
    // The pinned host area of the per-batch read-backs (host_mailbox), kept
    // between calls: pinning memory costs milliseconds per call.
    char *mbox_h = nullptr, *mbox_d = nullptr;
    size_t mbox_bytes = 0;
    // The block of the per-step outputs of the last freed result, handed to
    // the next call that needs no more: a result of the same workload then
    // allocates nothing (the pool mapped new memory for it, 12-16 ms, when
    // polyjectories were created and freed between calls).
    std::mutex spare_m;
    void *spare = nullptr;
    size_t spare_bytes = 0;
    // The call's screening and copy streams and its events, created once:
    // creating them per call goes through the driver, where a concurrent
    // query of the GPU (a clock monitor, say) can hold it up.
    cudaStream_t st = nullptr, cs = nullptr;
    cudaEvent_t ev[16] = {};
    cudaEvent_t ev_nt[2] = {};
};
scratch_cache &device_scratch_of(int dev)
{
    static scratch_cache caches[64];
    return caches[dev & 63];
}
scratch_cache &device_scratch()
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    return device_scratch_of(dev);
}
// The device's cached set for one call (or nothing, when another call holds
// it); next() hands out the slots in declaration order, the same each call.
struct scratch_lease {
    std::unique_lock<std::mutex> lk;
    scratch_cache *cache = nullptr;
    scratch_slot *slots = nullptr;
    int used = 0;
    scratch_lease()
    {
        scratch_cache &c = device_scratch();
        lk = std::unique_lock<std::mutex>(c.m, std::try_to_lock);
        if (lk.owns_lock()) {
            cache = &c;
            slots = c.slots;
        }
    }
    scratch_slot *next() { return (slots && used < SCRATCH_SLOTS) ? &slots[used++] : nullptr; }
};

// The spare output block of device dev: taken when it holds at least bytes.
void *take_spare(int dev, size_t bytes, size_t &got)
{
    scratch_cache &c = device_scratch_of(dev);
    std::lock_guard<std::mutex> lk(c.spare_m);
    if (!c.spare || c.spare_bytes < bytes) return nullptr;
    void *p = c.spare;
    got = c.spare_bytes;
    c.spare = nullptr;
    c.spare_bytes = 0;
    return p;
}
// A freed result's block becomes the spare (the larger of it and the
// current spare is kept; the other goes back to the pool).
void give_spare(int dev, void *p, size_t bytes)
{
    scratch_cache &c = device_scratch_of(dev);
    void *drop = nullptr;
    {
        std::lock_guard<std::mutex> lk(c.spare_m);
        if (c.spare && c.spare_bytes >= bytes) {
            drop = p;
        } else {
            drop = c.spare;
            c.spare = p;
            c.spare_bytes = bytes;
        }
    }
    if (drop) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(dev);
        cudaFreeAsync(drop, 0);
        cudaSetDevice(cur);
    }
}

template <typename T>
struct dbuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t fs = 0; // stream the block is freed on
    scratch_slot *sl = nullptr; // cached block backing this buffer, if any
    bool borrowed = false;      // a view into a block another buffer owns
    dbuf() = default;
    explicit dbuf(scratch_slot *slot) : sl(slot) {}
    dbuf(const dbuf &) = delete;
    dbuf &operator=(const dbuf &) = delete;
    ~dbuf() { release(); }
    void release()
    {
        if (p && !sl && !borrowed) cudaFreeAsync(p, fs);
        p = nullptr;
        n = 0;
        borrowed = false;
    }
    // A view of count elements at q, owned elsewhere.
    void borrow(T *q, size_t count)
    {
        release();
        p = q;
        n = count;
        borrowed = true;
    }
    void alloc(size_t count, cudaStream_t s)
    {
        release();
        fs = s;
        if (count == 0) return;
        ensure_pool();
        const size_t bytes = count * sizeof(T);
        if (sl) {
            // A cached block grows (stream-ordered) and is never shrunk.
            if (sl->bytes < bytes) {
                if (sl->p) CK(cudaFreeAsync(sl->p, s));
                sl->p = nullptr;
                sl->bytes = 0;
                CK(cudaMallocAsync(&sl->p, bytes, s));
                sl->bytes = bytes;
            }
            p = static_cast<T *>(sl->p);
            n = count;
            return;
        }
        CK(cudaMallocAsync(reinterpret_cast<void **>(&p), bytes, s));
        n = count;
    }
    // A queue of at least count entries: a cached block larger than that
    // (grown by an earlier call) is used whole, so a call whose queues the
    // earlier calls have outgrown once does not overflow them again.
    void alloc_queue(size_t count, cudaStream_t s)
    {
        alloc(count, s);
        if (sl && p) n = std::max(n, sl->bytes / sizeof(T));
    }
    // Grows to at least count elements, keeping the first keep elements.
    void grow(size_t count, size_t keep, cudaStream_t s)
    {
        if (count <= n) return;
        const size_t nn = std::max(count, n + n / 2);
        T *q = nullptr;
        ensure_pool();
        CK(cudaMallocAsync(reinterpret_cast<void **>(&q), nn * sizeof(T), s));
        if (keep) CK(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
        if (p) cudaFreeAsync(p, fs);
        p = q;
        n = nn;
        fs = s;
    }
};

std::string fmt_d(double x)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.17g", x);
    return buf;
}

// A host-readable view of a caller array: the array itself when it is host
// memory (pageable, pinned or managed), else a host copy of the device array.
// When the runtime cannot classify the pointer (no CUDA device at all, or an
// unregistered pointer) it is host memory.
template <typename T>
const T *host_view(const T *p, uint64_t n, std::vector<T> &keep)
{
    if (n == 0 || p == nullptr) return p;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, p) != cudaSuccess) {
        cudaGetLastError();
        return p;
    }
    if (pa.type != cudaMemoryTypeDevice) return p;
    keep.resize(n);
    CK(cudaMemcpy(keep.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost));
    return keep.data();
}

std::once_flag g_init_flags[64];

void init_device_consts()
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::call_once(g_init_flags[dev & 63], []() {
        CK(init_aabb_consts());
        CK(init_narrow_consts());
        CK(init_bvh_attrs());
    });
}

} // namespace

namespace
{

// ---- Staged upload (mzb_pj_create_async from pageable memory).
//
// The polyjectory arrives in time chunks so that screening can start on the
// first steps while the rest is in flight.  A chunk holds, for every object,
// the segments that start in its share of [0, maxT): ranges scattered over
// the caller's object-major array.  Host threads pack them into pieces of at
// most STAGE_SLOT_BYTES in pinned memory, the copy engine moves each piece to
// a device staging buffer and k_relayout_runs puts its segments in place.
// Every byte crosses host memory three times (read, packed, read by the copy
// engine), so the host's memory bandwidth bounds it: on the benchmark's host
// the day's 1.93 GB took 53 ms with 16 threads and 69 ms with 8, against
// 44 ms for the kernel that gathers pinned memory directly (which pinned
// callers get instead).
constexpr size_t STAGE_SLOT_BYTES = size_t(16) << 20;
constexpr uint64_t STAGE_MAX_RUNS = 8192;

struct stage_piece {
    uint64_t run_begin, run_end; // into stager::runs
    uint64_t n_seg;              // segments in the piece's data
};

// Pinned host slots kept by the process between uploads (pinning memory
// costs about as long as copying it).
struct pinned_slots {
    std::mutex m;
    std::vector<char *> free;
    char *take()
    {
        {
            std::lock_guard<std::mutex> lk(m);
            if (!free.empty()) {
                char *p = free.back();
                free.pop_back();
                return p;
            }
        }
        char *p = nullptr;
        CK(cudaHostAlloc(reinterpret_cast<void **>(&p), STAGE_SLOT_BYTES, cudaHostAllocPortable));
        return p;
    }
    void give(char *p)
    {
        std::lock_guard<std::mutex> lk(m);
        free.push_back(p);
    }
};
pinned_slots &stage_slots()
{
    static pinned_slots s;
    return s;
}

struct stager {
    int dev = 0;
    const double *traj = nullptr;
    uint64_t per_src = 0;
    int op1 = 0;
    double *coef = nullptr;
    unsigned long long *bad_seg = nullptr;
    std::vector<stage_run> runs;
    std::vector<stage_piece> pieces;
    std::vector<double> lo;          // chunk c: segments starting in [lo[c], lo[c + 1])
    std::vector<uint64_t> chunk_end; // pieces [0, chunk_end[c]) hold chunks 0..c
    std::vector<cudaEvent_t> piece_ev;
    std::mutex m;
    std::condition_variable cv;
    std::vector<char> done; // piece enqueued (copy, relayout and its event)
    uint64_t prefix = 0;    // pieces [0, prefix) are all enqueued
    std::string error;
    std::atomic<bool> abort{false};
    std::vector<std::thread> workers;

    stager() = default;
    stager(const stager &) = delete;
    stager &operator=(const stager &) = delete;
    ~stager()
    {
        join();
        for (cudaEvent_t e : piece_ev) cudaEventDestroy(e);
    }
    void join()
    {
        for (std::thread &t : workers)
            if (t.joinable()) t.join();
        workers.clear();
    }
    void start(unsigned n_workers)
    {
        done.assign(pieces.size(), 0);
        piece_ev.resize(pieces.size(), nullptr);
        for (cudaEvent_t &e : piece_ev) CK(cudaEventCreate(&e)); // timed: the call trace reads them
        n_workers = std::max(1u, std::min<unsigned>(n_workers, unsigned(std::max<size_t>(1, pieces.size()))));
        for (unsigned w = 0; w < n_workers; ++w) workers.emplace_back([this, w, n_workers]() { run(w, n_workers); });
    }
    // Worker w packs pieces w, w + W, ... through two pinned slots and two
    // device slots, each on its own stream: a slot is refilled once the copy
    // that read it has finished.
    void run(unsigned w, unsigned W)
    {
        cudaStream_t s = nullptr;
        cudaEvent_t fe[2] = {nullptr, nullptr};
        char *h[2] = {nullptr, nullptr};
        char *d[2] = {nullptr, nullptr};
        // Host-clock totals of the worker's phases, printed under MZB_TRACE.
        const bool trace = std::getenv("MZB_TRACE") != nullptr;
        using clk = std::chrono::steady_clock;
        const clk::time_point t_start = clk::now();
        double ms_wait = 0, ms_pack = 0, ms_issue = 0;
        uint64_t bytes = 0, n_done = 0;
        auto ms_since = [](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
        try {
            CK(cudaSetDevice(dev));
            int lo_prio = 0, hi_prio = 0;
            CK(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
            CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, hi_prio));
            for (cudaEvent_t &e : fe) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            unsigned k = 0;
            for (uint64_t j = w; j < pieces.size() && !abort.load(); j += W, ++k) {
                const int sl = int(k & 1u);
                clk::time_point t0 = clk::now();
                if (!h[sl]) {
                    h[sl] = stage_slots().take();
                    ensure_pool();
                    CK(cudaMallocAsync(reinterpret_cast<void **>(&d[sl]), STAGE_SLOT_BYTES, s));
                } else {
                    CK(cudaEventSynchronize(fe[sl]));
                }
                ms_wait += ms_since(t0);
                t0 = clk::now();
                const stage_piece &pc = pieces[j];
                const uint64_t nr = pc.run_end - pc.run_begin;
                const uint64_t data_off = 16 + nr * sizeof(stage_run);
                uint64_t *hdr = reinterpret_cast<uint64_t *>(h[sl]);
                hdr[0] = nr;
                hdr[1] = data_off;
                std::memcpy(h[sl] + 16, runs.data() + pc.run_begin, nr * sizeof(stage_run));
                double *dd = reinterpret_cast<double *>(h[sl] + data_off);
                for (uint64_t r = pc.run_begin; r < pc.run_end; ++r) {
                    const stage_run &rn = runs[r];
                    std::memcpy(dd + uint64_t(rn.src_seg) * per_src, traj + rn.dst_seg * per_src,
                                uint64_t(rn.n_seg) * per_src * sizeof(double));
                }
                ms_pack += ms_since(t0);
                t0 = clk::now();
                bytes += pc.n_seg * per_src * sizeof(double);
                ++n_done;
                CK(cudaMemcpyAsync(d[sl], h[sl], data_off + pc.n_seg * per_src * sizeof(double),
                                   cudaMemcpyHostToDevice, s));
                CK(cudaEventRecord(fe[sl], s));
                launch_relayout_runs(d[sl], nr, coef, op1, bad_seg, s);
                CK(cudaGetLastError());
                CK(cudaEventRecord(piece_ev[j], s));
                ms_issue += ms_since(t0);
                {
                    std::lock_guard<std::mutex> lk(m);
                    done[j] = 1;
                    while (prefix < done.size() && done[prefix]) ++prefix;
                }
                cv.notify_all();
            }
            CK(cudaStreamSynchronize(s));
            if (trace)
                std::fprintf(stderr,
                             "[mizuba_b200] upload worker %u: %llu pieces, %.1f MB packed in %.3f ms (%.1f GB/s), "
                             "waits %.3f ms, copy issue %.3f ms, done after %.3f ms\n",
                             w, (unsigned long long)n_done, bytes / 1e6, ms_pack, bytes / 1e6 / std::max(ms_pack, 1e-9),
                             ms_wait, ms_issue, ms_since(t_start));
        } catch (const std::exception &e) {
            {
                std::lock_guard<std::mutex> lk(m);
                if (error.empty()) error = e.what();
            }
            abort.store(true);
            cv.notify_all();
        }
        if (s) cudaStreamSynchronize(s);
        for (int sl = 0; sl < 2; ++sl) {
            if (d[sl]) cudaFreeAsync(d[sl], s);
            if (h[sl]) stage_slots().give(h[sl]);
        }
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        for (cudaEvent_t e : fe)
            if (e) cudaEventDestroy(e);
    }
    // Blocks until pieces [0, n) are enqueued; a worker's error is rethrown.
    void wait_enqueued(uint64_t n)
    {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&]() { return prefix >= n || !error.empty(); });
        if (!error.empty()) throw std::runtime_error("polyjectory upload failed: " + error);
    }
    // Makes `stream` wait for pieces [0, n) (their events are recorded once
    // they are enqueued).
    void wait_stream(cudaStream_t stream, uint64_t n)
    {
        wait_enqueued(n);
        for (uint64_t j = 0; j < n; ++j) CK(cudaStreamWaitEvent(stream, piece_ev[j], 0));
    }
    uint64_t pieces_for(double t_end) const
    {
        size_t c = 0;
        while (c + 1 < lo.size() && lo[c + 1] < t_end) ++c;
        return chunk_end[c];
    }
};

} // namespace

struct mzb_pj {
    int order = 0;
    uint64_t n_objs = 0, n_seg = 0;
    double maxT = 0;
    dbuf<double> coef, time;
    dbuf<uint64_t> seg_off, time_off;
    dbuf<uint32_t> nseg;
    // Lowest segment with a non-finite coefficient (all ones: none), written
    // by the upload kernels; h_seg_off / h_nseg map it back to its object.
    dbuf<unsigned long long> bad_seg;
    std::vector<uint64_t> h_seg_off, h_time_off;
    std::vector<uint32_t> h_nseg;
    // Asynchronous upload (mzb_pj_create_async): the coefficients arrive by
    // time chunk, gathered by a kernel on the stream `up` from pinned memory
    // (chunk c holds the segments starting in [up_lo[c], up_lo[c + 1]) and
    // is complete when up_ev[c] has fired), or packed and copied by the
    // staged upload `stg` from pageable memory.
    cudaStream_t up = nullptr;
    std::vector<cudaEvent_t> up_ev;
    std::vector<double> up_lo;
    std::unique_ptr<stager> stg;
    bool async_upload() const { return up || stg; }
    // Makes `stream` wait for every chunk a segment starting before t_end
    // needs (the gather's chunks run in order on one stream, so the last
    // such chunk's event).
    void wait_upload(cudaStream_t stream, double t_end) const
    {
        if (stg) stg->wait_stream(stream, stg->pieces_for(t_end));
        if (up_ev.empty()) return;
        size_t c = 0;
        while (c + 1 < up_ev.size() && up_lo[c + 1] < t_end) ++c;
        CK(cudaStreamWaitEvent(stream, up_ev[c], 0));
    }
    void wait_upload_all(cudaStream_t stream) const
    {
        if (stg) stg->wait_stream(stream, stg->pieces.size());
        if (!up_ev.empty()) CK(cudaStreamWaitEvent(stream, up_ev.back(), 0));
    }
    // Blocks the host until the whole upload has landed.
    void wait_upload_host() const
    {
        if (up) CK(cudaStreamSynchronize(up));
        if (!stg) return;
        stg->wait_enqueued(stg->pieces.size());
        for (cudaEvent_t e : stg->piece_ev) CK(cudaEventSynchronize(e));
    }
    // The reference's error for a non-finite trajectory value
    // (polyjectory.cpp:558-569), given the flag read back from bad_seg.
    void throw_if_bad(unsigned long long seg) const
    {
        if (seg == ~0ull) return;
        uint64_t obj = 0;
        for (uint64_t i = 0; i < n_objs; ++i)
            if (seg >= h_seg_off[i] && seg < h_seg_off[i] + h_nseg[i]) {
                obj = i;
                break;
            }
        throw std::invalid_argument("A non-finite value was found in the trajectory at index " + std::to_string(obj));
    }
    // Reads the flag on `stream` (after the work it has waited for).
    void check_data(cudaStream_t stream) const
    {
        unsigned long long h = ~0ull;
        CK(cudaMemcpyAsync(&h, bad_seg.p, sizeof(h), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        throw_if_bad(h);
    }
    ~mzb_pj()
    {
        stg.reset(); // waits for the staged upload's workers before the buffers go
        if (up) cudaStreamSynchronize(up);
        for (cudaEvent_t e : up_ev) cudaEventDestroy(e);
        if (up) cudaStreamDestroy(up);
    }
    dev_pj view() const
    {
        dev_pj v;
        v.order = order;
        v.op1 = order + 1;
        v.n_objs = n_objs;
        v.maxT = maxT;
        v.coef = coef.p;
        v.time = time.p;
        v.seg_off = seg_off.p;
        v.time_off = time_off.p;
        v.nseg = nseg.p;
        return v;
    }
};

struct mzb_result {
    uint64_t n_cd_steps = 0, n_objs = 0, cap = 0;
    uint64_t step_begin = 0, n_run = 0, n_launches = 0;
    std::vector<double> cd_end;
    // The per-step outputs below are views into one device block, which
    // becomes the device's spare output block when the result is freed (the
    // next call of the same workload then allocates nothing).
    void *block = nullptr;
    size_t block_bytes = 0;
    int dev = 0;
    dbuf<float> aabbs, srt_aabbs;
    dbuf<uint64_t> mcodes, srt_mcodes;
    dbuf<uint32_t> srt_idx, tree_size;
    dbuf<bvh_node> trees;
    dbuf<uint2> bp;
    uint64_t n_bp = 0;
    std::vector<uint64_t> bp_off; // [S][2]
    dbuf<conj_rec> conj;
    uint64_t n_conj = 0;
    uint64_t np[7] = {};
    uint64_t narrow_split[2] = {}; // mixed form: items past the screen, past the prefilter
    double stage_ms[8] = {};
    uint64_t broad_visits = 0; // node visits of the default broad-phase walk
    mzb_result() = default;
    mzb_result(const mzb_result &) = delete;
    mzb_result &operator=(const mzb_result &) = delete;
    ~mzb_result()
    {
        if (block) give_spare(dev, block, block_bytes);
    }
};

namespace
{

// Reference message for a device status word.
std::string status_message(const dev_status &s)
{
    switch (s.code) {
    case ERR_AABB_LB:
        return "The computation of the bounding box for the object at index " + std::to_string(s.a)
               + " produced the non-finite lower bound " + fmt_d(s.x);
    case ERR_AABB_UB:
        return "The computation of the bounding box for the object at index " + std::to_string(s.a)
               + " produced the non-finite upper bound " + fmt_d(s.x);
    case ERR_GLOBAL_AABB:
        return "A global bounding box with non-finite size was generated";
    case ERR_NP_INTERVAL:
        return "During the narrow phase collision detection of objects " + std::to_string(s.a) + " and "
               + std::to_string(s.b) + ", an invalid time interval for polynomial root finding was generated";
    case ERR_NP_NONFINITE:
        return "Non-finite value(s) detected during conjunction tracking for objects " + std::to_string(s.a) + " and "
               + std::to_string(s.b);
    case ERR_ISOLATION:
        return "The polynomial root isolation algorithm failed: the working list size is "
               + std::to_string(uint64_t(s.x)) + " and the number of isolating intervals is "
               + std::to_string(uint64_t(s.y));
    case ERR_TOMS_ITER:
        return "Polynomial root finding failed due to too many iterations";
    case ERR_TOMS_ERRNO:
        return "Polynomial root finding returned a nonzero errno with code '" + std::to_string(int(s.x)) + "'";
    case ERR_ROOT_NONFINITE:
        return "Polynomial root finding produced a non-finite root of " + fmt_d(s.x) + " involving objects "
               + std::to_string(s.a) + " and " + std::to_string(s.b);
    case ERR_ROOT_DER:
        return "Polynomial root finding produced the root " + fmt_d(s.x) + " with nonfinite derivative "
               + fmt_d(s.y) + " involving objects " + std::to_string(s.a) + " and " + std::to_string(s.b);
    case ERR_CONJ_D2:
        return "A non-finite conjunction distance square of " + fmt_d(s.x)
               + " was computed for the objects at indices " + std::to_string(s.a) + " and " + std::to_string(s.b);
    case ERR_UB_DER:
        return "An invalid value of " + fmt_d(s.x)
               + " was computed for the derivative of the distance square function at the upper boundary of a "
                 "trajectory";
    case ERR_UB_D2:
        return "An invalid value of " + fmt_d(s.x)
               + " was computed for a candidate minimum of the distance square function at the upper boundary of a "
                 "trajectory";
    case ERR_LB_DER:
        return "An invalid value of " + fmt_d(s.x)
               + " was computed for the derivative of the distance square function at the lower boundary of a "
                 "trajectory";
    case ERR_LB_D2:
        return "An invalid value of " + fmt_d(s.x)
               + " was computed for a candidate minimum of the distance square function at the lower boundary of a "
                 "trajectory";
    default:
        return "internal capacity error in the conjunction pipeline (code " + std::to_string(s.code) + ")";
    }
}

struct event_pair {
    cudaEvent_t a = nullptr, b = nullptr;
    bool own = true;
    event_pair()
    {
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
    }
    event_pair(cudaEvent_t x, cudaEvent_t y) : a(x), b(y), own(false) {}
    event_pair(const event_pair &) = delete;
    event_pair &operator=(const event_pair &) = delete;
    event_pair(event_pair &&o) noexcept : a(o.a), b(o.b), own(o.own) { o.own = false; }
    ~event_pair()
    {
        if (!own) return;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    float ms() const
    {
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        return t;
    }
};

// Trace of a screening call's phases on stderr, enabled by the environment
// variable MZB_TRACE (any value): host-clock milliseconds since the call
// began at each phase boundary, the device's stage times per batch, and at
// the end a device timeline (CUDA events on the screening and copy streams:
// when each batch's upload chunk was in, its stages done, its outputs
// copied). The reference prints its per-stage timings at trace log level
// (detect_conjunctions.cpp:444-454); this is the same facility, with the
// host-side phases (allocation, host synchronisations, queue reruns) and
// the transfers that a GPU call adds.
struct call_trace {
    bool on = std::getenv("MZB_TRACE") != nullptr;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    cudaEvent_t dev_t0 = nullptr;
    std::vector<std::pair<std::string, cudaEvent_t>> dev_marks;
    call_trace(const call_trace &) = delete;
    call_trace &operator=(const call_trace &) = delete;
    call_trace() = default;
    ~call_trace()
    {
        if (dev_t0) cudaEventDestroy(dev_t0);
        for (auto &m : dev_marks) cudaEventDestroy(m.second);
    }
    void mark(const char *what, const std::string &detail = std::string()) const
    {
        if (!on) return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "[mizuba_b200] %9.3f ms  %s%s%s\n", ms, what, detail.empty() ? "" : ": ",
                     detail.c_str());
    }
    // A device timestamp on `stream`; the first one is the origin.
    void dev_mark(const std::string &what, cudaStream_t stream)
    {
        if (!on) return;
        cudaEvent_t e = nullptr;
        CK(cudaEventCreate(&e));
        CK(cudaEventRecord(e, stream));
        if (!dev_t0) dev_t0 = e;
        else dev_marks.emplace_back(what, e);
    }
    // After the streams have drained; up: the staged upload of a
    // polyjectory created asynchronously, whose chunks are reported complete
    // when their last piece landed (negative times: before the screening
    // began).
    void print_timeline(const stager *up, const std::vector<cudaEvent_t> &gather) const
    {
        if (!on || !dev_t0) return;
        for (size_t c = 0; c < gather.size(); ++c) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, dev_t0, gather[c]) == cudaSuccess)
                std::fprintf(stderr, "[mizuba_b200]   device %9.3f ms  upload chunk %zu complete\n", ms, c);
            else
                cudaGetLastError();
        }
        for (size_t c = 0; up && c < up->chunk_end.size(); ++c) {
            float last = -1e30f;
            bool any = false;
            for (uint64_t j = c ? up->chunk_end[c - 1] : 0; j < up->chunk_end[c]; ++j) {
                float ms = 0;
                if (cudaEventElapsedTime(&ms, dev_t0, up->piece_ev[j]) == cudaSuccess) {
                    last = std::max(last, ms);
                    any = true;
                } else {
                    cudaGetLastError();
                }
            }
            if (any) std::fprintf(stderr, "[mizuba_b200]   device %9.3f ms  upload chunk %zu complete\n", last, c);
        }
        for (const auto &m : dev_marks) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, dev_t0, m.second) == cudaSuccess)
                std::fprintf(stderr, "[mizuba_b200]   device %9.3f ms  %s\n", ms, m.first.c_str());
        }
    }
};

// Counters and sizes the host reads back between a batch's stages (tree
// sizes, pair counts, queue counts, the status word) go through mapped pinned
// memory written by a kernel, not through copies: a device-to-host copy on
// the screening stream queues behind the outputs already streaming to the
// host on the copy engine (hundreds of MB per batch), which stalled every
// batch by the length of those copies.
struct to_host_seg {
    const uint32_t *src;
    uint32_t *dst;
    uint32_t n;
};
constexpr int TO_HOST_SEGS = 8;
struct to_host_job {
    to_host_seg seg[TO_HOST_SEGS];
    int n_seg;
};
__global__ void __launch_bounds__(256) k_to_host(to_host_job job)
{
    for (int k = 0; k < job.n_seg; ++k)
        for (uint32_t i = threadIdx.x; i < job.seg[k].n; i += blockDim.x) job.seg[k].dst[i] = job.seg[k].src[i];
}

struct host_mailbox {
    char *h = nullptr; // host view
    char *d = nullptr; // device view of the same pages
    size_t bytes = 0, used = 0;
    bool own = false; // a private area (another call holds the device's cached one)
    host_mailbox(scratch_cache *cache, size_t n)
    {
        n = std::max<size_t>(n, 64 << 10);
        if (cache && cache->mbox_bytes < n) {
            if (cache->mbox_h) CK(cudaFreeHost(cache->mbox_h));
            cache->mbox_h = cache->mbox_d = nullptr;
            cache->mbox_bytes = 0;
            CK(cudaHostAlloc(reinterpret_cast<void **>(&cache->mbox_h), n, cudaHostAllocMapped));
            CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&cache->mbox_d), cache->mbox_h, 0));
            cache->mbox_bytes = n;
        }
        if (cache) {
            h = cache->mbox_h;
            d = cache->mbox_d;
            bytes = cache->mbox_bytes;
            return;
        }
        CK(cudaHostAlloc(reinterpret_cast<void **>(&h), n, cudaHostAllocMapped));
        CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&d), h, 0));
        bytes = n;
        own = true;
    }
    host_mailbox(const host_mailbox &) = delete;
    host_mailbox &operator=(const host_mailbox &) = delete;
    ~host_mailbox()
    {
        if (own && h) cudaFreeHost(h);
    }
    // A host area for count elements of T (8-byte aligned).
    template <typename T>
    T *take(size_t count)
    {
        const size_t off = (used + 7) & ~size_t(7);
        if (off + count * sizeof(T) > bytes) throw std::logic_error("host mailbox too small");
        used = off + count * sizeof(T);
        return reinterpret_cast<T *>(h + off);
    }
    // One launch copying device arrays into areas taken above.
    struct batch {
        host_mailbox &m;
        to_host_job job{};
        template <typename T>
        batch &add(T *host_area, const T *dev_src, size_t count)
        {
            static_assert(sizeof(T) % 4 == 0, "word-sized elements");
            if (job.n_seg == TO_HOST_SEGS) throw std::logic_error("too many mailbox segments");
            to_host_seg &g = job.seg[job.n_seg++];
            g.src = reinterpret_cast<const uint32_t *>(dev_src);
            g.dst = reinterpret_cast<uint32_t *>(m.d + (reinterpret_cast<char *>(host_area) - m.h));
            g.n = uint32_t(count * sizeof(T) / 4);
            return *this;
        }
        void launch(cudaStream_t s)
        {
            k_to_host<<<1, 256, 0, s>>>(job);
            CK(cudaGetLastError());
        }
    };
    batch start() { return batch{*this}; }
};

// The streams and events of one screening call: the device's cached set
// when the call holds the device's scratch (created on first use), private
// ones otherwise.
struct call_streams {
    scratch_cache *c = nullptr;
    cudaStream_t st = nullptr, cs = nullptr;
    cudaEvent_t ev[14] = {};
    cudaEvent_t ev_sorted = nullptr, ev_built = nullptr;
    explicit call_streams(scratch_cache *cache) : c(cache)
    {
        if (c && !c->st) {
            CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
            CK(cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking));
            for (int k = 0; k < 14; ++k) CK(cudaEventCreate(&c->ev[k]));
            for (int k = 0; k < 2; ++k) CK(cudaEventCreateWithFlags(&c->ev_nt[k], cudaEventDisableTiming));
        }
        if (c) {
            st = c->st;
            cs = c->cs;
            for (int k = 0; k < 14; ++k) ev[k] = c->ev[k];
            ev_sorted = c->ev_nt[0];
            ev_built = c->ev_nt[1];
            return;
        }
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        for (int k = 0; k < 14; ++k) CK(cudaEventCreate(&ev[k]));
        CK(cudaEventCreateWithFlags(&ev_sorted, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_built, cudaEventDisableTiming));
    }
    call_streams(const call_streams &) = delete;
    call_streams &operator=(const call_streams &) = delete;
    ~call_streams()
    {
        if (st) cudaStreamSynchronize(st);
        if (cs) cudaStreamSynchronize(cs);
        if (c) return;
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        if (ev_sorted) cudaEventDestroy(ev_sorted);
        if (ev_built) cudaEventDestroy(ev_built);
        if (st) cudaStreamDestroy(st);
        if (cs) cudaStreamDestroy(cs);
    }
};

struct stream_guard {
    cudaStream_t s = nullptr;
    stream_guard() { CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~stream_guard()
    {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
};

// dst != nullptr: each batch's per-step arrays are also copied to the host
// buffers in dst on a second stream, as soon as the stage producing them has
// run, so the transfers overlap the later stages of the batch (and of the next
// batches).
void run_detection(const mzb_pj &pj, double thresh, double interval, const int32_t *otypes_host, bool skip_cd,
                   uint32_t spb, bool mixed, int bvh_threads, int broad_walk, int sort_threads,
                   const mzb_host_outputs *dst, mzb_result &R)
{
    call_trace tr;
    init_device_consts();
    const uint64_t N = pj.n_objs, S_all = R.n_cd_steps, S0 = R.step_begin, S = R.n_run;
    // Declared before the streams, so it is released only after their
    // destructors have drained them.
    scratch_lease lease;
    auto SL = [&lease]() { return lease.next(); };
    call_streams cst(lease.cache);
    cudaStream_t st = cst.st, cs = cst.cs;
    cudaEvent_t ev_sorted = cst.ev_sorted, ev_built = cst.ev_built;
    uint64_t tree_cursor = 0;
    // Host areas of the per-batch read-backs (see host_mailbox).
    const uint64_t nb_cap = std::max<uint64_t>(1, std::min<uint64_t>(S, spb));
    host_mailbox mbox(lease.cache, nb_cap * 4 + (nb_cap + 1) * 8 + 1024);
    uint32_t *h_tsz_pin = mbox.take<uint32_t>(nb_cap);
    uint64_t *h_so = mbox.take<uint64_t>(nb_cap + 1);
    unsigned long long *h_spill_p = mbox.take<unsigned long long>(1);
    // Queue counts: items, root items, conjunctions, screened, prefiltered,
    // then the 7 narrow-phase counters.
    unsigned long long *h_q = mbox.take<unsigned long long>(5 + 7);
    dev_status *h_status = mbox.take<dev_status>(1);
    unsigned long long *h_bad = mbox.take<unsigned long long>(1);
    unsigned long long *h_visits = mbox.take<unsigned long long>(1);
    // Copies of this batch's per-step rows [s0, s0 + nb) of a [S][row] array.
    auto stream_rows = [&](void *host, const void *dev, uint64_t row_bytes, uint64_t s0, uint32_t nb) {
        if (host && row_bytes && nb)
            CK(cudaMemcpyAsync(static_cast<char *>(host) + s0 * row_bytes,
                               static_cast<const char *>(dev) + s0 * row_bytes, nb * row_bytes,
                               cudaMemcpyDeviceToHost, cs));
    };
    const dev_pj P = pj.view();
    // Result buffers are allocated on the call's stream and handed over to
    // stream 0 for their later release, once this stream has drained.
    auto hand_over = [&R]() {
        R.aabbs.fs = R.srt_aabbs.fs = 0;
        R.mcodes.fs = R.srt_mcodes.fs = 0;
        R.srt_idx.fs = R.tree_size.fs = 0;
        R.trees.fs = 0;
        R.bp.fs = 0;
        R.conj.fs = 0;
    };
    try {

    // Step bounds (get_cd_begin_end, conjunctions.cpp:373-392), indexed
    // relative to the first screened step.
    std::vector<double2> cdb(S);
    R.cd_end.resize(S);
    for (uint64_t kk = 0; kk < S; ++kk) {
        const uint64_t k = S0 + kk;
        const double b = interval * static_cast<double>(k);
        const double e = (k == S_all - 1) ? pj.maxT : interval * static_cast<double>(k + 1);
        if (!std::isfinite(b) || !std::isfinite(e) || !(e > b) || b < 0 || e > pj.maxT)
            throw invalid_arg("Invalid conjunction step time range: [" + fmt_d(b) + ", " + fmt_d(e) + ")");
        cdb[kk] = make_double2(b, e);
        R.cd_end[kk] = e;
    }
    dbuf<double2> d_cdb(SL());
    d_cdb.alloc(S, st);
    // Mixed-form tables: nodes, inverse node differences, inverse binomials.
    dbuf<double> d_mixed(SL());
    std::vector<double> h_mixed;
    if (mixed) {
        const int op1 = pj.order + 1, n = pj.order;
        const cheb_nodes cn = make_cheb_nodes(op1);
        h_mixed.assign(size_t(op1) + size_t(op1) * op1 + op1, 0.0);
        for (int m = 0; m < op1; ++m) h_mixed[m] = cn.v[m];
        for (int k = 0; k < n; ++k)
            for (int j = k + 1; j < op1; ++j) h_mixed[op1 + size_t(k) * op1 + j] = 1.0 / (cn.v[j] - cn.v[j - k - 1]);
        double c = 1.0;
        for (int i = 0; i <= n; ++i) {
            h_mixed[op1 + size_t(op1) * op1 + i] = 1.0 / c;
            c = c * (n - i) / (i + 1);
        }
        d_mixed.alloc(h_mixed.size(), st);
        CK(cudaMemcpyAsync(d_mixed.p, h_mixed.data(), h_mixed.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    const double *mixed_tab = mixed ? d_mixed.p : nullptr;
    const double *mixed_inv_binom = mixed ? d_mixed.p + (pj.order + 1) + size_t(pj.order + 1) * (pj.order + 1) : nullptr;
    CK(cudaMemcpyAsync(d_cdb.p, cdb.data(), S * sizeof(double2), cudaMemcpyHostToDevice, st));
    dbuf<int32_t> d_ot(SL());
    d_ot.alloc(N, st);
    {
        std::vector<int32_t> ot(N, 1);
        if (otypes_host) std::memcpy(ot.data(), otypes_host, N * sizeof(int32_t));
        CK(cudaMemcpyAsync(d_ot.p, ot.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }

    tr.mark("inputs on the device", std::to_string(N) + " objects, " + std::to_string(S) + " steps, "
                                        + std::to_string(spb) + " per batch");
    // Results.
    R.cap = 2 * N;
    {
        uint64_t off = 0;
        auto place = [&off](uint64_t bytes) {
            const uint64_t at = off;
            off += (bytes + 255) & ~uint64_t(255);
            return at;
        };
        const uint64_t o_ab = place(S * (N + 1) * 8 * sizeof(float)), o_sab = place(S * (N + 1) * 8 * sizeof(float));
        const uint64_t o_mc = place(S * N * 8), o_smc = place(S * N * 8), o_idx = place(S * N * 4);
        const uint64_t o_tsz = place(S * 4), o_tr = place(S * R.cap * sizeof(bvh_node));
        CK(cudaGetDevice(&R.dev));
        size_t got = 0;
        if (void *sp = off ? take_spare(R.dev, off, got) : nullptr) {
            R.block = sp;
            R.block_bytes = got;
        } else if (off) {
            ensure_pool();
            CK(cudaMallocAsync(&R.block, off, st));
            R.block_bytes = off;
        }
        char *b0 = static_cast<char *>(R.block);
        R.aabbs.borrow(reinterpret_cast<float *>(b0 + o_ab), S * (N + 1) * 8);
        R.srt_aabbs.borrow(reinterpret_cast<float *>(b0 + o_sab), S * (N + 1) * 8);
        R.mcodes.borrow(reinterpret_cast<uint64_t *>(b0 + o_mc), S * N);
        R.srt_mcodes.borrow(reinterpret_cast<uint64_t *>(b0 + o_smc), S * N);
        R.srt_idx.borrow(reinterpret_cast<uint32_t *>(b0 + o_idx), S * N);
        R.tree_size.borrow(reinterpret_cast<uint32_t *>(b0 + o_tsz), S);
        R.trees.borrow(reinterpret_cast<bvh_node *>(b0 + o_tr), S * R.cap);
    }
    R.bp_off.assign(2 * S, 0);
    tr.mark("result buffers allocated");

    // Batch scratch.
    const uint32_t nb_max = uint32_t(std::min<uint64_t>(S, spb));
    dbuf<uint64_t> keys_a(SL()), offs(SL()), block_sums(SL()), step_off(SL()), total(SL());
    dbuf<uint32_t> vals_a(SL()), vals_b(SL()), counts(SL()), aux(SL()), cc_cnt(SL()), cc_off(SL()), cc_cur(SL());
    dbuf<int32_t> ropes(SL());
    dbuf<walk_node> walks(SL());
    dbuf<dev_status> d_st(SL());
    dbuf<unsigned long long> visits(SL()); // broad-phase node visits of the call
    dbuf<unsigned long long> ctr(SL()), rq_count(SL()), cq_count(SL());
    keys_a.alloc(uint64_t(nb_max) * N, st);
    vals_a.alloc(uint64_t(nb_max) * N, st);
    vals_b.alloc(uint64_t(nb_max) * N, st);
    dbuf<uint2> more(SL());
    dbuf<uint2> srange(SL());
    dbuf<unsigned long long> more_count(SL());
    // Mixed form: two distance-screen models (2 x 16 bytes each) per object
    // and step of the batch, written by the AABB pass.
    dbuf<float4> scr(SL());
    if (mixed) scr.alloc(uint64_t(nb_max) * N * 4, st);
    more.alloc(uint64_t(nb_max) * N, st);
    srange.alloc(uint64_t(nb_max) * N, st);
    more_count.alloc(1, st);
    ropes.alloc(uint64_t(nb_max) * R.cap, st);
    walks.alloc(uint64_t(nb_max) * R.cap, st);
    const uint64_t aux_step = bvh_aux_words(N, R.cap);
    aux.alloc(uint64_t(nb_max) * aux_step, st);
    counts.alloc(uint64_t(nb_max) * N, st);
    dbuf<uint32_t> leaf_of(SL()), stage(SL());
    dbuf<uint64_t> overflow(SL());
    dbuf<unsigned long long> overflow_count(SL());
    leaf_of.alloc(uint64_t(nb_max) * N, st);
    stage.alloc(uint64_t(nb_max) * N * BROAD_STAGE_K, st);
    overflow.alloc(uint64_t(nb_max) * N, st);
    overflow_count.alloc(1, st);
    // Partners beyond the staged ones; when more spill than this holds, the
    // overflowing objects are walked again instead.
    dbuf<ulonglong2> spill(SL());
    dbuf<unsigned long long> spill_count(SL());
    dbuf<unsigned long long> walk_next(SL());
    const uint64_t spill_cap = std::max<uint64_t>(1 << 16, uint64_t(nb_max) * N / 8);
    spill.alloc(spill_cap, st);
    spill_count.alloc(1, st);
    walk_next.alloc(1, st);
    offs.alloc(uint64_t(nb_max) * N, st);
    block_sums.alloc((uint64_t(nb_max) * N + 1023) / 1024 + 1, st);
    step_off.alloc(nb_max + 1, st);
    total.alloc(1, st);
    d_st.alloc(1, st);
    ctr.alloc(7, st);
    rq_count.alloc(1, st);
    cq_count.alloc(1, st);
    cc_cnt.alloc(nb_max + 1, st);
    cc_off.alloc(nb_max + 1, st);
    cc_cur.alloc(nb_max + 1, st);
    CK(cudaMemsetAsync(d_st.p, 0, sizeof(dev_status), st));
    visits.alloc(1, st);
    CK(cudaMemsetAsync(visits.p, 0, sizeof(unsigned long long), st));

    dbuf<root_item> rq(SL());
    dbuf<np_item> items(SL()), surv(SL()), cand(SL());
    dbuf<unsigned long long> item_count(SL()), surv_count(SL()), cand_count(SL());
    item_count.alloc(1, st);
    surv_count.alloc(1, st);
    cand_count.alloc(1, st);
    const unsigned narrow_grid = 148 * 3;
    dbuf<conj_out> cq(SL()), cgrp(SL());
    dbuf<double> wl(SL()), wl_full(SL());
    dbuf<uint32_t> retry(SL());
    dbuf<unsigned long long> retry_count(SL());
    retry_count.alloc(1, st);
    const unsigned roots_grid = 148 * 4, roots_grid_full = 8;
    const uint64_t ent = uint64_t(pj.order) + 3; // (lb, ub, order + 1 coefficients)
    wl.alloc(uint64_t(roots_grid) * 128 * ROOTS_WL_SMALL * ent, st);
    wl_full.alloc(uint64_t(roots_grid_full) * 128 * ROOTS_WL_FULL * ent, st);

    tr.mark("batch scratch allocated");
    tr.dev_mark("origin", st);
    std::vector<event_pair> ev;
    ev.reserve(7);
    for (int k = 0; k < 7; ++k) ev.emplace_back(cst.ev[2 * k], cst.ev[2 * k + 1]);
    // Queue entries per broad-phase pair seen so far in this call (items,
    // root items, conjunctions): the next batch's queues are sized from
    // them, since an overflow reruns the batch's narrow phase and root
    // finding.
    double items_per_pair = 2.0, roots_per_pair = 0.5, conj_per_pair = 0.125;
    const double thresh2 = thresh * thresh;
    const double radius = thresh / 2;

    // The device status word, after the trajectory check of an upload still
    // in flight (mzb_pj_create_async): the segments this stream has waited
    // for are flagged by now, and a non-finite trajectory value is the
    // reference's constructor error, which comes before any screening error.
    auto check_status = [&]() {
        *h_bad = ~0ull;
        auto job = mbox.start();
        job.add(h_status, d_st.p, 1);
        if (pj.async_upload()) job.add(h_bad, static_cast<const unsigned long long *>(pj.bad_seg.p), 1);
        job.launch(st);
        CK(cudaStreamSynchronize(st));
        const dev_status h = *h_status;
        pj.throw_if_bad(*h_bad);
        if (h.code != 0) {
            if (h.code == ERR_CAPACITY) throw std::runtime_error(status_message(h));
            throw invalid_arg(status_message(h));
        }
    };

    for (uint64_t s0 = 0; s0 < S; s0 += nb_max) {
        const uint32_t nb = uint32_t(std::min<uint64_t>(nb_max, S - s0));
        const uint32_t sf = uint32_t(s0);
        pj.wait_upload(st, R.cd_end[s0 + nb - 1]);
        const std::string bname = "batch " + std::to_string(s0) + "+" + std::to_string(nb);
        tr.dev_mark(bname + ": its upload chunks in", st);
        CK(cudaEventRecord(ev[0].a, st));
        launch_aabb(P, d_cdb.p, mixed_inv_binom, sf, nb, radius, R.aabbs.p, more.p, more_count.p,
                    mixed ? scr.p : nullptr, srange.p, d_st.p, st);
        CK(cudaEventRecord(ev[0].b, st));
        CK(cudaEventRecord(ev[1].a, st));
        launch_morton(R.aabbs.p, sf, nb, N, R.mcodes.p, st);
        launch_sort(R.aabbs.p, R.mcodes.p, sf, nb, N, keys_a.p, vals_a.p, vals_b.p, R.srt_idx.p,
                    R.srt_mcodes.p, R.srt_aabbs.p, sort_threads, st);
        CK(cudaEventRecord(ev[1].b, st));
        if (dst) {
            CK(cudaEventRecord(ev_sorted, st));
            CK(cudaStreamWaitEvent(cs, ev_sorted, 0));
            stream_rows(dst->aabbs, R.aabbs.p, (N + 1) * 8 * sizeof(float), s0, nb);
            stream_rows(dst->srt_aabbs, R.srt_aabbs.p, (N + 1) * 8 * sizeof(float), s0, nb);
            stream_rows(dst->mcodes, R.mcodes.p, N * sizeof(uint64_t), s0, nb);
            stream_rows(dst->srt_mcodes, R.srt_mcodes.p, N * sizeof(uint64_t), s0, nb);
            stream_rows(dst->srt_idx, R.srt_idx.p, N * sizeof(uint32_t), s0, nb);
        }
        CK(cudaEventRecord(ev[2].a, st));
        launch_bvh(R.srt_aabbs.p, R.srt_mcodes.p, sf, nb, N, R.trees.p, R.cap, ropes.p, aux.p, leaf_of.p,
                   R.tree_size.p, walks.p, d_st.p, bvh_threads, st);
        CK(cudaEventRecord(ev[2].b, st));
        // Trees: their sizes are read back with the pair counts below (or
        // here when the broad phase is skipped), then each step's tree goes
        // to its packed place in dst->trees.
        const bool want_trees = dst && dst->trees && nb > 0;
        uint32_t *h_tsz = h_tsz_pin;
        auto stream_trees = [&]() {
            if (!want_trees) return;
            CK(cudaStreamWaitEvent(cs, ev_built, 0));
            for (uint32_t b = 0; b < nb; ++b) {
                if (tree_cursor + h_tsz[b] > dst->trees_cap)
                    throw invalid_arg("mzb_conjunctions_stream: the trees need more than the "
                                      + std::to_string(dst->trees_cap) + " nodes of the destination buffer");
                if (h_tsz[b])
                    CK(cudaMemcpyAsync(static_cast<char *>(dst->trees) + tree_cursor * sizeof(bvh_node),
                                       R.trees.p + (s0 + b) * R.cap, h_tsz[b] * sizeof(bvh_node),
                                       cudaMemcpyDeviceToHost, cs));
                tree_cursor += h_tsz[b];
            }
        };
        if (want_trees) {
            CK(cudaEventRecord(ev_built, st));
            mbox.start().add(h_tsz, static_cast<const uint32_t *>(R.tree_size.p + s0), nb).launch(st);
            if (skip_cd) {
                CK(cudaStreamSynchronize(st));
                stream_trees();
            }
        }
        float t_bp = 0, t_np = 0, t_rt = 0;
        uint64_t n_narrow_launches = 0, n_roots_launches = 0, n_broad_launches = 0;
        // Mailbox read-backs of the batch: the status word, the tree sizes,
        // the pair counts and one per narrow-phase run.
        uint64_t n_mbox = want_trees ? 2 : 1;
        if (!skip_cd) {
            CK(cudaEventRecord(ev[3].a, st));
            launch_broad_half(R.srt_aabbs.p, R.trees.p, R.cap, ropes.p, walks.p, leaf_of.p, R.srt_idx.p, R.tree_size.p,
                              d_ot.p, sf, nb, N, counts.p, stage.p, spill.p, spill_cap, spill_count.p, walk_next.p,
                              broad_walk, visits.p, st);
            launch_scan(counts.p, uint64_t(nb) * N, offs.p, block_sums.p, total.p, st);
            launch_step_offsets(offs.p, N, nb, total.p, step_off.p, st);
            mbox.start()
                .add(h_so, static_cast<const uint64_t *>(step_off.p), nb + 1)
                .add(h_spill_p, static_cast<const unsigned long long *>(spill_count.p), 1)
                .launch(st);
            ++n_mbox;
            CK(cudaStreamSynchronize(st));
            const unsigned long long h_spill = *h_spill_p;
            tr.mark("broad-phase counts read", "steps " + std::to_string(s0) + "+" + std::to_string(nb));
            stream_trees();
            tr.dev_mark(bname + ": broad phase done", st);
            const uint64_t np_batch = h_so[nb];
            if (np_batch >= (1ull << 32)) throw std::runtime_error("too many broad-phase pairs in one batch");
            // The pair and conjunction lists of the call grow batch by batch;
            // each new block is sized for the whole call by extrapolating from
            // the steps screened so far (+15 %), so that a multi-batch call
            // reallocates them about once: a larger stream-ordered block than
            // the pool holds has the driver map new memory, measured at about
            // 25 ms per batch on the 30,000-object 7-day span.
            const double done_frac = double(s0 + nb) / double(S);
            auto whole_call = [done_frac](uint64_t so_far) {
                return uint64_t(double(so_far) / done_frac * 1.15) + 1024;
            };
            if (R.bp.n < R.n_bp + np_batch)
                R.bp.grow(std::max(R.n_bp + np_batch, whole_call(R.n_bp + np_batch)), R.n_bp, st);
            uint2 *bp_batch = R.bp.p + R.n_bp;
            launch_broad_copy(R.aabbs.p, R.trees.p, R.cap, ropes.p, R.srt_idx.p, d_ot.p, sf, nb, N, counts.p, offs.p,
                              stage.p, bp_batch, overflow.p, overflow_count.p, spill.p, spill_count.p,
                              h_spill <= spill_cap, st);
            n_broad_launches = h_spill <= spill_cap ? 8 : 7;
            CK(cudaEventRecord(ev[3].b, st));
            for (uint32_t b = 0; b < nb; ++b) {
                R.bp_off[2 * (s0 + b)] = R.n_bp + h_so[b];
                R.bp_off[2 * (s0 + b) + 1] = h_so[b + 1] - h_so[b];
            }
            R.n_bp += np_batch;

            // Narrow phase and minimum search: k_items appends sub-interval
            // items, the persistent k_narrow consumes them and appends
            // surviving items to the root queue, the persistent k_roots
            // consumes that (items whose working list outgrows the short one
            // are retried with the full list).  Queue sizes are read on the
            // device; one host synchronisation checks every capacity and the
            // stage reruns with grown queues on overflow.
            auto sized = [np_batch](double per_pair) { return uint64_t(double(np_batch) * per_pair * 1.1) + 1024; };
            // The mixed form screens items as they are found: no item queue,
            // the screen's queue (cand) and the prefilter's (surv) are sized
            // for every item instead.
            const uint64_t item_cap0 = std::max<uint64_t>(mixed ? cand.n : items.n, sized(items_per_pair));
            if (!mixed && items.n < item_cap0) items.alloc_queue(item_cap0, st);
            if (mixed && cand.n < item_cap0) cand.alloc_queue(item_cap0, st);
            if (mixed && surv.n < cand.n) surv.alloc_queue(cand.n, st);
            const uint64_t rq_cap0 = std::max<uint64_t>(rq.n, sized(roots_per_pair));
            if (rq.n < rq_cap0) rq.alloc_queue(rq_cap0, st);
            if (retry.n < rq.n) retry.alloc_queue(rq.n, st);
            const uint64_t cq_cap0 = std::max<uint64_t>(cq.n, sized(conj_per_pair));
            if (cq.n < cq_cap0) cq.alloc_queue(cq_cap0, st);
            tr.mark("pair list and queues allocated", std::to_string(np_batch) + " pairs");
            unsigned long long h_rq = 0, h_items = 0, h_cq = 0, h_ctr[7] = {}, h_cand = 0, h_surv = 0;
            for (;;) {
                CK(cudaMemsetAsync(ctr.p, 0, 7 * sizeof(unsigned long long), st));
                CK(cudaMemsetAsync(rq_count.p, 0, sizeof(unsigned long long), st));
                CK(cudaMemsetAsync(item_count.p, 0, sizeof(unsigned long long), st));
                CK(cudaMemsetAsync(cq_count.p, 0, sizeof(unsigned long long), st));
                CK(cudaMemsetAsync(retry_count.p, 0, sizeof(unsigned long long), st));
                CK(cudaEventRecord(ev[4].a, st));
                if (mixed) {
                    // Items screened as the merge walk finds them, the
                    // FMA-native prefilter, then the reference formulation on
                    // the survivors only.
                    CK(cudaMemsetAsync(surv_count.p, 0, sizeof(unsigned long long), st));
                    CK(cudaMemsetAsync(cand_count.p, 0, sizeof(unsigned long long), st));
                    launch_items_screen(P, d_cdb.p, sf, nb, bp_batch, step_off.p, srange.p, np_batch, thresh, scr.p,
                                        cand.p, cand.n, cand_count.p, item_count.p, ctr.p, d_st.p, st);
                    launch_narrow_prefilter(P, mixed_tab, d_cdb.p, sf, cand.p, cand_count.p, cand.n, thresh2,
                                            surv.p, surv.n, surv_count.p, ctr.p, d_st.p, narrow_grid, st);
                    launch_narrow(P, d_cdb.p, sf, surv.p, surv_count.p, surv.n, thresh2, rq.p, rq.n, rq_count.p,
                                  ctr.p, d_st.p, narrow_grid, st);
                    n_narrow_launches += 1;
                } else {
                    launch_items(P, d_cdb.p, sf, nb, bp_batch, step_off.p, srange.p, np_batch, items.p, items.n,
                                 item_count.p, ctr.p, d_st.p, st);
                    launch_narrow(P, d_cdb.p, sf, items.p, item_count.p, items.n, thresh2, rq.p, rq.n, rq_count.p,
                                  ctr.p, d_st.p, narrow_grid, st);
                }
                CK(cudaEventRecord(ev[4].b, st));
                CK(cudaEventRecord(ev[5].a, st));
                launch_roots(P, rq.p, rq_count.p, rq.n, nullptr, nullptr, thresh2, wl.p, ROOTS_WL_SMALL, roots_grid,
                             retry.p, retry_count.p, cq.p, cq.n, cq_count.p, ctr.p, d_st.p, st);
                launch_roots(P, rq.p, rq_count.p, rq.n, retry.p, retry_count.p, thresh2, wl_full.p, ROOTS_WL_FULL,
                             roots_grid_full, nullptr, nullptr, cq.p, cq.n, cq_count.p, ctr.p, d_st.p, st);
                CK(cudaEventRecord(ev[5].b, st));
                n_narrow_launches += 2;
                n_roots_launches += 2;
                {
                    auto job = mbox.start();
                    job.add(h_q + 0, static_cast<const unsigned long long *>(item_count.p), 1)
                        .add(h_q + 1, static_cast<const unsigned long long *>(rq_count.p), 1)
                        .add(h_q + 2, static_cast<const unsigned long long *>(cq_count.p), 1)
                        .add(h_q + 5, static_cast<const unsigned long long *>(ctr.p), 7);
                    if (mixed)
                        job.add(h_q + 3, static_cast<const unsigned long long *>(cand_count.p), 1)
                            .add(h_q + 4, static_cast<const unsigned long long *>(surv_count.p), 1);
                    job.launch(st);
                    ++n_mbox;
                }
                CK(cudaStreamSynchronize(st));
                h_items = h_q[0];
                h_rq = h_q[1];
                h_cq = h_q[2];
                h_cand = mixed ? h_q[3] : 0;
                h_surv = mixed ? h_q[4] : 0;
                for (int k = 0; k < 7; ++k) h_ctr[k] = h_q[5 + k];
                tr.mark("narrow phase and root finding run",
                        std::to_string(h_items) + " items, " + std::to_string(h_rq) + " root items, "
                            + std::to_string(h_cq) + " conjunctions");
                // Reruns after a queue overflow count in the stage times.
                t_np += ev[4].ms();
                t_rt += ev[5].ms();
                bool again = false;
                if (h_items > (mixed ? cand.n : items.n)) {
                    if (mixed) {
                        cand.alloc_queue(h_items + h_items / 4, st);
                        surv.alloc_queue(cand.n, st);
                    } else {
                        items.alloc_queue(h_items + h_items / 4, st);
                    }
                    again = true;
                }
                if (h_rq > rq.n) {
                    rq.alloc_queue(h_rq + h_rq / 4, st);
                    retry.alloc_queue(rq.n, st);
                    again = true;
                }
                if (h_cq > cq.n) {
                    cq.alloc_queue(h_cq + h_cq / 4, st);
                    again = true;
                }
                if (!again) break;
            }
            if (np_batch) {
                items_per_pair = std::max(items_per_pair, double(h_items) / double(np_batch));
                roots_per_pair = std::max(roots_per_pair, double(h_rq) / double(np_batch));
                conj_per_pair = std::max(conj_per_pair, double(h_cq) / double(np_batch));
            }
            for (int k = 0; k < 7; ++k) R.np[k] += h_ctr[k];
            R.narrow_split[0] += h_cand;
            R.narrow_split[1] += h_surv;
            // Per-step ordering, appended to the result.
            if (cgrp.n < h_cq) cgrp.alloc(h_cq, st);
            if (R.conj.n < R.n_conj + h_cq)
                R.conj.grow(std::max<uint64_t>(R.n_conj + h_cq, whole_call(R.n_conj + h_cq)), R.n_conj, st);
            CK(cudaEventRecord(ev[6].a, st));
            launch_conj_sort(cq.p, h_cq, nb, cc_cnt.p, cc_off.p, cc_cur.p, cgrp.p, R.conj.p + R.n_conj, st);
            CK(cudaEventRecord(ev[6].b, st));
            R.n_conj += h_cq;
            t_bp = ev[3].ms();
        }
        // aabb (2 passes + global box) + morton + sort + bvh; broad half walk, 3 scan kernels,
        // step offsets, copy + spill scatter + list sort (or the overflow walk),
        // items + narrow, roots (+ retry), 5 conj-order kernels.
        R.n_launches += 6 + n_mbox;
        if (!skip_cd) R.n_launches += n_broad_launches + n_narrow_launches + n_roots_launches + 5;
        tr.dev_mark(bname + ": screened", st);
        if (dst) tr.dev_mark(bname + ": per-step outputs copied", cs);
        check_status();
        if (tr.on) {
            char b[160];
            std::snprintf(b, sizeof(b), "aabb %.3f, morton+sort %.3f, bvh %.3f, broad %.3f, narrow %.3f, roots %.3f, "
                          "order %.3f ms", ev[0].ms(), ev[1].ms(), ev[2].ms(), skip_cd ? 0.f : t_bp,
                          skip_cd ? 0.f : t_np, skip_cd ? 0.f : t_rt, skip_cd ? 0.f : ev[6].ms());
            tr.mark("batch done", b);
        }
        R.stage_ms[0] += ev[0].ms();
        R.stage_ms[1] += ev[1].ms();
        R.stage_ms[2] += ev[2].ms();
        if (!skip_cd) {
            R.stage_ms[3] += t_bp;
            R.stage_ms[4] += t_np;
            R.stage_ms[5] += t_rt;
            R.stage_ms[6] += ev[6].ms();
        }
    }
    for (int k = 0; k < 7; ++k) R.stage_ms[7] += R.stage_ms[k];
    {
        mbox.start().add(h_visits, static_cast<const unsigned long long *>(visits.p), 1).launch(st);
        R.n_launches += 1;
        CK(cudaStreamSynchronize(st));
        R.broad_visits = *h_visits;
    }
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamSynchronize(cs));
    tr.mark("call done");
    tr.print_timeline(pj.stg.get(), pj.up_ev);
    if (dst && dst->cd_end_times) std::memcpy(dst->cd_end_times, R.cd_end.data(), S * sizeof(double));
    } catch (...) {
        cudaStreamSynchronize(st);
        cudaStreamSynchronize(cs);
        hand_over();
        throw;
    }
    hand_over();
}

template <typename F>
int guarded(F &&f)
{
    try {
        f();
        return MZB_OK;
    } catch (const std::invalid_argument &e) {
        g_err = e.what();
        return MZB_INVALID_ARGUMENT;
    } catch (const std::out_of_range &e) {
        g_err = e.what();
        return MZB_OUT_OF_RANGE;
    } catch (const std::exception &e) {
        g_err = e.what();
        return MZB_RUNTIME_ERROR;
    } catch (...) {
        g_err = "unknown error";
        return MZB_RUNTIME_ERROR;
    }
}

// State evaluation shared by state_eval and state_meval: every (object,
// time) evaluation e * n_t + j reads tm[e * tm_stride_obj + j * tm_stride_t]
// and writes 7 doubles.  The evaluation errors of pj_eval_obj_state
// (polyjectory.cpp:1100-1104, a non-finite time) and of polyjectory::operator[]
// (polyjectory.cpp:1006-1016, an object index out of range) are checked on the
// host before any work, in evaluation order.  The work is split into chunks of
// objects so that device buffers stay below 1 GiB.
void run_state_eval(const mzb_pj *pj, double *out, const double *tm, uint64_t tm_stride_obj, uint64_t tm_stride_t,
                    const uint64_t *sel, uint64_t n_eval, uint64_t n_t)
{
    if (n_eval == 0 || n_t == 0) return;
    for (uint64_t e = 0; e < n_eval; ++e) {
        if (tm_stride_obj != 0 || e == 0)
            for (uint64_t j = 0; j < n_t; ++j) {
                const double t = tm[e * tm_stride_obj + j * tm_stride_t];
                if (!std::isfinite(t))
                    throw invalid_arg("An non-finite evaluation time of " + fmt_d(t)
                                      + " was detected during the evaluation of a polyjectory");
                if (tm_stride_t == 0) break;
            }
        if (sel && sel[e] >= pj->n_objs)
            throw out_of_range_err("Invalid object index " + std::to_string(sel[e])
                                   + " specified - the total number of objects in the polyjectory is only "
                                   + std::to_string(pj->n_objs));
    }
    if (pj->async_upload()) { // any time may need any chunk
        pj->wait_upload_host();
        pj->check_data(0);
    }
    const dev_pj v = pj->view();
    const uint64_t row_bytes = n_t * 7 * sizeof(double) + sizeof(uint64_t) + (tm_stride_obj ? n_t : 0) * sizeof(double);
    const uint64_t rows = std::max<uint64_t>(1, std::min<uint64_t>(n_eval, (1ull << 30) / row_bytes));
    const uint64_t tm_shared = tm_stride_obj ? 0 : (tm_stride_t ? n_t : 1);
    dbuf<double> d_tm, d_out;
    dbuf<uint64_t> d_sel;
    if (tm_shared) {
        d_tm.alloc(tm_shared, 0);
        CK(cudaMemcpy(d_tm.p, tm, tm_shared * sizeof(double), cudaMemcpyDefault));
    }
    for (uint64_t e0 = 0; e0 < n_eval; e0 += rows) {
        const uint64_t ne = std::min(rows, n_eval - e0);
        if (!tm_shared) {
            const uint64_t cnt = ne * tm_stride_obj;
            if (d_tm.n < cnt) d_tm.alloc(cnt, 0);
            CK(cudaMemcpy(d_tm.p, tm + e0 * tm_stride_obj, cnt * sizeof(double), cudaMemcpyDefault));
        }
        if (sel) {
            if (d_sel.n < ne) d_sel.alloc(ne, 0);
            CK(cudaMemcpy(d_sel.p, sel + e0, ne * sizeof(uint64_t), cudaMemcpyDefault));
        }
        if (d_out.n < ne * n_t * 7) d_out.alloc(ne * n_t * 7, 0);
        launch_state_eval(v, d_tm.p, tm_stride_obj, tm_stride_t, sel ? d_sel.p : nullptr, ne, n_t, d_out.p, 0);
        CK(cudaGetLastError());
        CK(cudaMemcpy(out + e0 * n_t * 7, d_out.p, ne * n_t * 7 * sizeof(double), cudaMemcpyDefault));
    }
    CK(cudaDeviceSynchronize());
}

// ---- Output files (mizuba/detect_conjunctions.cpp:92-126, :466-534).
//
// Device results are streamed into new files through two pinned staging
// buffers: the copy of chunk k + 1 from HBM runs while chunk k is written.
struct file_stager {
    static constexpr size_t CAP = size_t(32) << 20;
    void *buf[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    file_stager()
    {
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            CK(cudaMallocHost(&buf[k], CAP));
            CK(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
        }
    }
    ~file_stager()
    {
        if (st) cudaStreamSynchronize(st);
        for (int k = 0; k < 2; ++k) {
            if (buf[k]) cudaFreeHost(buf[k]);
            if (ev[k]) cudaEventDestroy(ev[k]);
        }
        if (st) cudaStreamDestroy(st);
    }
    file_stager(const file_stager &) = delete;
    file_stager &operator=(const file_stager &) = delete;
};

void write_fully(int fd, const char *p, size_t n, const std::string &path)
{
    while (n) {
        const ssize_t w = ::write(fd, p, n);
        if (w < 0) {
            if (errno == EINTR) continue;
            throw std::runtime_error("Error while writing the file '" + path + "': " + std::strerror(errno));
        }
        p += w;
        n -= size_t(w);
    }
}

// Creates path (which must not exist), writes bytes of device memory into it,
// or the sentinel when there are none, and leaves it readable by the owner
// only (mark_file_read_only, file_utils.cpp:253-259).
void device_to_file(file_stager &sg, const std::string &path, const void *dev, uint64_t bytes, const char *sentinel,
                    size_t sentinel_bytes)
{
    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_EXCL | O_CLOEXEC, 0600);
    if (fd < 0) throw std::runtime_error("Unable to create the file '" + path + "': " + std::strerror(errno));
    try {
        const char *src = static_cast<const char *>(dev);
        int k = 0;
        if (bytes) {
            CK(cudaMemcpyAsync(sg.buf[0], src, std::min<uint64_t>(bytes, file_stager::CAP), cudaMemcpyDeviceToHost,
                               sg.st));
            CK(cudaEventRecord(sg.ev[0], sg.st));
        }
        for (uint64_t off = 0; off < bytes;) {
            const uint64_t c = std::min<uint64_t>(bytes - off, file_stager::CAP);
            const uint64_t noff = off + c;
            if (noff < bytes) {
                CK(cudaMemcpyAsync(sg.buf[k ^ 1], src + noff, std::min<uint64_t>(bytes - noff, file_stager::CAP),
                                   cudaMemcpyDeviceToHost, sg.st));
                CK(cudaEventRecord(sg.ev[k ^ 1], sg.st));
            }
            CK(cudaEventSynchronize(sg.ev[k]));
            write_fully(fd, static_cast<const char *>(sg.buf[k]), c, path);
            off = noff;
            k ^= 1;
        }
        if (bytes == 0 && sentinel_bytes) write_fully(fd, sentinel, sentinel_bytes, path);
    } catch (...) {
        cudaStreamSynchronize(sg.st);
        ::close(fd);
        throw;
    }
    if (::close(fd) != 0) throw std::runtime_error("Error while closing the file '" + path + "'");
    if (::chmod(path.c_str(), S_IRUSR) != 0)
        throw std::runtime_error("Unable to mark the file '" + path + "' as read-only");
}

} // namespace

extern "C" {

const char *mzb_last_error(void) { return g_err.c_str(); }

// Checks the arguments and fills everything but the coefficients (times,
// offsets and segment counts are uploaded synchronously: they are small).
// The checks are the polyjectory constructor's (polyjectory.cpp:352-600) and
// run on the host before any device work: offsets within the data, time
// points finite, non-negative and strictly increasing per object, at least
// one non-empty trajectory, and maxT equal to the largest end time.  Trajectory
// values are checked by the upload kernels (they read every value anyway).
static mzb_pj *pj_prepare(const double *time, uint64_t traj_size, const uint64_t *traj_offsets, uint64_t time_size,
                          const uint64_t *time_offsets, uint64_t n_objs, uint32_t order, double maxT)
{
    const call_trace tr;
    if (order < 2 || order + 1 > uint32_t(MAX_OP1))
        throw invalid_arg("Unsupported polynomial order " + std::to_string(order)
                          + ": this build handles orders 2 to " + std::to_string(MAX_OP1 - 1));
    if (n_objs == 0) throw invalid_arg("Cannot initialise a polyjectory object from an empty list of trajectories");
    if (n_objs >= (1ull << 32)) throw invalid_arg("too many objects (object indices are 32-bit)");
    const uint64_t per = uint64_t(order + 1) * 7;
    if (traj_size % per != 0) throw invalid_arg("inconsistent trajectory data size");
    const uint64_t n_seg = traj_size / per;
    std::vector<uint64_t> soff(n_objs), toff(n_objs);
    std::vector<uint32_t> ns(n_objs);
    std::vector<uint64_t> keep_to, keep_tm;
    std::vector<double> keep_time;
    const uint64_t *h_to = host_view(traj_offsets, 2 * n_objs, keep_to);
    const uint64_t *h_tm = host_view(time_offsets, n_objs, keep_tm);
    const double *h_time = host_view(time, time_size, keep_time);
    // The checks of every object, in parallel over object ranges for large
    // inputs; the error reported is the one of the lowest object index, as a
    // serial pass over the objects would report it.
    struct range_result {
        uint64_t n_total = 0, bad = ~0ull;
        double max_end = 0;
        std::string msg;
    };
    auto check_range = [&](uint64_t i0, uint64_t i1, range_result &r) {
        for (uint64_t i = i0; i < i1; ++i) {
            const uint64_t off = h_to[2 * i], steps = h_to[2 * i + 1];
            std::string err;
            if (off % per != 0 || off / per > n_seg || steps > n_seg - off / per)
                err = "invalid trajectory offsets for the object at index " + std::to_string(i);
            else if (steps > 0 && (h_tm[i] > time_size || steps + 1 > time_size - h_tm[i]))
                err = "invalid time offsets for the object at index " + std::to_string(i);
            else if (steps >= (1ull << 32))
                err = "too many trajectory steps";
            const double *t = err.empty() ? h_time + h_tm[i] : nullptr;
            for (uint64_t j = 0; err.empty() && steps > 0 && j <= steps; ++j) {
                if (!std::isfinite(t[j]))
                    err = "A non-finite time coordinate was found for the object at index " + std::to_string(i);
                else if (t[j] < 0)
                    err = "A negative time coordinate was found for the object at index " + std::to_string(i);
                else if (j > 0 && !(t[j] > t[j - 1]))
                    err = "The sequence of times for the object at index " + std::to_string(i)
                          + " is not monotonically increasing";
            }
            if (!err.empty()) {
                r.bad = i;
                r.msg = std::move(err);
                return;
            }
            if (steps > 0) r.max_end = std::max(r.max_end, t[steps]);
            r.n_total += steps;
            soff[i] = off / per;
            ns[i] = uint32_t(steps);
            toff[i] = h_tm[i];
        }
    };
    const unsigned n_thr = n_objs < 4096 ? 1u : std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    std::vector<range_result> parts(n_thr);
    {
        std::vector<std::thread> th;
        for (unsigned k = 1; k < n_thr; ++k)
            th.emplace_back(check_range, n_objs * k / n_thr, n_objs * (k + 1) / n_thr, std::ref(parts[k]));
        check_range(0, n_objs / n_thr, parts[0]);
        for (std::thread &t : th) t.join();
    }
    tr.mark("polyjectory checks done", std::to_string(n_thr) + " threads");
    uint64_t n_total = 0;
    double max_end = 0;
    for (const range_result &r : parts) {
        if (r.bad != ~0ull) throw invalid_arg(r.msg);
        n_total += r.n_total;
        max_end = std::max(max_end, r.max_end);
    }
    if (n_total == 0)
        throw invalid_arg(
            "All the trajectories in a polyjectory have a number of steps equal to zero: this is not allowed");
    if (!(maxT == max_end))
        throw invalid_arg("The maxT of " + fmt_d(maxT) + " does not equal the largest trajectory end time of "
                          + fmt_d(max_end));
    auto *P = new mzb_pj;
    try {
        P->order = int(order);
        P->n_objs = n_objs;
        P->n_seg = n_seg;
        P->maxT = maxT;
        init_device_consts();
        P->coef.alloc(n_seg * 7 * uint64_t(row_ld(int(order + 1))), 0);
        tr.mark("coefficient buffer allocated");
        P->time.alloc(time_size, 0);
        P->seg_off.alloc(n_objs, 0);
        P->time_off.alloc(n_objs, 0);
        P->nseg.alloc(n_objs, 0);
        P->bad_seg.alloc(1, 0);
        P->h_seg_off = std::move(soff);
        P->h_nseg = std::move(ns);
        P->h_time_off = std::move(toff);
        if (time_size) CK(cudaMemcpy(P->time.p, h_time, time_size * sizeof(double), cudaMemcpyDefault));
        CK(cudaMemcpy(P->seg_off.p, P->h_seg_off.data(), n_objs * sizeof(uint64_t), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(P->time_off.p, P->h_time_off.data(), n_objs * sizeof(uint64_t), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(P->nseg.p, P->h_nseg.data(), n_objs * sizeof(uint32_t), cudaMemcpyHostToDevice));
        CK(cudaMemset(P->bad_seg.p, 0xff, sizeof(unsigned long long)));
        tr.mark("time points and offsets on the device");
    } catch (...) {
        delete P;
        throw;
    }
    return P;
}

int mzb_pj_create(const double *traj, uint64_t traj_size, const uint64_t *traj_offsets, const double *time,
                  uint64_t time_size, const uint64_t *time_offsets, uint64_t n_objs, uint32_t order, double maxT,
                  mzb_pj **out)
{
    return guarded([&]() {
        mzb_pj *P = pj_prepare(time, traj_size, traj_offsets, time_size, time_offsets, n_objs, order, maxT);
        try {
            dbuf<double> raw;
            raw.alloc(traj_size, 0);
            if (traj_size) CK(cudaMemcpy(raw.p, traj, traj_size * sizeof(double), cudaMemcpyDefault));
            launch_relayout(raw.p, P->coef.p, P->n_seg, int(order + 1), P->bad_seg.p, 0);
            CK(cudaDeviceSynchronize());
            P->check_data(0);
        } catch (...) {
            delete P;
            throw;
        }
        *out = P;
    });
}

// Pinned host memory the device can address: a kernel on a high-priority
// stream gathers each time chunk straight from it into the working layout
// (every byte crosses host memory once; packing pageable data for the copy
// engine moves it three times and is bound by the host's memory bandwidth).
static int create_gathered(const double *src, uint64_t traj_size, const uint64_t *traj_offsets, const double *time,
                           uint64_t time_size, const uint64_t *time_offsets, uint64_t n_objs, uint32_t order,
                           double maxT, uint32_t n_chunks, mzb_pj **out)
{
    return guarded([&]() {
        const call_trace tr;
        mzb_pj *P = pj_prepare(time, traj_size, traj_offsets, time_size, time_offsets, n_objs, order, maxT);
        tr.mark("polyjectory prepared");
        try {
            int lo_prio = 0, hi_prio = 0;
            CK(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
            CK(cudaStreamCreateWithPriority(&P->up, cudaStreamNonBlocking, hi_prio));
            const uint32_t K = std::clamp<uint32_t>(n_chunks ? n_chunks : 8, 1, 64);
            P->up_lo.resize(K);
            for (uint32_t c = 0; c < K; ++c) P->up_lo[c] = maxT * double(c) / double(K);
            const dev_pj V = P->view();
            for (uint32_t c = 0; c < K; ++c) {
                const double hi = (c + 1 < K) ? P->up_lo[c + 1] : maxT;
                launch_upload_chunk(src, P->coef.p, V.seg_off, V.time_off, V.nseg, V.time, n_objs, int(order + 1),
                                    P->up_lo[c], hi, c == 0, c + 1 == K, P->bad_seg.p, P->up);
                cudaEvent_t e = nullptr;
                CK(cudaEventCreate(&e)); // timed: the call trace reports when each chunk arrived
                P->up_ev.push_back(e);
                CK(cudaEventRecord(e, P->up));
            }
            CK(cudaGetLastError());
            tr.mark("upload chunks launched");
        } catch (...) {
            delete P;
            throw;
        }
        *out = P;
    });
}

int mzb_pj_create_async(const double *traj, uint64_t traj_size, const uint64_t *traj_offsets, const double *time,
                        uint64_t time_size, const uint64_t *time_offsets, uint64_t n_objs, uint32_t order,
                        double maxT, uint32_t n_chunks, mzb_pj **out)
{
    // Device trajectory data: the synchronous upload (a device-side copy).
    cudaPointerAttributes pa{};
    const bool attrs = traj_size && cudaPointerGetAttributes(&pa, traj) == cudaSuccess;
    cudaGetLastError(); // a pageable pointer may leave an error behind
    const bool on_device = attrs && (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
    const bool mapped = attrs && pa.type == cudaMemoryTypeHost && pa.devicePointer != nullptr;
    if (on_device || traj_size == 0)
        return mzb_pj_create(traj, traj_size, traj_offsets, time, time_size, time_offsets, n_objs, order, maxT, out);
    if (mapped) return create_gathered(static_cast<const double *>(pa.devicePointer), traj_size, traj_offsets, time,
                                       time_size, time_offsets, n_objs, order, maxT, n_chunks, out);
    return guarded([&]() {
        mzb_pj *P = pj_prepare(time, traj_size, traj_offsets, time_size, time_offsets, n_objs, order, maxT);
        try {
            const uint32_t K = std::clamp<uint32_t>(n_chunks ? n_chunks : 8, 1, 64);
            auto st = std::make_unique<stager>();
            CK(cudaGetDevice(&st->dev));
            st->traj = traj;
            st->op1 = int(order + 1);
            st->per_src = uint64_t(order + 1) * 7;
            st->coef = P->coef.p;
            st->bad_seg = P->bad_seg.p;
            st->lo.resize(K);
            for (uint32_t c = 0; c < K; ++c) st->lo[c] = maxT * double(c) / double(K);
            // Chunk boundaries of every object (first segment starting at or
            // after lo[c]), one pass over its time points.
            std::vector<uint64_t> keep_tm;
            std::vector<double> keep_time;
            const uint64_t *h_tm = host_view(time_offsets, n_objs, keep_tm);
            const double *h_time = host_view(time, time_size, keep_time);
            std::vector<uint32_t> bnd(size_t(n_objs) * (K + 1));
            for (uint64_t i = 0; i < n_objs; ++i) {
                const uint32_t ns = P->h_nseg[i];
                const double *t = h_time + h_tm[i];
                uint32_t *b = bnd.data() + i * (K + 1);
                b[0] = 0;
                uint32_t s = 0;
                for (uint32_t c = 1; c < K; ++c) {
                    while (s < ns && t[s] < st->lo[c]) ++s;
                    b[c] = s;
                }
                b[K] = ns;
            }
            // Pieces: runs of one chunk, in object order, split where a piece
            // (header + runs + data) would outgrow its slot.
            const uint64_t seg_bytes = st->per_src * sizeof(double);
            uint64_t cur_runs = 0, cur_seg = 0, run0 = 0;
            auto close_piece = [&]() {
                if (cur_runs) st->pieces.push_back(stage_piece{run0, run0 + cur_runs, cur_seg});
                run0 = st->runs.size();
                cur_runs = cur_seg = 0;
            };
            for (uint32_t c = 0; c < K; ++c) {
                for (uint64_t i = 0; i < n_objs; ++i) {
                    uint64_t a = bnd[i * (K + 1) + c];
                    const uint64_t e = bnd[i * (K + 1) + c + 1];
                    while (a < e) {
                        const uint64_t used = 16 + (cur_runs + 1) * sizeof(stage_run) + cur_seg * seg_bytes;
                        const uint64_t room = used < STAGE_SLOT_BYTES ? (STAGE_SLOT_BYTES - used) / seg_bytes : 0;
                        if (room == 0 || cur_runs == STAGE_MAX_RUNS) {
                            close_piece();
                            continue;
                        }
                        const uint64_t take = std::min<uint64_t>(e - a, room);
                        st->runs.push_back(stage_run{P->h_seg_off[i] + a, uint32_t(take), uint32_t(cur_seg)});
                        ++cur_runs;
                        cur_seg += take;
                        a += take;
                    }
                }
                close_piece();
                st->chunk_end.push_back(st->pieces.size());
            }
            // Host threads that pack the pieces: the environment variable
            // MZB_UPLOAD_THREADS, else half the hardware threads, at most 8
            // (8 threads copy at 75 GB/s on the benchmark's host, above the
            // link's 56 GB/s).
            unsigned W = std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2));
            if (const char *env = std::getenv("MZB_UPLOAD_THREADS")) {
                const long v = std::strtol(env, nullptr, 10);
                if (v > 0) W = unsigned(std::min<long>(v, 64));
            }
            st->start(W);
            P->stg = std::move(st);
        } catch (...) {
            delete P;
            throw;
        }
        *out = P;
    });
}

int mzb_pj_upload_wait(const mzb_pj *pj)
{
    return guarded([&]() {
        if (pj && pj->async_upload()) {
            pj->wait_upload_host();
            pj->check_data(0);
        }
    });
}

void mzb_pj_free(mzb_pj *pj) { delete pj; }

static int conjunctions_call(const mzb_pj *pj, double conj_thresh, double conj_det_interval, const int32_t *otypes,
                             const mzb_opts *opts, const mzb_host_outputs *dst, mzb_result **out)
{
    return guarded([&]() {
        if (!pj) throw invalid_arg("null polyjectory");
        // Argument checks of conjunctions::conjunctions (conjunctions.cpp:278-332).
        if (!std::isfinite(conj_thresh) || conj_thresh <= 0)
            throw invalid_arg("The conjunction threshold must be finite and positive, but instead a value of "
                              + fmt_d(conj_thresh) + " was provided");
        if (!std::isfinite(conj_thresh * conj_thresh))
            throw invalid_arg("A conjunction threshold of " + fmt_d(conj_thresh)
                              + " is too large and results in an overflow error");
        if (!std::isfinite(conj_det_interval) || conj_det_interval <= 0)
            throw invalid_arg("The conjunction detection interval must be finite and positive, but instead a value "
                              "of "
                              + fmt_d(conj_det_interval) + " was provided");
        bool skip_cd = true;
        if (otypes) {
            for (uint64_t i = 0; i < pj->n_objs; ++i) {
                const int32_t v = otypes[i];
                if (v != 1 && v != 2 && v != 4)
                    throw invalid_arg("The value of an object type must be one of [1, 2, 4], but a value of "
                                      + std::to_string(v) + " was detected instead");
                skip_cd = skip_cd && (v != 1);
            }
        } else {
            skip_cd = false;
        }
        const double nsd = std::ceil(pj->maxT / conj_det_interval);
        if (!(nsd >= 0) || !(nsd < 9.2e18)) throw invalid_arg("bad numeric conversion: number of conjunction steps");
        const uint64_t S = uint64_t(nsd);
        if (S == 0) throw invalid_arg("bad numeric conversion: zero conjunction steps");
        uint64_t sb = 0, se = S;
        if (opts && (opts->step_begin || opts->step_end)) {
            sb = opts->step_begin;
            se = std::min<uint64_t>(opts->step_end, S);
            if (!(sb < se)) throw invalid_arg("empty step range");
        }
        auto *R = new mzb_result;
        try {
            R->n_cd_steps = S;
            R->step_begin = sb;
            R->n_run = se - sb;
            R->n_objs = pj->n_objs;
            uint32_t spb = (opts && opts->steps_per_batch) ? opts->steps_per_batch : 0;
            if (spb == 0) {
                // Batch scratch is ~184 bytes per object and step (248 in the
                // mixed form); stay near 3 GB.
                const uint64_t per_step = 248ull * pj->n_objs + 4096;
                spb = uint32_t(std::clamp<uint64_t>((3ull << 30) / per_step, 16, 1024));
            }
            const bool mixed = opts && opts->form == MZB_FORM_MIXED;
            if (opts && opts->form != MZB_FORM_PLAIN && opts->form != MZB_FORM_MIXED)
                throw invalid_arg("unknown screening form " + std::to_string(opts->form));
            const uint32_t bvh_threads = opts ? opts->bvh_threads : 0;
            if (bvh_threads != 0 && bvh_threads != 256 && bvh_threads != 512 && bvh_threads != 1024)
                throw invalid_arg("unsupported BVH block size " + std::to_string(bvh_threads)
                                  + ": expected 0 (automatic), 256, 512 or 1024");
            const uint32_t broad_walk = opts ? opts->broad_walk : 0;
            if (broad_walk > 2)
                throw invalid_arg("unsupported broad-phase walk " + std::to_string(broad_walk)
                                  + ": expected 0 (one position per thread), 1 (warp-coherent) or 2 (walks with "
                                    "work refill)");
            if (opts && opts->reserved != 0) throw invalid_arg("mzb_opts.reserved must be 0");
            const uint32_t sort_threads = opts ? opts->sort_threads : 0;
            if (sort_threads != 0 && sort_threads != 256 && sort_threads != 512)
                throw invalid_arg("unsupported sort block size " + std::to_string(sort_threads)
                                  + ": expected 0 (automatic), 256 or 512");
            run_detection(*pj, conj_thresh, conj_det_interval, otypes, skip_cd, spb, mixed,
                          int(bvh_threads), int(broad_walk),
                          sort_threads ? int(sort_threads) : 512, dst, *R);
        } catch (...) {
            delete R;
            throw;
        }
        *out = R;
    });
}

int mzb_conjunctions(const mzb_pj *pj, double conj_thresh, double conj_det_interval, const int32_t *otypes,
                     const mzb_opts *opts, mzb_result **out)
{
    return conjunctions_call(pj, conj_thresh, conj_det_interval, otypes, opts, nullptr, out);
}

int mzb_conjunctions_stream(const mzb_pj *pj, double conj_thresh, double conj_det_interval, const int32_t *otypes,
                            const mzb_opts *opts, const mzb_host_outputs *dst, mzb_result **out)
{
    return conjunctions_call(pj, conj_thresh, conj_det_interval, otypes, opts, dst, out);
}

void mzb_result_free(mzb_result *r) { delete r; }
uint64_t mzb_result_n_cd_steps(const mzb_result *r) { return r->n_cd_steps; }
uint64_t mzb_result_n_objs(const mzb_result *r) { return r->n_objs; }
uint64_t mzb_result_step_begin(const mzb_result *r) { return r->step_begin; }
uint64_t mzb_result_n_steps_run(const mzb_result *r) { return r->n_run; }
uint64_t mzb_result_n_launches(const mzb_result *r) { return r->n_launches; }

#define MZB_COPY(name, field, T, count)                                                                              \
    int name(const mzb_result *r, T *dst)                                                                              \
    {                                                                                                                  \
        return guarded([&]() {                                                                                         \
            const size_t n_ = (count);                                                                                 \
            if (n_) CK(cudaMemcpy(dst, r->field.p, n_ * sizeof(T), cudaMemcpyDefault));                               \
        });                                                                                                            \
    }

MZB_COPY(mzb_result_copy_aabbs, aabbs, float, r->n_run * (r->n_objs + 1) * 8)
MZB_COPY(mzb_result_copy_srt_aabbs, srt_aabbs, float, r->n_run * (r->n_objs + 1) * 8)
MZB_COPY(mzb_result_copy_mcodes, mcodes, uint64_t, r->n_run * r->n_objs)
MZB_COPY(mzb_result_copy_srt_mcodes, srt_mcodes, uint64_t, r->n_run * r->n_objs)
MZB_COPY(mzb_result_copy_srt_idx, srt_idx, uint32_t, r->n_run * r->n_objs)
#undef MZB_COPY

int mzb_result_copy_cd_end_times(const mzb_result *r, double *dst)
{
    return guarded([&]() { CK(cudaMemcpy(dst, r->cd_end.data(), r->cd_end.size() * sizeof(double), cudaMemcpyDefault)); });
}

int mzb_result_tree_offsets(const mzb_result *r, uint64_t *os)
{
    return guarded([&]() {
        std::vector<uint32_t> sz(r->n_run);
        CK(cudaMemcpy(sz.data(), r->tree_size.p, sz.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        uint64_t off = 0;
        for (uint64_t s = 0; s < r->n_run; ++s) {
            os[2 * s] = off;
            os[2 * s + 1] = sz[s];
            off += sz[s];
        }
    });
}

uint64_t mzb_result_n_tree_nodes(const mzb_result *r)
{
    std::vector<uint32_t> sz(r->n_run);
    if (cudaMemcpy(sz.data(), r->tree_size.p, sz.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return 0;
    uint64_t t = 0;
    for (auto v : sz) t += v;
    return t;
}

int mzb_result_copy_trees(const mzb_result *r, void *dst)
{
    return guarded([&]() {
        std::vector<uint32_t> sz(r->n_run);
        CK(cudaMemcpy(sz.data(), r->tree_size.p, sz.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        std::vector<uint64_t> off(r->n_run);
        uint64_t tot = 0;
        for (uint64_t s = 0; s < r->n_run; ++s) {
            off[s] = tot;
            tot += sz[s];
        }
        if (tot == 0) return;
        // Trees live at a fixed per-step capacity: pack them on the device,
        // then one copy to the caller.
        dbuf<uint64_t> d_off;
        dbuf<bvh_node> packed;
        d_off.alloc(off.size(), 0);
        packed.alloc(tot, 0);
        CK(cudaMemcpy(d_off.p, off.data(), off.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
        launch_tree_gather(r->trees.p, r->cap, d_off.p, r->tree_size.p, r->n_run, packed.p, 0);
        CK(cudaMemcpy(dst, packed.p, tot * sizeof(bvh_node), cudaMemcpyDefault));
    });
}

int mzb_result_bp_offsets(const mzb_result *r, uint64_t *os)
{
    return guarded([&]() { std::memcpy(os, r->bp_off.data(), r->bp_off.size() * sizeof(uint64_t)); });
}

uint64_t mzb_result_n_bp(const mzb_result *r) { return r->n_bp; }

uint64_t mzb_result_broad_visits(const mzb_result *r) { return r->broad_visits; }

int mzb_result_copy_bp(const mzb_result *r, void *dst)
{
    return guarded([&]() {
        if (r->n_bp) CK(cudaMemcpy(dst, r->bp.p, r->n_bp * sizeof(uint2), cudaMemcpyDefault));
    });
}

uint64_t mzb_result_n_conj(const mzb_result *r) { return r->n_conj; }

int mzb_result_copy_conj(const mzb_result *r, void *dst)
{
    return guarded([&]() {
        if (r->n_conj) CK(cudaMemcpy(dst, r->conj.p, r->n_conj * sizeof(conj_rec), cudaMemcpyDefault));
    });
}

int mzb_result_write_files(const mzb_result *r, const char *data_dir)
{
    return guarded([&]() {
        if (!r) throw invalid_arg("null result");
        if (!data_dir) throw invalid_arg("null data directory");
        struct stat sb;
        if (::stat(data_dir, &sb) != 0 || !S_ISDIR(sb.st_mode))
            throw invalid_arg(std::string("The data directory '") + data_dir + "' does not exist");
        const std::string dir(data_dir);
        const uint64_t S = r->n_run, N = r->n_objs;
        file_stager sg;
        device_to_file(sg, dir + "/aabbs", r->aabbs.p, S * (N + 1) * 8 * sizeof(float), nullptr, 0);
        device_to_file(sg, dir + "/srt_aabbs", r->srt_aabbs.p, S * (N + 1) * 8 * sizeof(float), nullptr, 0);
        device_to_file(sg, dir + "/mcodes", r->mcodes.p, S * N * sizeof(uint64_t), nullptr, 0);
        device_to_file(sg, dir + "/srt_mcodes", r->srt_mcodes.p, S * N * sizeof(uint64_t), nullptr, 0);
        device_to_file(sg, dir + "/vidx", r->srt_idx.p, S * N * sizeof(uint32_t), nullptr, 0);
        // Trees sit at a fixed capacity per step: pack them first.
        {
            std::vector<uint32_t> sz(S);
            if (S) CK(cudaMemcpy(sz.data(), r->tree_size.p, S * sizeof(uint32_t), cudaMemcpyDeviceToHost));
            std::vector<uint64_t> off(S);
            uint64_t tot = 0;
            for (uint64_t k = 0; k < S; ++k) {
                off[k] = tot;
                tot += sz[k];
            }
            dbuf<uint64_t> d_off;
            dbuf<bvh_node> packed;
            if (tot) {
                d_off.alloc(S, 0);
                packed.alloc(tot, 0);
                CK(cudaMemcpy(d_off.p, off.data(), S * sizeof(uint64_t), cudaMemcpyHostToDevice));
                launch_tree_gather(r->trees.p, r->cap, d_off.p, r->tree_size.p, S, packed.p, 0);
                CK(cudaDeviceSynchronize());
            }
            device_to_file(sg, dir + "/bvh", packed.p, tot * sizeof(bvh_node), nullptr, 0);
        }
        // No pairs: one value-initialised aabb_collision; no conjunctions: a
        // single byte (detect_conjunctions.cpp:466-487).
        static const char zeros[sizeof(uint2)] = {};
        device_to_file(sg, dir + "/bp", r->bp.p, r->n_bp * sizeof(uint2), zeros, sizeof(uint2));
        device_to_file(sg, dir + "/conjunctions", r->conj.p, r->n_conj * sizeof(conj_rec), zeros, 1);
    });
}

struct mzb_sgp4_pj {
    std::unique_ptr<sgp4pj::sgp4_pj_out> o;
};

int mzb_make_sgp4_polyjectory(const mzb_gpe *gpes, uint64_t n_gpes, double jd_begin, double jd_end,
                              double reentry_radius, double exit_radius, mzb_sgp4_pj **out)
{
    return guarded([&]() {
        std::vector<mzb_gpe> keep;
        const mzb_gpe *g = host_view(gpes, n_gpes, keep);
        auto r = std::make_unique<mzb_sgp4_pj>();
        r->o.reset(sgp4pj::make_sgp4_pj(g, n_gpes, jd_begin, jd_end, reentry_radius, exit_radius));
        *out = r.release();
    });
}

void mzb_sgp4_pj_sizes(const mzb_sgp4_pj *p, uint64_t out[4])
{
    out[0] = p->o->status.size();
    out[1] = p->o->n_traj;
    out[2] = p->o->time.size();
    out[3] = uint64_t(sgp4pj::ORDER);
}

void mzb_sgp4_pj_epoch(const mzb_sgp4_pj *p, double out[3])
{
    out[0] = p->o->epoch.hi;
    out[1] = p->o->epoch.lo;
    out[2] = p->o->maxT;
}

int mzb_sgp4_pj_copy(const mzb_sgp4_pj *p, double *traj, uint64_t *traj_offsets, double *time,
                     uint64_t *time_offsets, int32_t *status)
{
    return guarded([&]() {
        const sgp4pj::sgp4_pj_out &o = *p->o;
        auto put = [](void *dst, const void *src, size_t bytes) {
            if (dst && bytes) CK(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
        };
        put(traj, o.d_traj, o.n_traj * sizeof(double));
        put(traj_offsets, o.traj_off.data(), o.traj_off.size() * sizeof(uint64_t));
        put(time, o.time.data(), o.time.size() * sizeof(double));
        put(time_offsets, o.time_off.data(), o.time_off.size() * sizeof(uint64_t));
        put(status, o.status.data(), o.status.size() * sizeof(int32_t));
    });
}

void mzb_sgp4_pj_free(mzb_sgp4_pj *p) { delete p; }

void mzb_sgp4_pj_timing(const mzb_sgp4_pj *p, double out[2])
{
    out[0] = p->o->kernel_ms;
    out[1] = p->o->gather_ms;
}

int mzb_sgp4_propagate(const mzb_gpe *gpes, uint64_t n_gpes, const double *tsince, uint64_t n_times, double *out,
                       int32_t *err)
{
    return guarded([&]() {
        std::vector<mzb_gpe> keep;
        const mzb_gpe *g = host_view(gpes, n_gpes, keep);
        sgp4pj::sgp4_propagate(g, n_gpes, tsince, n_times, out, err);
    });
}

int mzb_sort_step_noalloc(const float *aabbs, const uint64_t *mcodes, uint64_t n_objs, uint32_t *srt_idx,
                          uint64_t *srt_mcodes, float *srt_aabbs, void *stream)
{
    return guarded([&]() {
        if (n_objs == 0) throw invalid_arg("mzb_sort_step_noalloc: the number of objects must be positive");
        if (n_objs > sort_noalloc_max_objs())
            throw invalid_arg("mzb_sort_step_noalloc: " + std::to_string(n_objs)
                              + " objects exceed the capacity of the built-in scratch array ("
                              + std::to_string(sort_noalloc_max_objs()) + " objects)");
        CK(sort_step_noalloc(aabbs, mcodes, n_objs, srt_idx, srt_mcodes, srt_aabbs,
                             static_cast<cudaStream_t>(stream)));
    });
}

int mzb_pj_state_eval(const mzb_pj *pj, double *out, uint64_t out_rows, const double *tm, int64_t tm_size,
                      const uint64_t *sel, int64_t sel_size)
{
    return guarded([&]() {
        if (!pj) throw invalid_arg("null polyjectory");
        // Size checks of polyjectory::state_eval_impl (polyjectory.cpp:1168-1228).
        const bool has_sel = sel_size >= 0, tm_arr = tm_size >= 0;
        const uint64_t n_eval = has_sel ? uint64_t(sel_size) : pj->n_objs;
        if (has_sel) {
            if (out_rows != n_eval)
                throw invalid_arg("Invalid output array passed to state_eval(): the number of objects selected for "
                                  "evaluation is "
                                  + std::to_string(n_eval) + " but the size of the first dimension of the array is "
                                  + std::to_string(out_rows) + " (the two numbers must be equal)");
            if (tm_arr && uint64_t(tm_size) != n_eval)
                throw invalid_arg("Invalid time array passed to state_eval(): the number of selected objects is "
                                  + std::to_string(n_eval) + " but the size of the array is "
                                  + std::to_string(tm_size) + " (the two numbers must be equal)");
        } else {
            if (out_rows != n_eval)
                throw invalid_arg("Invalid output array passed to state_eval(): the number of objects is "
                                  + std::to_string(n_eval) + " but the size of the first dimension of the array is "
                                  + std::to_string(out_rows) + " (the two numbers must be equal)");
            if (tm_arr && uint64_t(tm_size) != n_eval)
                throw invalid_arg("Invalid time array passed to state_eval(): the number of objects is "
                                  + std::to_string(n_eval) + " but the size of the array is "
                                  + std::to_string(tm_size) + " (the two numbers must be equal)");
        }
        run_state_eval(pj, out, tm, tm_arr ? 1 : 0, 0, has_sel ? sel : nullptr, n_eval, 1);
    });
}

int mzb_pj_state_meval(const mzb_pj *pj, double *out, uint64_t out_d0, uint64_t out_d1, const double *tm,
                       uint32_t tm_ndim, uint64_t tm_d0, uint64_t tm_d1, const uint64_t *sel, int64_t sel_size)
{
    return guarded([&]() {
        if (!pj) throw invalid_arg("null polyjectory");
        if (tm_ndim != 1 && tm_ndim != 2)
            throw invalid_arg("The time array passed to state_meval() must have either 1 or 2 dimensions, but the "
                              "number of dimensions is "
                              + std::to_string(tm_ndim) + " instead");
        // Size checks of polyjectory::state_meval_impl (polyjectory.cpp:1258-1336).
        const uint64_t n_t = tm_ndim == 1 ? tm_d0 : tm_d1;
        if (out_d1 != n_t)
            throw invalid_arg("Invalid output array passed to state_meval(): the number of time evaluations per "
                              "object is "
                              + std::to_string(n_t) + " but the size of the second dimension of the array is "
                              + std::to_string(out_d1) + " (the two numbers must be equal)");
        const bool has_sel = sel_size >= 0;
        const uint64_t n_eval = has_sel ? uint64_t(sel_size) : pj->n_objs;
        const char *what = has_sel ? "selected objects" : "objects";
        if (out_d0 != n_eval)
            throw invalid_arg(std::string("Invalid output array passed to state_meval(): the number of ") + what
                              + " is " + std::to_string(n_eval)
                              + " but the size of the first dimension of the array is " + std::to_string(out_d0)
                              + " (the two numbers must be equal)");
        if (tm_ndim == 2 && tm_d0 != n_eval)
            throw invalid_arg(std::string("Invalid time array passed to state_meval(): the number of ") + what
                              + " is " + std::to_string(n_eval)
                              + " but the size of the first dimension of the array is " + std::to_string(tm_d0)
                              + " (the two numbers must be equal)");
        run_state_eval(pj, out, tm, tm_ndim == 2 ? n_t : 0, 1, has_sel ? sel : nullptr, n_eval, n_t);
    });
}

int mzb_scratch_release(void)
{
    return guarded([&]() {
        scratch_cache &c = device_scratch();
        std::lock_guard<std::mutex> lk(c.m);
        for (scratch_slot &sl : c.slots) {
            if (sl.p) CK(cudaFreeAsync(sl.p, 0));
            sl.p = nullptr;
            sl.bytes = 0;
        }
        {
            std::lock_guard<std::mutex> lk2(c.spare_m);
            if (c.spare) CK(cudaFreeAsync(c.spare, 0));
            c.spare = nullptr;
            c.spare_bytes = 0;
        }
        CK(cudaStreamSynchronize(0));
    });
}

uint64_t mzb_scratch_bytes(void)
{
    uint64_t b = 0;
    try {
        scratch_cache &c = device_scratch();
        std::lock_guard<std::mutex> lk(c.m);
        for (const scratch_slot &sl : c.slots) b += sl.bytes;
        std::lock_guard<std::mutex> lk2(c.spare_m);
        b += c.spare_bytes;
    } catch (...) {
    }
    return b;
}

int mzb_measure_fp64_rate(double *dfma_per_second)
{
    return guarded([&]() { CK(measure_dfma_rate(dfma_per_second)); });
}

void mzb_result_narrow_split(const mzb_result *r, uint64_t out[2])
{
    out[0] = r->narrow_split[0];
    out[1] = r->narrow_split[1];
}

void mzb_result_np_report(const mzb_result *r, uint64_t out[7])
{
    for (int k = 0; k < 7; ++k) out[k] = r->np[k];
}

void mzb_result_stage_ms(const mzb_result *r, double out[8])
{
    for (int k = 0; k < 8; ++k) out[k] = r->stage_ms[k];
}
}
