/*
 * mizuba_b200: B200 (sm_100a) conjunction screening behind a C ABI.
 *
 * This is the drop-in boundary for mizuba's conjunction-detection hot path:
 * plain pointers and sizes, status codes instead of exceptions, no C++ or
 * torch types.  Every entry point names the reference interface it replaces
 * (paths relative to the mizuba source tree).
 *
 * Units and layouts are mizuba's: polyjectory times in the polyjectory's time
 * unit (days for SGP4 polyjectories), trajectory data as per-object
 * [n_steps][order + 1][7] doubles (x, y, z, vx, vy, vz, r), and the output
 * records byte-identical to conjunctions::bvh_node (48 B),
 * conjunctions::aabb_collision (8 B) and conjunctions::conj (120 B).
 */
#ifndef MIZUBA_B200_H
#define MIZUBA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MZB_OK 0
#define MZB_INVALID_ARGUMENT 1 /* std::invalid_argument in the reference */
#define MZB_OUT_OF_RANGE 2     /* std::out_of_range in the reference */
#define MZB_RUNTIME_ERROR 3    /* CUDA or allocation failure */

typedef struct mzb_pj mzb_pj;         /* a polyjectory resident in HBM */
typedef struct mzb_result mzb_result; /* a conjunctions result resident in HBM */

/* Screening forms.
 * MZB_FORM_PLAIN: the reference's FP64 formulation operation for operation
 *   (boxes, codes, order, trees and pairs bit-exact with the oracle).
 * MZB_FORM_MIXED: FMA-native FP64 enclosures widened by an a-posteriori
 *   rounding bound (boxes provably contain the plain form's, so overlapping
 *   pairs are a superset), FP32 broad phase as in the plain form, a
 *   rigorous distance screen (linear model with a Taylor remainder bound),
 *   and an FMA-native FP64 prefilter of the narrow phase (shifted-node
 *   evaluation, conservative prune) whose survivors are recomputed with the
 *   reference formulation: the conjunction records are the plain form's
 *   (the narrow-phase counters are not: fewer items reach root finding). */
#define MZB_FORM_PLAIN 0u
#define MZB_FORM_MIXED 1u

/* Options of one screening call (NULL = defaults). */
typedef struct mzb_opts {
    uint32_t steps_per_batch; /* conjunction steps per batch (0 = automatic) */
    uint32_t form;            /* MZB_FORM_PLAIN (default) or MZB_FORM_MIXED */
    uint64_t step_begin;      /* screen only steps [step_begin, step_end); */
    uint64_t step_end;        /* 0, 0 = all steps (a shard of the time axis) */
    uint32_t bvh_threads;     /* BVH build: 0 = one-pass build; 256, 512, 1024 = level-by-level build with that CTA size */
    uint32_t broad_walk;      /* broad phase: 0 = one position per thread, 1 = warp-coherent, 2 = walks with work refill */
    uint32_t sort_threads;    /* CTA size of the step sort: 256, 512 (0 = 512) */
    uint32_t reserved;        /* must be 0 */
} mzb_opts;

/* Message of the last failed call on this thread (the reference's exception
 * text where one exists). */
const char *mzb_last_error(void);

/* Uploads a polyjectory once.  Replaces the in-memory polyjectory
 * constructor's data handling (mizuba/polyjectory.cpp:352-619) and the
 * per-object accessor polyjectory::operator[] (mizuba/polyjectory.cpp:1006-1036):
 * traj_offsets holds, per object, (offset in doubles into traj, n_steps);
 * time_offsets holds per object the offset into time (n_steps + 1 values, or
 * none for an empty trajectory).  Arrays are host or device pointers (UVA).
 * The constructor's checks come first, with its messages: offsets within the
 * data, time points finite, non-negative and strictly increasing per object,
 * at least one non-empty trajectory (mizuba/polyjectory.cpp:460-600), maxT
 * equal to the largest end time, and finite trajectory values (checked on
 * the device while the data are uploaded); any failure returns
 * MZB_INVALID_ARGUMENT and creates nothing. */
int mzb_pj_create(const double *traj, uint64_t traj_size, const uint64_t *traj_offsets, const double *time,
                  uint64_t time_size, const uint64_t *time_offsets, uint64_t n_objs, uint32_t order, double maxT,
                  mzb_pj **out);
void mzb_pj_free(mzb_pj *pj);

/* mzb_pj_create that returns before the trajectory data is on the device.
 * The segments are uploaded in n_chunks time chunks (0 = 8), each chunk
 * holding the segments that start in its share of [0, maxT).  When traj is
 * pinned host memory the device can address (cudaHostAlloc, cudaMallocHost,
 * torch's pin_memory, or cudaHostRegister with the mapped flag), a kernel on
 * a high-priority stream gathers each chunk straight from it; other host
 * memory (pageable, e.g. a memory-mapped file) is packed chunk by chunk by
 * host threads (MZB_UPLOAD_THREADS, default half the hardware threads, at
 * most 8) into 16 MB pinned pieces that the copy engine moves and a kernel
 * puts in place.  Screening calls on this polyjectory then wait, batch by
 * batch, only for the chunks their steps need, so the upload overlaps the
 * screening of the earlier steps and the copies of their outputs (pass
 * steps_per_batch to get several batches).  traj must stay valid and
 * unchanged until mzb_pj_upload_wait returns (or the polyjectory is freed,
 * which waits).  With a device pointer this is mzb_pj_create.  The other
 * arrays are read before the call returns.  No counterpart in the reference
 * (its polyjectory is memory-mapped files). */
int mzb_pj_create_async(const double *traj, uint64_t traj_size, const uint64_t *traj_offsets, const double *time,
                        uint64_t time_size, const uint64_t *time_offsets, uint64_t n_objs, uint32_t order,
                        double maxT, uint32_t n_chunks, mzb_pj **out);
/* Blocks until the trajectory upload of mzb_pj_create_async has finished
 * (returns at once for other polyjectories).  The trajectory values of an
 * asynchronous upload are checked as they arrive: a non-finite value makes
 * this call, and any screening or evaluation call that has waited for it,
 * return MZB_INVALID_ARGUMENT with the constructor's message. */
int mzb_pj_upload_wait(const mzb_pj *pj);

/* State evaluation on the GPU.  Replaces polyjectory::state_eval
 * (mizuba/polyjectory.cpp:1162-1251), whose per-evaluation work is
 * pj_eval_obj_state (mizuba/polyjectory.cpp:1092-1159): the 7 state
 * variables of each selected object at one time, by Horner's scheme in the
 * reference's operation order; NaN where the object has no data at that time
 * (no trajectory, before its first time point, at or after its last).
 *   out      double[out_rows][7] (host memory);
 *   tm       tm_size < 0: one time *tm for every evaluated object;
 *            otherwise an array of tm_size times, one per evaluated object;
 *   sel      sel_size < 0: all objects in order (sel ignored); otherwise
 *            sel_size object indices.
 * Same size checks and messages as the reference; a non-finite time returns
 * MZB_INVALID_ARGUMENT, an object index out of range MZB_OUT_OF_RANGE. */
int mzb_pj_state_eval(const mzb_pj *pj, double *out, uint64_t out_rows, const double *tm, int64_t tm_size,
                      const uint64_t *sel, int64_t sel_size);

/* Multiple-time state evaluation.  Replaces polyjectory::state_meval
 * (mizuba/polyjectory.cpp:1253-1366).
 *   out      double[out_d0][out_d1][7] (host memory);
 *   tm       tm_ndim 1: tm_d0 times shared by every evaluated object;
 *            tm_ndim 2: double[tm_d0][tm_d1], one row per evaluated object;
 *   sel      as in mzb_pj_state_eval. */
int mzb_pj_state_meval(const mzb_pj *pj, double *out, uint64_t out_d0, uint64_t out_d1, const double *tm,
                       uint32_t tm_ndim, uint64_t tm_d0, uint64_t tm_d1, const uint64_t *sel, int64_t sel_size);

/* Runs conjunction detection.  Replaces conjunctions::conjunctions
 * (mizuba/conjunctions.cpp:263-360) and conjunctions::detect_conjunctions
 * (mizuba/detect_conjunctions.cpp:53-537): same argument checks and messages,
 * same n_cd_steps = ceil(maxT / conj_det_interval), same outputs.  otypes may
 * be NULL (all primaries, mizuba/conjunctions.cpp:301-332).  Outputs stay in
 * HBM until copied out with the accessors below. */
int mzb_conjunctions(const mzb_pj *pj, double conj_thresh, double conj_det_interval, const int32_t *otypes,
                     const mzb_opts *opts, mzb_result **out);
void mzb_result_free(mzb_result *r);

/* Host destinations of a streaming screening call (NULL members are skipped).
 * Sizes as for the accessors below, over the screened steps:
 *   aabbs, srt_aabbs float[n_steps_run][n_objs + 1][2][4]; mcodes, srt_mcodes
 *   uint64[n_steps_run][n_objs]; srt_idx uint32[n_steps_run][n_objs];
 *   cd_end_times double[n_steps_run]; trees: room for trees_cap 48-byte
 *   nodes, filled packed in step order (at most n_steps_run * (2 n_objs - 1)
 *   nodes are needed). */
typedef struct mzb_host_outputs {
    float *aabbs;
    float *srt_aabbs;
    uint64_t *mcodes;
    uint64_t *srt_mcodes;
    uint32_t *srt_idx;
    double *cd_end_times;
    void *trees;
    uint64_t trees_cap;
} mzb_host_outputs;

/* mzb_conjunctions that also streams the per-step arrays and the trees into
 * host memory while it computes: each batch's boxes, codes and order are
 * copied on a second stream as soon as the sort has run, its trees as soon as
 * they are built, so the transfers overlap the broad and narrow phases.  This
 * is the GPU form of the reference's writer thread, which writes each step's
 * outputs while later steps are screened (mizuba/detect_conjunctions.cpp:184-242).
 * The buffers should be pinned (cudaHostAlloc / cudaHostRegister) for the
 * copies to overlap; they are complete when the call returns.  Pairs and
 * conjunctions are read afterwards with the accessors, as are the copies
 * above (the result keeps its device arrays). */
int mzb_conjunctions_stream(const mzb_pj *pj, double conj_thresh, double conj_det_interval, const int32_t *otypes,
                            const mzb_opts *opts, const mzb_host_outputs *dst, mzb_result **out);

/* Sizes (conjunctions::get_n_cd_steps, mizuba/conjunctions.cpp:461-464).
 * The per-step outputs below cover the screened steps
 * [mzb_result_step_begin, mzb_result_step_begin + mzb_result_n_steps_run),
 * which is all n_cd_steps steps unless mzb_opts selected a shard. */
uint64_t mzb_result_n_cd_steps(const mzb_result *r);
uint64_t mzb_result_n_objs(const mzb_result *r);
uint64_t mzb_result_step_begin(const mzb_result *r);
uint64_t mzb_result_n_steps_run(const mzb_result *r);

/* Copies of the dense per-step outputs into caller memory (host or device):
 *   aabbs, srt_aabbs  float[n_cd_steps][n_objs + 1][2][4]  (conjunctions.cpp:394-408)
 *   mcodes, srt_mcodes uint64[n_cd_steps][n_objs]          (conjunctions.cpp:410-418)
 *   srt_idx           uint32[n_cd_steps][n_objs]           (conjunctions.cpp:420-423)
 *   cd_end_times      double[n_cd_steps]                   (conjunctions.cpp:399-402) */
int mzb_result_copy_aabbs(const mzb_result *r, float *dst);
int mzb_result_copy_srt_aabbs(const mzb_result *r, float *dst);
int mzb_result_copy_mcodes(const mzb_result *r, uint64_t *dst);
int mzb_result_copy_srt_mcodes(const mzb_result *r, uint64_t *dst);
int mzb_result_copy_srt_idx(const mzb_result *r, uint32_t *dst);
int mzb_result_copy_cd_end_times(const mzb_result *r, double *dst);

/* BVH trees (conjunctions::get_bvh_tree, mizuba/conjunctions.cpp:425-441):
 * per-step (offset, size) pairs in nodes, then all trees concatenated. */
int mzb_result_tree_offsets(const mzb_result *r, uint64_t *offsets_sizes /* [n_cd_steps][2] */);
uint64_t mzb_result_n_tree_nodes(const mzb_result *r);
int mzb_result_copy_trees(const mzb_result *r, void *dst /* 48-byte nodes */);

/* Broad-phase collisions (conjunctions::get_aabb_collisions,
 * mizuba/conjunctions.cpp:443-459): per-step (offset, size), concatenated. */
int mzb_result_bp_offsets(const mzb_result *r, uint64_t *offsets_sizes /* [n_cd_steps][2] */);
uint64_t mzb_result_n_bp(const mzb_result *r);
int mzb_result_copy_bp(const mzb_result *r, void *dst /* 8-byte pairs */);

/* Conjunctions (conjunctions::get_conjunctions, mizuba/conjunctions.cpp:478-491),
 * sorted per step by (tca, record) and concatenated in step order. */
uint64_t mzb_result_n_conj(const mzb_result *r);
int mzb_result_copy_conj(const mzb_result *r, void *dst /* 120-byte records */);

/* Writes the result into the files mizuba keeps in a conjunctions object's
 * data directory (mizuba/detect_conjunctions.cpp:92-126 and :466-534):
 * aabbs, srt_aabbs, mcodes, srt_mcodes, vidx, bvh, bp and conjunctions, as
 * the raw arrays above (trees and pairs packed in step order), with the
 * reference's sentinels (one zeroed aabb_collision in bp when there are no
 * pairs, a single byte in conjunctions when there are no conjunctions), each
 * left readable by its owner only.  data_dir must exist; the files must not.
 * The data leave HBM through pinned staging buffers, copy and write
 * overlapped. */
int mzb_result_write_files(const mzb_result *r, const char *data_dir);

/* Narrow-phase statistics (conjunctions::np_report, mizuba/conjunctions.hpp:150-175):
 * candidates, dist2-pruned, root findings, fast exclusions, no-root,
 * minima, discarded minima. */
void mzb_result_np_report(const mzb_result *r, uint64_t out[7]);

/* Mixed form only (zeros otherwise): the items that passed the distance
 * screen, and of those the ones the FMA prefilter kept for the reference
 * formulation.  No counterpart in the reference (its narrow phase has
 * neither stage). */
void mzb_result_narrow_split(const mzb_result *r, uint64_t out[2]);

/* Device time per stage in ms (the stopwatch breakdown of
 * mizuba/detect_conjunctions.cpp:444-454): aabb, morton + sort, bvh, broad,
 * narrow, roots, per-step conjunction ordering, total. */
void mzb_result_stage_ms(const mzb_result *r, double out[8]);

/* Broad-phase tree-node visits of the call (the default walk counts them;
 * 0 for the alternative walks): the work unit of the broad phase's
 * roofline.  No counterpart in the reference. */
uint64_t mzb_result_broad_visits(const mzb_result *r);

/* Number of kernel launches the call issued (mizuba's stages have no
 * counterpart: it runs on CPU threads). */
uint64_t mzb_result_n_launches(const mzb_result *r);

/* Screening calls keep their batch scratch (a few GB at the default batch
 * size, sized by the largest call so far) on the device between calls, so
 * that repeated calls allocate nothing; a freed result's block of per-step
 * outputs is also kept, as the spare the next call of the same size takes.
 * This returns the current device's cached blocks and spare to the
 * stream-ordered pool; it waits for a screening call in progress on the
 * device to finish.  No counterpart in the reference (its buffers are host
 * memory owned by each call). */
int mzb_scratch_release(void);
/* Bytes of batch scratch and spare output block cached on the current
 * device. */
uint64_t mzb_scratch_bytes(void);

/* Measures the current device's FP64 FMA issue rate (instructions per
 * second) with a DFMA throughput kernel: the denominator of the roofline of
 * the FP64-bound stages.  No counterpart in the reference (a measurement
 * utility; it allocates and frees a small buffer). */
int mzb_measure_fp64_rate(double *dfma_per_second);

/* ---- SGP4 polyjectories on the GPU. */

/* One general perturbations element set, byte-identical to mizuba's gpe
 * struct (mizuba/make_sgp4_polyjectory.hpp): NORAD ID; epoch as a two-part
 * UTC Julian date; mean motion n0 [rad/min]; eccentricity e0; inclination
 * i0, right ascension of the ascending node node0, argument of perigee
 * omega0 and mean anomaly m0 [rad]; drag term bstar [1/earth radii]. */
typedef struct mzb_gpe {
    uint64_t norad_id;
    double epoch_jd1, epoch_jd2;
    double n0, e0, i0, node0, omega0, m0, bstar;
} mzb_gpe;

typedef struct mzb_sgp4_pj mzb_sgp4_pj; /* a produced polyjectory (host arrays) */

/* Builds the polyjectory of a set of element sets over [jd_begin, jd_end)
 * (UTC Julian dates) on the GPU.  Replaces make_sgp4_polyjectory
 * (mizuba/make_sgp4_polyjectory.cpp:1461-1603, the interpolation of
 * :478-913): the same argument checks and messages (dates, radii, finite
 * fields, order by NORAD ID then epoch); one object per NORAD ID, each
 * element set used from its epoch (the first one from jd_begin) to the next
 * set's epoch; steps of Keplerian motion from the SGP4 state, order-18
 * Chebyshev interpolation of x, y, z, vx, vy, vz, r in days from the
 * polyjectory epoch (jd_begin in TAI), bisection below 1e-7 km of position
 * error; per object the reference's status code (0, the propagator's 1-6,
 * 10 non-finite, 11 reentry, 12 exit, 13 step under 1 s, 14 more than 20
 * polynomials in a step).  Near-Earth and deep-space (SDP4) element sets
 * alike.  An object whose status is not 0 keeps the steps completed before
 * the failure. */
int mzb_make_sgp4_polyjectory(const mzb_gpe *gpes, uint64_t n_gpes, double jd_begin, double jd_end,
                              double reentry_radius, double exit_radius, mzb_sgp4_pj **out);
/* out = {objects, doubles in traj, doubles in time, polynomial order}. */
void mzb_sgp4_pj_sizes(const mzb_sgp4_pj *p, uint64_t out[4]);
/* out = {epoch hi, epoch lo (the TAI Julian date of jd_begin as a normalised
 * pair), maxT (days)}. */
void mzb_sgp4_pj_epoch(const mzb_sgp4_pj *p, double out[3]);
/* Copies the arrays out in mizuba's layout: traj [segments][order + 1][7],
 * traj_offsets [objects][2] (offset in doubles, segments), time, and
 * time_offsets [objects], status [objects] (host or device destinations;
 * the trajectory coefficients are copied straight from device memory). */
int mzb_sgp4_pj_copy(const mzb_sgp4_pj *p, double *traj, uint64_t *traj_offsets, double *time,
                     uint64_t *time_offsets, int32_t *status);
void mzb_sgp4_pj_free(mzb_sgp4_pj *p);
/* Device time of the production (ms): out = {interpolation kernel, layout
 * kernel}.  No counterpart in the reference (a measurement aid). */
void mzb_sgp4_pj_timing(const mzb_sgp4_pj *p, double out[2]);

/* Batched SGP4/SDP4 on the GPU (WGS72, 'a' operation mode): each element
 * set at each of n_times times (minutes from its own epoch).
 * out [n_gpes][n_times][6] = x, y, z [km], vx, vy, vz [km/s] (TEME);
 * err [n_gpes][n_times] = 0 or the propagator's error code (10 for a
 * deep-space resonant orbit more than 270 years from its epoch); a
 * non-finite time returns MZB_INVALID_ARGUMENT.  The GPU form
 * of the propagators make_sgp4_polyjectory evaluates
 * (mizuba/make_sgp4_polyjectory.cpp:194-277).  Arrays are host or device
 * pointers. */
int mzb_sgp4_propagate(const mzb_gpe *gpes, uint64_t n_gpes, const double *tsince, uint64_t n_times, double *out,
                       int32_t *err);

/* Allocation-free step sort.  No counterpart in the reference: it is the
 * Morton sort of one conjunction step (the stage mzb_conjunctions runs after
 * the Morton codes) for callers that cannot allocate device memory where they
 * sort, e.g. hosts that hand all device memory to their own allocator at
 * start-up, or allocation-free hot loops.  Inputs and outputs are device
 * pointers owned by the caller, laid out as one step of mzb_conjunctions'
 * outputs: aabbs float[n_objs + 1][2][4] (row n_objs = the step's global
 * box), mcodes uint64[n_objs]; outputs srt_idx uint32[n_objs],
 * srt_mcodes uint64[n_objs], srt_aabbs float[n_objs + 1][2][4].  stream is a
 * cudaStream_t (NULL = the default stream); the call only enqueues work.
 * The scratch is an 8 MiB array inside the library's device image, held by
 * every GPU that loads the library until exit, so n_objs is limited to
 * 524288 (larger sizes return MZB_INVALID_ARGUMENT).  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress), so it
 * should come before any stream capture.  Calls share the array: calls
 * whose work overlaps on the GPU race on it.  No cudaMalloc, cudaFree or
 * other allocating routine is called. */
int mzb_sort_step_noalloc(const float *aabbs, const uint64_t *mcodes, uint64_t n_objs, uint32_t *srt_idx,
                          uint64_t *srt_mcodes, float *srt_aabbs, void *stream);

#ifdef __cplusplus
}
#endif

#endif
