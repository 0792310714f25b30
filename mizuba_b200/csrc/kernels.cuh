// Kernel launchers shared between the stage files and the host pipeline.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

#include "common.cuh"
#include "mizuba_b200.h"
#include "sgp4pj.cuh"

namespace mzb
{

// A narrow-phase sub-interval whose distance enclosure reaches below the
// threshold: the root-finding stage's unit of work.
struct root_item {
    uint32_t i, j, step, flags; // flags: 1 = end of trajectory data, 2 = start
    double lb_rf, rf_int, di, dj;
    uint64_t seg_i, seg_j;
    double ptd2[MAX_OP1];
};

// One narrow-phase candidate: objects i < j of batch step b over their
// segments it_i - 1 and it_j - 1 (time indices as in step_range).
struct np_item {
    uint32_t i, j, b, it_i, it_j, pad;
};

// A detected conjunction tagged with its step (index within the batch).
struct conj_out {
    conj_rec c;
    uint32_t step;
    uint32_t pad;
};

cudaError_t init_aabb_consts();
cudaError_t measure_dfma_rate(double *per_second);
cudaError_t init_narrow_consts();
cudaError_t init_bvh_attrs();

void launch_state_eval(const dev_pj &pj, const double *tm, uint64_t tm_stride_obj, uint64_t tm_stride_t,
                       const uint64_t *sel, uint64_t n_eval, uint64_t n_t, double *out, cudaStream_t stream);
void launch_relayout(const double *src, double *dst, uint64_t n_seg, int op1, unsigned long long *bad_seg,
                     cudaStream_t stream);
void launch_upload_chunk(const double *src, double *dst, const uint64_t *seg_off, const uint64_t *time_off,
                         const uint32_t *nseg, const double *time, uint64_t n_objs, int op1, double t_lo,
                         double t_hi, bool first, bool last, unsigned long long *bad_seg, cudaStream_t stream);
// A run of the staged upload: n_seg consecutive segments starting at global
// segment dst_seg, stored from segment src_seg of the piece's data.
struct stage_run {
    uint64_t dst_seg;
    uint32_t n_seg, src_seg;
};
static_assert(sizeof(stage_run) == 16, "stage_run layout");
void launch_relayout_runs(const char *piece, uint64_t n_runs, double *coef, int op1, unsigned long long *bad_seg,
                          cudaStream_t stream);
void launch_aabb(const dev_pj &pj, const double2 *cdb, const double *inv_binom, uint32_t s_first, uint32_t nb,
                 double radius, float *aabbs, uint2 *more, unsigned long long *more_count, float4 *scr,
                 uint2 *srange, dev_status *st, cudaStream_t stream);
void launch_morton(const float *aabbs, uint32_t s_first, uint32_t nb, uint64_t N, uint64_t *mcodes,
                   cudaStream_t stream);
void launch_sort(const float *aabbs, const uint64_t *mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                 uint64_t *keys_a, uint32_t *vals_a, uint32_t *vals_b, uint32_t *srt_idx,
                 uint64_t *srt_mcodes, float *srt_aabbs, int threads, cudaStream_t stream);
cudaError_t sort_step_noalloc(const float *aabbs, const uint64_t *mcodes, uint64_t n_objs, uint32_t *srt_idx,
                              uint64_t *srt_mcodes, float *srt_aabbs, cudaStream_t stream);
uint64_t sort_noalloc_max_objs();
void launch_bvh(const float *srt_aabbs, const uint64_t *srt_mcodes, uint32_t s_first, uint32_t nb, uint64_t N,
                bvh_node *trees, uint64_t cap, int32_t *ropes, uint32_t *aux, uint32_t *leaf_of, uint32_t *tree_size,
                walk_node *walks, dev_status *st, int threads, cudaStream_t stream);
uint64_t bvh_aux_words(uint64_t N, uint64_t cap);
void launch_tree_gather(const bvh_node *trees, uint64_t cap, const uint64_t *offs, const uint32_t *sizes,
                        uint64_t n_steps, bvh_node *out, cudaStream_t stream);
constexpr int BROAD_STAGE_K = 4; // partners staged per object by the half traversal
void launch_broad_half(const float *srt_aabbs, const bvh_node *trees, uint64_t cap, const int32_t *ropes,
                       const walk_node *walks, const uint32_t *leaf_of, const uint32_t *srt_idx,
                       const uint32_t *tree_size, const int32_t *otypes, uint32_t s_first, uint32_t nb, uint64_t N,
                       uint32_t *counts, uint32_t *stage, ulonglong2 *spill, uint64_t spill_cap,
                       unsigned long long *spill_count, unsigned long long *walk_next, int walk,
                       unsigned long long *visits, cudaStream_t stream);
void launch_broad_copy(const float *aabbs, const bvh_node *trees, uint64_t cap, const int32_t *ropes,
                       const uint32_t *srt_idx, const int32_t *otypes, uint32_t s_first, uint32_t nb, uint64_t N,
                       uint32_t *counts, const uint64_t *offs, const uint32_t *stage, uint2 *pairs,
                       uint64_t *overflow, unsigned long long *overflow_count, const ulonglong2 *spill,
                       const unsigned long long *spill_count, bool spilled_ok, cudaStream_t stream);
void launch_scan(const uint32_t *counts, uint64_t n, uint64_t *offs, uint64_t *block_sums, uint64_t *total,
                 cudaStream_t stream);
void launch_step_offsets(const uint64_t *offs, uint64_t N, uint32_t nb, const uint64_t *total, uint64_t *step_off,
                         cudaStream_t stream);
void launch_items(const dev_pj &pj, const double2 *cdb, uint32_t s_first, uint32_t nb, const uint2 *pairs,
                  const uint64_t *step_off, const uint2 *srange, uint64_t n_pairs, np_item *items, uint64_t cap,
                  unsigned long long *item_count, unsigned long long *counters, dev_status *st, cudaStream_t stream);
void launch_narrow(const dev_pj &pj, const double2 *cdb, uint32_t s_first, const np_item *items,
                   const unsigned long long *item_count, uint64_t item_cap, double thresh2, root_item *rq,
                   uint64_t rq_cap, unsigned long long *rq_count, unsigned long long *counters, dev_status *st,
                   unsigned grid, cudaStream_t stream);
void launch_items_screen(const dev_pj &pj, const double2 *cdb, uint32_t s_first, uint32_t nb, const uint2 *pairs,
                         const uint64_t *step_off, const uint2 *srange, uint64_t n_pairs, double thresh,
                         const float4 *scr, np_item *cand, uint64_t cand_cap, unsigned long long *cand_count,
                         unsigned long long *item_count, unsigned long long *counters, dev_status *st,
                         cudaStream_t stream);
void launch_narrow_prefilter(const dev_pj &pj, const double *tab, const double2 *cdb, uint32_t s_first,
                             const np_item *items, const unsigned long long *item_count, uint64_t item_cap,
                             double thresh2, np_item *surv, uint64_t surv_cap, unsigned long long *surv_count,
                             unsigned long long *counters, dev_status *st, unsigned grid, cudaStream_t stream);
constexpr int ROOTS_WL_SMALL = 24;  // working-list entries per thread, first pass
constexpr int ROOTS_WL_FULL = 251;  // the reference's bound (list size > 250 fails)
void launch_roots(const dev_pj &pj, const root_item *rq, const unsigned long long *rq_count, uint64_t rq_cap,
                  const uint32_t *item_list, const unsigned long long *item_list_count, double thresh2,
                  double *wl_scratch, int wl_cap, unsigned grid, uint32_t *retry, unsigned long long *retry_count,
                  conj_out *cq, uint64_t cq_cap, unsigned long long *cq_count, unsigned long long *counters,
                  dev_status *st, cudaStream_t stream);
void launch_conj_sort(const conj_out *cq, uint64_t n, uint32_t nb, uint32_t *cnt, uint32_t *off, uint32_t *cursor,
                      conj_out *grp, conj_rec *out, cudaStream_t stream);

// SGP4 polyjectory production (k_sgp4.cu).
namespace sgp4pj
{
using gpe_host = mzb_gpe;
// The produced polyjectory in mizuba's layout: the trajectory coefficients
// stay on the device until the caller copies them out; times, offsets and
// statuses are on the host.
struct sgp4_pj_out {
    double *d_traj = nullptr;
    uint64_t n_traj = 0;
    std::vector<double> time;
    std::vector<uint64_t> traj_off, time_off;
    std::vector<int32_t> status;
    dfl epoch{};
    double maxT = 0;
    uint64_t n_launches = 0;
    float kernel_ms = 0, gather_ms = 0; // device time of the production and gather kernels
    sgp4_pj_out() = default;
    sgp4_pj_out(const sgp4_pj_out &) = delete;
    sgp4_pj_out &operator=(const sgp4_pj_out &) = delete;
    ~sgp4_pj_out()
    {
        if (d_traj) cudaFree(d_traj);
    }
};
dfl utc_to_tai(dfl utc);
void gpe_check(const gpe_host *g, uint64_t n, double jd_begin, double jd_end, double reentry, double exit_r);
sgp4_pj_out *make_sgp4_pj(const gpe_host *g, uint64_t n, double jd_begin, double jd_end, double reentry,
                          double exit_r);
void free_sgp4_pj(sgp4_pj_out *p);
void sgp4_propagate(const gpe_host *g, uint64_t n, const double *tsince, uint64_t n_t, double *out, int32_t *err);
} // namespace sgp4pj

} // namespace mzb
