"""Launch-shape autotuning for the screening kernels.

The per-step kernels run one CTA per conjunction step, so the best CTA size
depends on how many steps a batch holds against the 148 SMs: large CTAs
finish each tree sooner, small ones let several steps build at once on an
SM.  The broad phase has walks with the same result: warp-coherent (a warp
of spatial neighbours walks together) and one walk per thread; which is
faster depends on how coherent the neighbours' walks are.  ``autotune``
times the candidates on one batch of the caller's own
workload (a full batch, the unit the kernels see) and returns the settings
to pass as ``tuning=`` to ``conjunctions`` / ``device_conjunctions``.  The
choice changes launch shapes only, never results.
"""

from __future__ import annotations

import time

from .conjunctions import device_conjunctions

# The candidates timed by default are the ones that won on some workload:
# the one-pass BVH build everywhere (the level-by-level builds, selectable
# with bvh_threads 256 / 512 / 1024, lost on every catalogue: 2.3-3.9 ms
# against 1.7 ms on the 20,000-object day); one walk per thread on the
# catalogue days and the warp-coherent walk on the 60,000-object span with
# dense shells at 20 km (66 against 75 ms per batch); the work-refill walk
# (broad_walk 2) lost everywhere and is not timed by default.
BVH_CANDIDATES = (0,)
BROAD_WALKS = (0, 1)  # one position per thread, warp-coherent
SORT_CANDIDATES = (256, 512)


def autotune(pj, conj_thresh, conj_det_interval, form="mixed", step_range=None, repeats=2,
             candidates=BVH_CANDIDATES, walks=BROAD_WALKS):
    """Times the BVH builds in ``candidates`` (0: one pass; 256, 512, 1024:
    level by level with that CTA size), then the broad phase with each walk
    in ``walks``, then the step sort with each CTA size, on the conjunction
    steps ``step_range`` (default: the first automatic batch) and returns ``{"bvh_threads": .., "bvh_ms":
    {build: ms}, "broad_walk": .., "broad_ms": {walk: ms}, "sort_threads": ..,
    "sort_ms": {size: ms}, "step_range": ..., "tune_s": seconds}``."""
    t0 = time.perf_counter()
    if step_range is None:
        probe = device_conjunctions(pj, conj_thresh, conj_det_interval, form=form, step_range=(0, 1))
        n_steps = probe.n_cd_steps
        del probe
        per_step = 248 * pj.n_objs + 4096
        step_range = (0, min(n_steps, max(16, min(1024, (3 << 30) // per_step))))
    step_range = (int(step_range[0]), int(step_range[1]))
    timings = {}
    for c in candidates:
        best = float("inf")
        for _ in range(repeats + 1):  # the first run warms up
            r = device_conjunctions(pj, conj_thresh, conj_det_interval, form=form, step_range=step_range,
                                    tuning={"bvh_threads": c})
            best = min(best, r.stage_ms["bvh"])
            del r
        timings[c] = best
    choice = min(timings, key=timings.get)
    # Broad phase: the warp-coherent walk against one walk per thread.
    walk_candidates = walks
    walks = {}
    for w in walk_candidates:
        best = float("inf")
        for _ in range(repeats + 1):
            r = device_conjunctions(pj, conj_thresh, conj_det_interval, form=form, step_range=step_range,
                                    tuning={"bvh_threads": choice, "broad_walk": w})
            best = min(best, r.stage_ms["broad"])
            del r
        walks[w] = best
    walk = min(walks, key=walks.get)
    # Step sort: 256 against 512 threads per CTA.
    sorts = {}
    for t in SORT_CANDIDATES:
        best = float("inf")
        for _ in range(repeats + 1):
            r = device_conjunctions(pj, conj_thresh, conj_det_interval, form=form, step_range=step_range,
                                    tuning={"bvh_threads": choice, "broad_walk": walk, "sort_threads": t})
            best = min(best, r.stage_ms["morton_sort"])
            del r
        sorts[t] = best
    sort_t = min(sorts, key=sorts.get)
    return {"bvh_threads": int(choice), "bvh_ms": {int(k): float(v) for k, v in timings.items()},
            "broad_walk": int(walk), "broad_ms": {int(k): float(v) for k, v in walks.items()},
            "sort_threads": int(sort_t), "sort_ms": {int(k): float(v) for k, v in sorts.items()},
            "step_range": list(step_range), "tune_s": time.perf_counter() - t0}
