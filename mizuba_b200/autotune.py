"""Launch-shape autotuning for the screening kernels.

The per-step kernels run one CTA per conjunction step, so the best CTA size
depends on how many steps a batch holds against the 148 SMs: large CTAs
finish each tree sooner, small ones let several steps build at once on an
SM.  ``autotune`` times the candidates on one batch of the caller's own
workload (a full batch, the unit the kernels see) and returns the settings
to pass as ``tuning=`` to ``conjunctions`` / ``device_conjunctions``.  The
choice changes launch shapes only, never results.
"""

from __future__ import annotations

import time

from .conjunctions import device_conjunctions

BVH_CANDIDATES = (256, 512, 1024)


def autotune(pj, conj_thresh, conj_det_interval, form="mixed", step_range=None, repeats=2,
             candidates=BVH_CANDIDATES):
    """Times the BVH build with each CTA size on the conjunction steps
    ``step_range`` (default: the first automatic batch) and returns
    ``{"bvh_threads": best, "bvh_ms": {size: ms}, "step_range": ..., "tune_s": seconds}``."""
    t0 = time.perf_counter()
    if step_range is None:
        probe = device_conjunctions(pj, conj_thresh, conj_det_interval, form=form, step_range=(0, 1))
        n_steps = probe.n_cd_steps
        del probe
        per_step = 160 * pj.n_objs + 4096
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
    return {"bvh_threads": int(choice), "bvh_ms": {int(k): float(v) for k, v in timings.items()},
            "step_range": list(step_range), "tune_s": time.perf_counter() - t0}
