"""Comparison helpers: the CUDA path's outputs against the oracle's."""

from __future__ import annotations

import numpy as np

# Conjunction tolerances of the plain FP64 form: |dTCA| <= 1e-6 s (in the
# polyjectory time unit: days for SGP4-style data, so 1e-6 / 86400) and a
# relative DCA difference <= 1e-9.
TCA_TOL_DAYS = 1e-6 / 86400.0
DCA_RTOL = 1e-9


def assert_dense_equal(gpu, ref, s0=0):
    """Bit-exact AABBs, Morton codes, order, gathered arrays and end times
    for steps [s0, s0 + ref['n_run'])."""
    s1 = s0 + ref["n_run"]
    for key in ("aabbs", "srt_aabbs", "mcodes", "srt_mcodes", "srt_idx"):
        g = getattr(gpu, key)[s0:s1]
        r = ref[key]
        assert g.shape == r.shape, key
        assert np.array_equal(g.view(np.uint8), r.view(np.uint8)), key
    assert np.array_equal(gpu.cd_end_times[s0:s1], ref["cd_end_times"])


def assert_trees_pairs_equal(gpu, ref, s0=0):
    for k in range(ref["n_run"]):
        t = gpu.get_bvh_tree(s0 + k)
        assert np.array_equal(t.view(np.uint8), ref["bvh"][k].view(np.uint8)), f"tree step {s0 + k}"
        b = gpu.get_aabb_collisions(s0 + k)
        assert np.array_equal(b.view(np.uint8), ref["bp"][k].view(np.uint8)), f"pairs step {s0 + k}"


def conj_match(g, r, thresh, tca_tol=TCA_TOL_DAYS, dca_rtol=DCA_RTOL):
    """Matches conjunction records by (i, j) and nearest tca.  Records whose
    dca lies within 1e-9 relative of the threshold may appear on one side
    only (listed separately).  Returns (n_matched, borderline, max |dTCA|,
    max relative dDCA)."""
    border = []
    used = np.zeros(len(g), dtype=bool)
    max_dt = 0.0
    max_dd = 0.0
    by_pair = {}
    for k, rec in enumerate(g):
        by_pair.setdefault((int(rec["i"]), int(rec["j"])), []).append(k)
    for rec in r:
        cand = [k for k in by_pair.get((int(rec["i"]), int(rec["j"])), []) if not used[k]]
        best = None
        for k in cand:
            dt = abs(g[k]["tca"] - rec["tca"])
            if dt <= tca_tol and (best is None or dt < abs(g[best]["tca"] - rec["tca"])):
                best = k
        if best is None:
            if abs(rec["dca"] - thresh) <= 1e-9 * thresh:
                border.append(("oracle-only", rec))
                continue
            raise AssertionError(f"conjunction missing on the GPU: {rec}")
        used[best] = True
        max_dt = max(max_dt, abs(g[best]["tca"] - rec["tca"]))
        dd = abs(g[best]["dca"] - rec["dca"]) / max(abs(rec["dca"]), 1e-300)
        if rec["dca"] != 0 or g[best]["dca"] != 0:
            assert dd <= dca_rtol or abs(g[best]["dca"] - rec["dca"]) <= 1e-15, (rec, g[best])
            max_dd = max(max_dd, dd)
    for k in np.nonzero(~used)[0]:
        if abs(g[k]["dca"] - thresh) <= 1e-9 * thresh:
            border.append(("gpu-only", g[k]))
            continue
        raise AssertionError(f"extra conjunction on the GPU: {g[k]}")
    return int(used.sum()), border, max_dt, max_dd
