"""The catalogue workloads at their full sizes on the GPU (needs a B200).

* 20,000 objects x 1 day, 5 km (the benchmark's workload) and 20,000 objects
  with 6,000 in dense shells x 1 day, 10 km: every one of the 480 steps
  against the oracle, in both forms (plain: bit-exact boxes, codes, order,
  trees and pairs; both forms: the oracle's conjunction records).
* 30,000 objects x 7 days (3,360 steps, low-perigee objects with short
  segments) at 5 km and 60,000 objects with 15,000 in dense shells x 3 days
  (1,440 steps) at 20 km: the whole span screened in one call of each form;
  48 steps (six blocks of eight spread over the span) against the oracle;
  the mixed form's conjunctions equal the plain form's over the whole span.
* On sampled steps of every workload, the reference's debug verifiers
  (global box, BVH structure and node boxes, N^2 broad-phase superset) run
  on the GPU outputs, and on every step the mixed form's pairs contain
  every plain pair whose boxes overlap.

The dense per-step arrays of the long spans are copied into device tensors
and only the sampled steps come back to the host.
"""

import numpy as np
import pytest

import oracle
from parity import TCA_TOL_DAYS, assert_dense_equal, assert_trees_pairs_equal, conj_match

pytestmark = pytest.mark.gpu

INTERVAL = 3.0 / 1440.0


@pytest.fixture(scope="module")
def mzb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mizuba_b200

    return mizuba_b200


def pair_keys(b):
    return b["i"].astype(np.uint64) << np.uint64(32) | b["j"].astype(np.uint64)


def check_verifiers(res, steps, n_threads=None):
    """The reference's debug checks on the GPU outputs of the given steps
    (``res`` exposes per-step accessors); returns the true box overlaps."""
    n_true = 0
    for k in steps:
        a = res.aabbs_step(k)
        oracle.validate_global_aabbs(a)
        oracle.verify_bvh_tree(res.srt_mcodes_step(k), res.srt_aabbs_step(k), res.get_bvh_tree(k))
        n_true += oracle.verify_broad_phase(a, res.get_aabb_collisions(k), n_threads=n_threads)
    return n_true


class HostSteps:
    """Per-step accessors over a result copied whole to the host."""

    def __init__(self, g):
        self.g = g

    def aabbs_step(self, k):
        return self.g.aabbs[k]

    def srt_aabbs_step(self, k):
        return self.g.srt_aabbs[k]

    def srt_mcodes_step(self, k):
        return self.g.srt_mcodes[k]

    def get_bvh_tree(self, k):
        return self.g.get_bvh_tree(k)

    def get_aabb_collisions(self, k):
        return self.g.get_aabb_collisions(k)


class DeviceSteps:
    """Per-step accessors over a device-resident result: each dense array is
    copied once into a device tensor through the C ABI accessors (which
    take device destinations), and only the requested steps reach the
    host.  Trees and pairs are copied packed, with their offset tables."""

    def __init__(self, g):
        import torch

        self.g = g
        self.L, self.h = g._L, g._h
        self.S, self.N = g._S, g._n
        self.torch = torch
        self._dev = {}

    def _rows(self, fn, dtype, row_shape):
        torch = self.torch
        if fn not in self._dev:
            row = int(np.prod(row_shape)) * np.dtype(dtype).itemsize
            t = torch.empty(self.S * row, dtype=torch.uint8, device="cuda")
            assert getattr(self.L, fn)(self.h, t.data_ptr()) == 0, self.L.mzb_last_error()
            self._dev[fn] = (t, row)
        return self._dev[fn]

    def _step(self, fn, dtype, row_shape, k):
        t, row = self._rows(fn, dtype, row_shape)
        return t[k * row:(k + 1) * row].cpu().numpy().view(dtype).reshape(row_shape)

    def aabbs_step(self, k):
        return self._step("mzb_result_copy_aabbs", np.float32, (self.N + 1, 2, 4), k)

    def srt_aabbs_step(self, k):
        return self._step("mzb_result_copy_srt_aabbs", np.float32, (self.N + 1, 2, 4), k)

    def mcodes_step(self, k):
        return self._step("mzb_result_copy_mcodes", np.uint64, (self.N,), k)

    def srt_mcodes_step(self, k):
        return self._step("mzb_result_copy_srt_mcodes", np.uint64, (self.N,), k)

    def srt_idx_step(self, k):
        return self._step("mzb_result_copy_srt_idx", np.uint32, (self.N,), k)

    def get_bvh_tree(self, k):
        torch = self.torch
        if "trees" not in self._dev:
            os_ = np.empty((self.S, 2), dtype=np.uint64)
            self.L.mzb_result_tree_offsets(self.h, os_.ctypes.data)
            tot = int(os_[:, 1].sum())
            t = torch.empty(max(tot, 1) * 48, dtype=torch.uint8, device="cuda")
            assert self.L.mzb_result_copy_trees(self.h, t.data_ptr()) == 0, self.L.mzb_last_error()
            self._dev["trees"] = (os_, t)
        os_, t = self._dev["trees"]
        o, s = int(os_[k, 0]), int(os_[k, 1])
        return t[o * 48:(o + s) * 48].cpu().numpy().view(oracle.BVH_NODE)

    def get_aabb_collisions(self, k):
        return self.g.get_aabb_collisions(k)  # the packed pair list is small enough for the host


def compare_steps(res, r, s0):
    """Bit-exact comparison of the oracle's steps [s0, s0 + n_run) with a
    DeviceSteps result."""
    for kk in range(r["n_run"]):
        k = s0 + kk
        for key, got in (("aabbs", res.aabbs_step(k)), ("srt_aabbs", res.srt_aabbs_step(k)),
                         ("mcodes", res.mcodes_step(k)), ("srt_mcodes", res.srt_mcodes_step(k)),
                         ("srt_idx", res.srt_idx_step(k))):
            assert np.array_equal(got.view(np.uint8), r[key][kk].view(np.uint8)), (key, k)
        assert np.array_equal(res.get_bvh_tree(k).view(np.uint8), r["bvh"][kk].view(np.uint8)), ("tree", k)
        assert np.array_equal(res.get_aabb_collisions(k).view(np.uint8), r["bp"][kk].view(np.uint8)), ("pairs", k)


def boxes_overlap(a, i, j):
    """The reference's closed-interval overlap test of objects i and j in one
    step's boxes (detect_conjunctions_broad_phase.cpp:269-271)."""
    return np.all(a[i, 1] >= a[j, 0], axis=-1) & np.all(a[i, 0] <= a[j, 1], axis=-1)


def superset_per_step(plain, mixed, steps):
    """Every plain-form pair whose boxes overlap is a mixed-form pair (the
    mixed boxes contain the plain ones).  Plain pairs that come only from a
    multi-object leaf's over-approximation (the leaf's box overlaps, the
    member's box does not) depend on the tree, which differs between the
    forms, and may be absent.  Returns (plain pairs, mixed pairs)."""
    n_p = n_m = 0
    for k in steps:
        pb, mb = plain.get_aabb_collisions(k), mixed.get_aabb_collisions(k)
        p, m = pair_keys(pb), pair_keys(mb)
        miss = ~np.isin(p, m, assume_unique=True)
        if miss.any():
            a = plain.aabbs_step(k)
            i = pb["i"][miss].astype(np.int64)
            j = pb["j"][miss].astype(np.int64)
            assert not np.any(boxes_overlap(a, i, j)), k
        n_p += len(p)
        n_m += len(m)
    return n_p, n_m


def conj_sorted(c):
    return c[np.lexsort((c["tca"], c["j"], c["i"]))]


@pytest.mark.parametrize("name,thresh", [("c2_20k_1d", 5.0), ("c3_20k_shells_1d", 10.0)])
def test_full_day_every_step(mzb, name, thresh):
    from mizuba_b200 import synth

    pj = synth.workload(name)
    r = oracle.run(pj, thresh, INTERVAL)
    assert r["n_run"] == 480
    g = mzb.conjunctions(pj, thresh, INTERVAL)
    assert_dense_equal(g, r)
    assert_trees_pairs_equal(g, r)
    rc = r["conjunctions"]
    assert len(rc) > 0
    assert np.array_equal(g.conjunctions.view(np.uint8), rc.view(np.uint8))
    assert g.np_report == r["np_report"]
    x = mzb.conjunctions(pj, thresh, INTERVAL, form="mixed")
    n_matched, border, max_dt, max_dd = conj_match(x.conjunctions, rc, thresh)
    assert n_matched == len(rc) and not border
    assert max_dt <= TCA_TOL_DAYS
    # Every step: the mixed pairs contain every plain pair whose boxes overlap.
    n_p, n_m = superset_per_step(HostSteps(g), HostSteps(x), range(480))
    assert n_m >= n_p
    # The reference's debug checks on the GPU outputs of sampled steps.
    steps = [0, 97, 239, 381, 479]
    n_true = check_verifiers(HostSteps(g), steps)
    check_verifiers(HostSteps(x), steps)
    print(f"{name}: {len(rc)} conjunctions; pairs plain {n_p}, mixed {n_m} (ratio {n_m / n_p:.6f}); "
          f"true box overlaps on {len(steps)} sampled steps {n_true}; mixed vs oracle max |dTCA| "
          f"{max_dt * 86400:.3e} s, max rel dDCA {max_dd:.3e}")


def blocks(S, n_blocks=6, per=8):
    starts = np.linspace(0, S - per, n_blocks).astype(int)
    return [(int(s), int(s) + per) for s in starts]


@pytest.mark.parametrize("name,thresh", [("c4_30k_7d", 5.0), ("c5_60k_shells_3d", 20.0)])
def test_long_span_sampled_steps(mzb, name, thresh):
    from mizuba_b200 import synth
    from mizuba_b200.conjunctions import device_conjunctions

    pj = synth.workload(name)
    S = int(np.ceil(pj.maxT / INTERVAL))
    g = device_conjunctions(pj, thresh, INTERVAL)
    assert g.n_cd_steps == S
    res = DeviceSteps(g)
    cd_end = g.cd_end_times
    gc = g.conjunctions
    for s0, s1 in blocks(S):
        r = oracle.run(pj, thresh, INTERVAL, step_begin=s0, step_end=s1)
        assert np.array_equal(cd_end[s0:s1], r["cd_end_times"])
        compare_steps(res, r, s0)
        # The block's conjunctions: a screen of the block's steps alone (a
        # record's step is not recoverable from its TCA, which can round to
        # the step's end) equals the oracle's, and is a contiguous slice of
        # the whole span's records, which are concatenated in step order.
        part = device_conjunctions(pj, thresh, INTERVAL, step_range=(s0, s1)).conjunctions
        rc = r["conjunctions"]
        assert np.array_equal(part.view(np.uint8), rc.view(np.uint8)), (s0, s1)
        if len(rc):
            hits = np.nonzero(gc["tca"] == rc["tca"][0])[0]
            assert any(np.array_equal(gc[h:h + len(rc)].view(np.uint8), rc.view(np.uint8)) for h in hits), (s0, s1)
    # The mixed form over the whole span: the plain form's conjunctions, a
    # superset of its pairs on every step.
    x = device_conjunctions(pj, thresh, INTERVAL, form="mixed")
    xc = x.conjunctions
    assert len(xc) == len(gc)
    assert np.array_equal(conj_sorted(xc).view(np.uint8), conj_sorted(gc).view(np.uint8))
    n_p, n_m = superset_per_step(res, DeviceSteps(x), range(S))
    steps = [0, S // 3, S - 1]
    n_true = check_verifiers(res, steps)
    print(f"{name}: {S} steps, {len(gc)} conjunctions; pairs plain {n_p}, mixed {n_m} "
          f"(ratio {n_m / max(n_p, 1):.6f}); true box overlaps on {len(steps)} sampled steps {n_true}")
