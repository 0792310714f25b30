"""The CUDA path against the oracle (needs a B200).

Bit-exact: AABBs, Morton codes, sort order, gathered boxes and codes, BVH
trees and broad-phase pair lists.  Conjunctions: identical sets with
|dTCA| <= 1e-6 s and relative dDCA <= 1e-9 (tests/parity.py); every case
here in fact reproduces the oracle's records bit for bit as well.
"""

import math

import numpy as np
import pytest

import cases
import oracle
from parity import assert_dense_equal, assert_trees_pairs_equal, conj_match

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mzb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mizuba_b200

    return mizuba_b200


def full_compare(mzb, pj, thresh, interval, otypes=None, **kw):
    g = mzb.conjunctions(pj, thresh, interval, otypes=otypes, **kw)
    r = oracle.run(pj, thresh, interval, otypes=otypes)
    assert g.n_cd_steps == r["n_cd_steps"]
    assert_dense_equal(g, r)
    assert_trees_pairs_equal(g, r)
    gc, rc = g.conjunctions, r["conjunctions"]
    conj_match(gc, rc, thresh)
    assert g.np_report == r["np_report"]
    return g, r


def test_zero_aabbs(mzb):
    g, _ = full_compare(mzb, cases.zero_aabbs_pj(), np.finfo(float).eps, 0.1)
    a = g.aabbs
    assert np.all(a[:, :, 0, :3] == np.nextafter(np.float32(1), np.float32(-np.inf)))
    assert np.all(a[:, :, 1, 3] == np.nextafter(np.float32(math.sqrt(3.0)), np.float32(np.inf)))


def test_no_traj_data(mzb):
    g, _ = full_compare(mzb, cases.no_traj_data_pj(), 1e-16, 1.0)
    assert np.all(g.mcodes[1, :10] == np.uint64(2**64 - 1))
    assert np.all(np.isinf(g.srt_aabbs[1, -11:-1]))
    assert g.srt_idx[1, -11] == 17


def test_bvh_cases(mzb):
    g, _ = full_compare(mzb, cases.bvh_single_pj(), 1e-16, 1.0)
    assert len(g.get_bvh_tree(0)) == 1
    with pytest.raises(IndexError, match="Cannot fetch the BVH tree for the conjunction timestep at index 1"):
        g.get_bvh_tree(1)
    g, _ = full_compare(mzb, cases.bvh_twins_pj(), 1e-16, 1.0)
    t = g.get_bvh_tree(0)
    assert len(t) == 1 and t[0]["end"] == 2 and t[0]["left"] == -1
    g, _ = full_compare(mzb, cases.bvh_lastbit_pj(), 1e-16, 1.0)
    assert g.mcodes[0, -2] == np.uint64(2**64 - 1) and g.mcodes[0, -1] == np.uint64(2**64 - 2)
    assert g.srt_idx[0, -1] == 7 and g.srt_idx[0, -2] == 8


@pytest.mark.parametrize("case", [1, 2, 3, 4, 5, 6])
def test_cd_begin_end(mzb, case):
    pj, expected = cases.cd_begin_end_pj(case)
    g, _ = full_compare(mzb, pj, 1e-6, 2.0 / 3.0)
    c = g.conjunctions
    if expected == 0:
        assert len(c) == 0
    else:
        assert len(c) >= 1
        assert abs(c["tca"][0] - 1.0) < 5e-16 and abs(c["dca"][0]) <= 1e-15


@pytest.mark.parametrize("shift", [0.0, 1.1])
def test_boundary(mzb, shift):
    g, _ = full_compare(mzb, cases.boundary_incoming_pj(shift), 0.25, 0.03)
    c = g.conjunctions
    assert len(c) == 1 and abs(c["tca"][0] - (0.9 + shift)) < 5e-16 and abs(c["dca"][0] - 0.2) < 5e-16
    g, _ = full_compare(mzb, cases.boundary_outgoing_pj(shift), 0.25, 0.03)
    c = g.conjunctions
    assert len(c) == 1 and abs(c["tca"][0] - shift) < 5e-16


@pytest.mark.parametrize("interval", [0.01, 0.5, 7.0])
def test_planar_circular(mzb, interval):
    g, _ = full_compare(mzb, cases.planar_circ_pj(), 0.1, interval)
    assert len(g.conjunctions) == 0


def test_argument_errors(mzb):
    pj = cases.planar_circ_pj()
    with pytest.raises(ValueError, match="The conjunction threshold must be finite and positive"):
        mzb.conjunctions(pj, 0.0, 0.1)
    with pytest.raises(ValueError, match="is too large and results in an overflow error"):
        mzb.conjunctions(pj, float(np.finfo(float).max), 0.1)
    with pytest.raises(ValueError, match="The conjunction detection interval must be finite and positive"):
        mzb.conjunctions(pj, 1.0, float("nan"))
    with pytest.raises(ValueError, match="expected size is 1, but the actual size is 0"):
        mzb.conjunctions(pj, 0.1, 0.1, otypes=[])
    with pytest.raises(ValueError, match=r"one of \[1, 2, 4\], but a value of 5"):
        mzb.conjunctions(pj, 0.1, 0.1, otypes=[5])
    with pytest.raises(ValueError, match="cannot be provided at the same time"):
        mzb.conjunctions(pj, 0.1, 0.1, data_dir="", tmpdir="")


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_random_ragged(mzb, seed):
    pj = cases.random_linear_pj(300, seed=seed, box=20.0, speed=20.0)
    full_compare(mzb, pj, 1.5, 0.05)


def test_otypes(mzb):
    pj = cases.random_linear_pj(200, seed=9, box=10.0, speed=20.0)
    ot = np.random.default_rng(3).choice([1, 2, 4], size=200)
    full_compare(mzb, pj, 1.5, 0.05, otypes=ot)
    g = mzb.conjunctions(pj, 1.5, 0.05, otypes=[2] * 200)
    assert all(len(g.get_aabb_collisions(k)) == 0 for k in range(g.n_cd_steps))
    assert len(g.conjunctions) == 0


@pytest.mark.parametrize("seed", [21, 22])
def test_clusters_and_multi_object_leaves(mzb, seed):
    pj = cases.clustered_pj(seed)
    g, r = full_compare(mzb, pj, 0.5, 0.05)
    # the case really exercises multi-object leaves and long partner lists
    t = g.get_bvh_tree(0)
    leaves = t[t["left"] == -1]
    assert np.any(leaves["end"] - leaves["begin"] > 1)
    b = g.get_aabb_collisions(0)
    assert np.bincount(b["i"]).max() > 4


def test_batching_invariance(mzb):
    pj = cases.random_linear_pj(150, seed=5, box=10.0, speed=20.0)
    a = mzb.conjunctions(pj, 1.0, 0.03, steps_per_batch=7)
    b = mzb.conjunctions(pj, 1.0, 0.03)
    for key in ("aabbs", "srt_idx", "srt_mcodes"):
        assert np.array_equal(getattr(a, key), getattr(b, key))
    assert np.array_equal(a.conjunctions.view(np.uint8), b.conjunctions.view(np.uint8))
    for k in range(a.n_cd_steps):
        assert np.array_equal(a.get_aabb_collisions(k), b.get_aabb_collisions(k))


def test_step_range_shard(mzb):
    # A shard of the time axis equals the matching slice of the full screen.
    pj = cases.random_linear_pj(150, seed=8, box=10.0, speed=20.0)
    full = mzb.conjunctions(pj, 1.0, 0.03)
    b, e = 11, 23
    part = mzb.conjunctions(pj, 1.0, 0.03, step_range=(b, e))
    assert part.n_cd_steps == full.n_cd_steps and part.step_begin == b
    for key in ("aabbs", "srt_aabbs", "mcodes", "srt_mcodes", "srt_idx", "cd_end_times"):
        assert np.array_equal(getattr(part, key), getattr(full, key)[b:e]), key
    for k in range(e - b):
        assert np.array_equal(part.get_bvh_tree(k), full.get_bvh_tree(b + k))
        assert np.array_equal(part.get_aabb_collisions(k), full.get_aabb_collisions(b + k))
    fc = full.conjunctions
    sel = (fc["tca"] >= full.cd_end_times[b - 1]) & (fc["tca"] < full.cd_end_times[e - 1])
    assert np.array_equal(part.conjunctions.view(np.uint8), fc[sel].view(np.uint8))


@pytest.mark.parametrize("order", [2, 7, 18, 25, 32])
def test_orders(mzb, order):
    from mizuba_b200 import synth

    pj = synth.build_polyjectory(synth.elements_for("c1_1k_1d")[:120], 0.05, order=order)
    full_compare(mzb, pj, 50.0, 3.0 / 1440.0)


@pytest.mark.parametrize("name,n,days,thresh", [
    # dense shells (72 planes x N slots) mixed into the base catalogue
    ("c3_20k_shells_1d", 2500, 0.25, 10.0),
    # low-perigee, high-drag objects: segment counts spread over 100x, some
    # trajectories ending early (decay)
    ("c4_30k_7d", 2500, 0.5, 5.0),
    # dense shells with a 20 km threshold (many candidate pairs)
    ("c5_60k_shells_3d", 2500, 0.25, 20.0),
])
def test_catalogue_configs(mzb, name, n, days, thresh):
    from mizuba_b200 import synth

    el = synth.elements_for(name)
    # keep the config's mix: base objects from the front, shells from the back
    w = synth.WORKLOADS[name]
    if w["shells"]:
        k = int(round(n * w["shells"] / w["n"]))
        el = np.concatenate([el[: n - k], el[w["n"] - k:]])
    else:
        el = el[:n]
    pj = synth.build_polyjectory(el, days)
    g, r = full_compare(mzb, pj, thresh, 3.0 / 1440.0)
    assert np.array_equal(g.conjunctions.view(np.uint8), r["conjunctions"].view(np.uint8))
    x = mzb.conjunctions(pj, thresh, 3.0 / 1440.0, form="mixed")
    assert np.array_equal(x.conjunctions.view(np.uint8), r["conjunctions"].view(np.uint8))


def test_catalogue_c1_full_day(mzb):
    # 1,000 objects, 1 day, 3 min, 5 km: every step against the oracle.
    from mizuba_b200 import synth

    pj = synth.workload("c1_1k_1d")
    g, r = full_compare(mzb, pj, 5.0, 3.0 / 1440.0)
    assert len(r["conjunctions"]) > 0
    assert np.array_equal(g.conjunctions.view(np.uint8), r["conjunctions"].view(np.uint8))


def test_catalogue_c2_properties(mzb):
    # 20,000 objects, full day on the GPU; the first 12 steps against the
    # oracle, the rest through size-independent properties.
    from mizuba_b200 import synth

    pj = synth.workload("c2_20k_1d")
    thresh = 5.0
    g = mzb.conjunctions(pj, thresh, 3.0 / 1440.0)
    r = oracle.run(pj, thresh, 3.0 / 1440.0, step_begin=0, step_end=12)
    assert_dense_equal(g, r)
    assert_trees_pairs_equal(g, r)
    S, N = g.n_cd_steps, pj.n_objs
    sm = g.srt_mcodes
    assert np.all(sm[:, 1:] >= sm[:, :-1])
    idx = g.srt_idx.astype(np.int64)
    assert np.all(np.sort(idx, axis=1) == np.arange(N))
    assert np.array_equal(np.take_along_axis(g.mcodes, idx, axis=1), sm)
    for k in range(0, S, 37):
        t = g.get_bvh_tree(k)
        leaves = t[t["left"] == -1]
        assert int((leaves["end"] - leaves["begin"]).sum()) == int(t[0]["end"])
        b = g.get_aabb_collisions(k)
        assert np.all(b["i"] < b["j"])
        key = b["i"].astype(np.uint64) << np.uint64(32) | b["j"].astype(np.uint64)
        assert np.all(key[1:] > key[:-1])
    c = g.conjunctions
    d = np.linalg.norm(c["ri"] - c["rj"], axis=1)
    assert np.allclose(c["dca"], d, rtol=1e-14, atol=0)
    assert np.all(c["dca"] < thresh)
    ends = g.cd_end_times
    step_of = np.searchsorted(ends, c["tca"], side="right")
    assert np.all(np.diff(step_of) >= 0)
    # conjunctions of the oracle's steps match
    sub = c[c["tca"] < ends[11]]
    conj_match(sub, r["conjunctions"], thresh)


def test_sort_block_size(mzb):
    # The 256-thread sort gives the reference order (ties by index included).
    full_compare(mzb, cases.clustered_pj(3), 0.5, 0.05, tuning={"sort_threads": 256})
    full_compare(mzb, cases.random_linear_pj(500, seed=21), 1.0, 0.05, tuning={"sort_threads": 256})
    with pytest.raises(ValueError, match="unsupported sort block size"):
        mzb.conjunctions(cases.clustered_pj(3), 0.5, 0.05, tuning={"sort_threads": 128})


@pytest.mark.parametrize("threads", [256, 512, 1024])
def test_bvh_block_sizes(mzb, threads):
    # Every CTA size the autotuner may pick builds the reference's trees.
    pj = cases.clustered_pj(4)
    full_compare(mzb, pj, 0.5, 0.05, tuning={"bvh_threads": threads})
    with pytest.raises(ValueError, match="unsupported BVH block size"):
        mzb.conjunctions(pj, 0.5, 0.05, tuning={"bvh_threads": 300})


@pytest.mark.parametrize("n", [30000, 40000])
def test_large_step_bvh(mzb, n):
    # Past 27,648 objects the one-pass BVH build searches the codes in global
    # memory; past 36,864 its depth arrays live there too.
    pj = cases.random_linear_pj(n, seed=n, span=0.02, nseg_max=2, box=1000.0, speed=50.0)
    full_compare(mzb, pj, 1.0, 0.01)


def test_autotune_choice(mzb):
    pj = cases.random_linear_pj(400, seed=9, box=20.0, speed=10.0)
    t = mzb.autotune(pj, 1.0, 0.05)
    assert t["bvh_threads"] == 0 and set(t["bvh_ms"]) == {0}
    assert t["broad_walk"] in (0, 1) and set(t["broad_ms"]) == {0, 1}
    assert t["sort_threads"] in (256, 512) and set(t["sort_ms"]) == {256, 512}
    full_compare(mzb, pj, 1.0, 0.05, tuning=t)


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("make", [lambda: cases.clustered_pj(8), lambda: cases.random_linear_pj(350, seed=4)])
def test_alternative_broad_walks(mzb, make, walk):
    # The default walk takes one position per thread; the warp-coherent walk
    # and the walk that refills lanes with new positions must give the same
    # (reference) pairs.
    full_compare(mzb, make(), 0.5, 0.05, tuning={"broad_walk": walk})
    with pytest.raises(ValueError, match="unsupported broad-phase walk"):
        mzb.conjunctions(make(), 0.5, 0.05, tuning={"broad_walk": 3})


@pytest.mark.parametrize("n", [250, 450])
def test_dense_clump_partner_lists(mzb, n):
    # Every box overlaps every other: objects have up to n - 1 partners.  At
    # 250 objects the partners beyond the staged four fit the spill list and
    # are scattered and sorted; at 450 they overflow it and the overflowing
    # objects are walked again in full.  Both must give the reference lists.
    pj = cases.random_linear_pj(n, seed=n, span=0.05, nseg_max=2, box=1.0, speed=0.5)
    full_compare(mzb, pj, 3.0, 0.05)
