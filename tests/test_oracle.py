"""The oracle against the known answers of mizuba's own tests (CPU only).

These pin the CPU restatement before it is trusted as the checker of the
CUDA path.  Each test cites the reference test it restates.
"""

import math

import numpy as np
import pytest

import cases
import oracle
from mizuba_b200.polyjectory import polyjectory


def test_zero_aabbs_exact():
    # mizuba/test/test_conjunctions.py:586-626
    r = oracle.run(cases.zero_aabbs_pj(), np.finfo(float).eps, 0.1)
    a = r["aabbs"]
    one_dn = np.nextafter(np.float32(1), np.float32(-np.inf))
    one_up = np.nextafter(np.float32(1), np.float32(np.inf))
    s3 = np.float32(math.sqrt(3.0))
    assert np.all(a[:, :, 0, :3] == one_dn)
    assert np.all(a[:, :, 1, :3] == one_up)
    assert np.all(a[:, :, 0, 3] == np.nextafter(s3, np.float32(-np.inf)))
    assert np.all(a[:, :, 1, 3] == np.nextafter(s3, np.float32(np.inf)))


def test_no_traj_data_sorted_last():
    # mizuba/test/test_conjunctions.py:628-692
    r = oracle.run(cases.no_traj_data_pj(), 1e-16, 1.0)
    assert np.all(np.isinf(r["aabbs"][1, :10]))
    assert np.all(np.isinf(r["srt_aabbs"][1, -11:-1]))
    assert np.all(r["mcodes"][1, :10] == np.uint64(2**64 - 1))
    assert r["mcodes"][1, -1] == np.uint64(2**64 - 1)
    assert np.all(r["srt_mcodes"][1, -11:] == np.uint64(2**64 - 1))
    # the finite all-ones object sorts before every object without data
    assert r["srt_idx"][1, -11] == 17


def test_bvh_corner_cases():
    # mizuba/test/test_conjunctions.py:694-784
    r = oracle.run(cases.bvh_single_pj(), 1e-16, 1.0)
    assert len(r["bvh"][0]) == 1
    r = oracle.run(cases.bvh_twins_pj(), 1e-16, 1.0)
    t = r["bvh"][0]
    assert len(t) == 1 and t[0]["begin"] == 0 and t[0]["end"] == 2
    assert t[0]["left"] == -1 and t[0]["right"] == -1
    r = oracle.run(cases.bvh_lastbit_pj(), 1e-16, 1.0)
    assert r["mcodes"][0, -2] == np.uint64(2**64 - 1)
    assert r["mcodes"][0, -1] == np.uint64(2**64 - 2)
    assert r["srt_idx"][0, -1] == 7 and r["srt_idx"][0, -2] == 8


@pytest.mark.parametrize("case", [1, 2, 3, 4, 5, 6])
def test_cd_begin_end(case):
    # mizuba/test/test_conjunctions.py:1071-1324
    pj, expected = cases.cd_begin_end_pj(case)
    c = oracle.run(pj, 1e-6, 2.0 / 3.0)["conjunctions"]
    if expected == 0:
        assert len(c) == 0
        return
    if expected is None:
        assert len(c) >= 1
    else:
        assert len(c) == expected
    assert np.all(c["i"] == 0) and np.all(c["j"] == 1)
    assert abs(c["tca"][0] - 1.0) < 5e-16
    assert abs(c["dca"][0]) <= 1e-15
    assert np.allclose(c["ri"][0], [0, 0, 0], atol=1e-15, rtol=0)
    assert np.allclose(c["rj"][0], [0, 0, 0], atol=1e-15, rtol=0)
    assert np.allclose(c["vi"][0], [-1, 0, 0], atol=1e-15, rtol=0)
    assert np.allclose(c["vj"][0], [1, 0, 0], atol=1e-15, rtol=0)


@pytest.mark.parametrize("shift", [0.0, 1.1])
def test_boundary_incoming(shift):
    # mizuba/test/test_boundary_conjunctions.py:24-123
    c = oracle.run(cases.boundary_incoming_pj(shift), 0.25, 0.03)["conjunctions"]
    assert len(c) == 1
    assert abs(c["tca"][0] - (0.9 + shift)) < 5e-16
    assert abs(c["dca"][0] - 0.2) < 5e-16
    assert c["i"][0] == 0 and c["j"][0] == 1
    assert np.allclose(c["ri"][0], [0.1, 0, 0], rtol=1e-15, atol=0)
    assert np.allclose(c["rj"][0], [-0.1, 0, 0], rtol=1e-15, atol=0)
    assert np.allclose(c["vi"][0], [-1, 0, 0], rtol=1e-15, atol=0)
    assert np.allclose(c["vj"][0], [1, 0, 0], rtol=1e-15, atol=0)


@pytest.mark.parametrize("shift", [0.0, 1.1])
def test_boundary_outgoing(shift):
    # mizuba/test/test_boundary_conjunctions.py:125-198
    c = oracle.run(cases.boundary_outgoing_pj(shift), 0.25, 0.03)["conjunctions"]
    assert len(c) == 1
    assert abs(c["tca"][0] - shift) < 5e-16
    assert abs(c["dca"][0] - 0.2) < 5e-16
    assert np.allclose(c["vi"][0], [1, 0, 0], rtol=1e-15, atol=0)
    assert np.allclose(c["vj"][0], [-1, 0, 0], rtol=1e-15, atol=0)


@pytest.mark.parametrize("interval", [0.01, 0.1, 0.5, 2.0, 5.0, 7.0])
@pytest.mark.parametrize("shift", [0.0, 1.0])
def test_planar_circular(interval, shift):
    # mizuba/test/test_conjunctions.py:284-406 and :1016-1069
    pj = cases.planar_circ_pj(shift)
    r = oracle.run(pj, 0.1, interval)
    a = r["aabbs"]
    assert r["cd_end_times"][-1] == pj[0][1][-1]
    assert np.array_equal(a[:, 0], a[:, 1])
    assert np.array_equal(a, r["srt_aabbs"])
    fin = np.isfinite(a[:, 0, 0, 0])
    assert np.all(a[fin, 0, 0, 2] >= -0.05001) and np.all(a[fin, 0, 1, 2] <= 0.05001)
    assert np.all(a[fin, 0, 0, 3] >= 1 - 0.05001) and np.all(a[fin, 0, 1, 3] <= 1 + 0.05001)
    assert all(len(b) == 0 for b in r["bp"])
    assert len(r["conjunctions"]) == 0
    # positions at random times lie strictly inside the boxes
    rng = np.random.default_rng(42)
    tr, tm, _ = pj[0]
    for k, te in enumerate(r["cd_end_times"]):
        tb = 0.0 if k == 0 else r["cd_end_times"][k - 1]
        if not fin[k]:
            assert tm[-1] <= tb or tm[0] >= te
            continue
        for t in rng.uniform(tb, te, 5):
            s = np.searchsorted(tm, t, side="right")
            if s == 0 or s == len(tm):
                continue
            h = t - tm[s - 1]
            for ci, bi in zip([0, 1, 2, 6], range(4)):
                v = np.polyval(tr[s - 1][::-1, ci], h)
                assert a[k, 0, 0, bi] < v < a[k, 0, 1, bi]


def test_argument_errors():
    # mizuba/test/test_conjunctions.py:175-216, :371-398
    pj = cases.planar_circ_pj()
    with pytest.raises(ValueError, match="The conjunction threshold must be finite and positive"):
        oracle.run(pj, 0.0, 0.1)
    with pytest.raises(ValueError, match="is too large and results in an overflow error"):
        oracle.run(pj, float(np.finfo(float).max), 0.1)
    with pytest.raises(ValueError, match="The conjunction detection interval must be finite and positive"):
        oracle.run(pj, 1.0, float("nan"))
    with pytest.raises(ValueError, match=r"must be one of \[1, 2, 4\], but a value of -5"):
        oracle.run(pj, 0.1, 0.1, otypes=[-5])


def test_empty_trajectories():
    # mizuba/test/test_conjunctions.py:974-1014
    tr, tm = cases.planar_circ_arrays()
    empty = np.zeros((0,) + tr.shape[1:])
    for layout in ([tr, empty], [empty, tr, empty], [empty, empty, tr]):
        times = [tm if x is tr else [] for x in layout]
        pj = polyjectory(layout, times, [0] * len(layout))
        assert len(oracle.run(pj, 1.0, 0.1)["conjunctions"]) == 0


def test_morton_interleave_matches_reference_encoder():
    # Pins the oracle's bit layout against mizuba's own encoder header
    # (mizuba/detail/mortonND_LUT.h), compiled in place when available.
    rng = np.random.default_rng(7)
    f = rng.integers(0, 2**16, size=(2000, 4), dtype=np.uint64)
    f[:4] = [[65535] * 4, [0] * 4, [1, 0, 0, 0], [0, 0, 0, 1]]
    ref = oracle.morton_ref(f)
    if ref is None:
        pytest.skip("reference tree not mounted: oracle/_ref/morton_ref not built")
    mine = np.zeros(len(f), dtype=np.uint64)
    for k in range(16):
        for d in range(4):
            mine |= ((f[:, d] >> np.uint64(k)) & np.uint64(1)) << np.uint64(4 * k + d)
    assert np.array_equal(ref, mine)


def test_otype_masking_properties():
    # Pairs respect i < j and the otype filter (broad_phase.cpp:294-310).
    pj = cases.random_linear_pj(60, seed=3)
    r_all = oracle.run(pj, 2.0, 0.25)
    rng = np.random.default_rng(1)
    ot = rng.choice([1, 2, 4], size=60)
    r_m = oracle.run(pj, 2.0, 0.25, otypes=ot)
    for b_all, b_m in zip(r_all["bp"], r_m["bp"]):
        assert np.all(b_all["i"] < b_all["j"])
        keep = (ot[b_all["i"]] + ot[b_all["j"]]) <= 3
        assert np.array_equal(b_all[keep], b_m)
    # all secondaries/masked -> no broad or narrow phase at all
    r_none = oracle.run(pj, 2.0, 0.25, otypes=[2] * 60)
    assert all(len(b) == 0 for b in r_none["bp"]) and len(r_none["conjunctions"]) == 0


def test_planar_circular_interval_past_max_time():
    # mizuba/test/test_conjunctions.py:400-404: an interval longer than the
    # trajectory gives one step ending at the last time point.
    pj = cases.planar_circ_pj()
    r = oracle.run(pj, 0.1, 42.0)
    assert r["n_cd_steps"] == 1 and r["cd_end_times"][0] == pj[0][1][-1]


@pytest.mark.parametrize("make", [lambda: cases.random_linear_pj(300, seed=2, box=20.0, speed=20.0),
                                  lambda: cases.clustered_pj(21), lambda: cases.no_traj_data_pj()])
def test_debug_verifiers_accept_oracle_outputs(make):
    # The restated debug verifiers of the reference hold on the oracle's own
    # outputs (ragged trajectories, multi-object leaves, no-data objects).
    pj = make()
    r = oracle.run(pj, 1.5 if pj.n_objs > 50 else 1e-16, 0.05 if pj.n_objs > 50 else 1.0)
    for k in range(r["n_run"]):
        oracle.validate_global_aabbs(r["aabbs"][k])
        oracle.verify_bvh_tree(r["srt_mcodes"][k], r["srt_aabbs"][k], r["bvh"][k])
        n_true = oracle.verify_broad_phase(r["aabbs"][k], r["bp"][k])
        assert n_true <= len(r["bp"][k])


def test_debug_verifiers_catch_planted_mistakes():
    # Mistakes planted in oracle outputs on the CPU: a missing pair, a wrong
    # node box, swapped children ranges, a moved global box.
    pj = cases.random_linear_pj(300, seed=3, box=20.0, speed=20.0)
    r = oracle.run(pj, 1.5, 0.05)
    k = next(k for k in range(r["n_run"]) if len(r["bp"][k]) > 3)
    with pytest.raises(AssertionError, match="not in the pair list"):
        oracle.verify_broad_phase(r["aabbs"][k], np.delete(r["bp"][k], 1))
    with pytest.raises(AssertionError, match="strictly increasing"):
        oracle.verify_broad_phase(r["aabbs"][k], r["bp"][k][::-1].copy())
    t = r["bvh"][k].copy()
    t[2]["ub"][1] += 1.0
    with pytest.raises(AssertionError, match="min/max"):
        oracle.verify_bvh_tree(r["srt_mcodes"][k], r["srt_aabbs"][k], t)
    t = r["bvh"][k].copy()
    t[0]["left"], t[0]["right"] = t[0]["right"], t[0]["left"]
    with pytest.raises(AssertionError):
        oracle.verify_bvh_tree(r["srt_mcodes"][k], r["srt_aabbs"][k], t)
    a = r["aabbs"][k].copy()
    a[-1, 0, 0] -= 1.0
    with pytest.raises(AssertionError, match="global box"):
        oracle.validate_global_aabbs(a)
