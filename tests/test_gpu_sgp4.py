"""SGP4 on the GPU (needs a B200).

* mzb_sgp4_propagate against the reference's own SGP4 propagator (compiled in
  place from the reference tree into oracle/_ref) on near-Earth and
  deep-space element sets of the reference's 26,389-object catalogue,
  before, at and after epoch.
* mzb_make_sgp4_polyjectory on the reference's own test element sets, checked
  the way mizuba/test/test_make_sgp4_polyjectory.py:32-330 checks
  make_sgp4_polyjectory: at random times inside every segment against the
  propagator, 1e-8 km and 1e-11 km/s; the ISS case through state_eval.
* The GPU production against the oracle's CPU restatement on a catalogue
  sample: same statuses, the same step ends for nearly every object, and
  there the same states to 1e-8 km and 1e-11 km/s at random times.
* The screening of a GPU-produced catalogue against the oracle, every step.
"""

import numpy as np
import pytest

import oracle
from parity import assert_dense_equal, assert_trees_pairs_equal
from test_sgp4_cpu import CASES, GOLDEN, check_against_propagator, tsince_min

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mzb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if oracle.sgp4_ref_lib() is None:
        pytest.skip("the reference's SGP4 propagator was not built (reference tree absent)")
    import mizuba_b200

    return mizuba_b200


def near_earth(g):
    return ~oracle.sgp4_ref_is_deep_space(g)


def pj_arrays(pj):
    a = pj.arrays
    return {k: a[k] for k in ("traj", "traj_offsets", "time", "time_offsets")}


def test_propagate_matches_reference(mzb):
    cat = GOLDEN["strack_20240705"]
    g = cat[np.sort(np.random.default_rng(1).choice(len(cat), 4000, replace=False))]
    ne = near_earth(g)
    t = np.array([-1440.0, -300.0, -1.0, 0.0, 17.3, 720.0, 1440.0])
    out, err = mzb.sgp4_propagate(g, t)
    ref, rerr = oracle.sgp4_ref(g, t)
    assert np.array_equal(err, rerr)
    ok = err == 0
    assert ok.sum() > 0.9 * ok.size
    # Near-Earth: rounding only.  Deep space: the resonance integration
    # carries the rounding differences of the device's math functions along
    # (about 1e-12 relative over a day for 12-hour orbits).
    okn = ok & ne[:, None]
    assert np.max(np.abs(out - ref)[okn][:, :3]) <= 1e-8
    assert np.max(np.abs(out - ref)[okn][:, 3:]) <= 1e-11
    okd = ok & ~ne[:, None]
    assert np.max(np.abs(out - ref)[okd][:, :3]) <= 1e-7
    assert np.max(np.abs(out - ref)[okd][:, 3:]) <= 1e-10
    print(f"{ne.sum()} near-Earth and {(~ne).sum()} deep-space sets x {len(t)} times: max |dr| "
          f"{np.abs(out - ref)[okn][:, :3].max():.2e} / {np.abs(out - ref)[okd][:, :3].max():.2e} km")


@pytest.mark.parametrize("name", ["single_gpe", "single_gpe_ds", "syncom_gpe", "multi_gpes", "iss_gpes"])
def test_production_reference_cases(mzb, name):
    g = GOLDEN[name]
    jd0, jd1, patol, vatol = CASES[name]
    pj, ids = mzb.make_sgp4_polyjectory(g, jd0, jd1)
    assert np.array_equal(ids, np.unique(g["norad_id"]))
    assert pj.n_objs == len(ids)
    assert np.all(pj.status == 0)
    for k in range(pj.n_objs):
        assert pj[k][1][0] == 0.0
    check_against_propagator(pj_arrays(pj), g, jd0, np.random.default_rng(123), patol, vatol)
    if name == "iss_gpes":
        # test_make_sgp4_polyjectory.py:241-334: 100 random times through the
        # GPU state evaluation, the element set in force chosen by epoch.
        for jb, je in ((2460667.0, 2460684.0), (2460672.0, 2460679.0)):
            pj, _ = mzb.make_sgp4_polyjectory(g, jb, je)
            rng = np.random.default_rng(123)
            ep = (g["epoch_jd1"] - jb) + g["epoch_jd2"]
            for tm in rng.uniform(0, je - jb, 100):
                idx = max(int(np.searchsorted(ep, tm, side="right")) - 1, 0)
                st, e = oracle.sgp4_ref(g[idx:idx + 1], [tsince_min(g[idx], jb, tm)])
                assert e[0, 0] == 0
                s = pj.state_eval(tm)
                assert np.allclose(st[0, 0, :3], s[0, :3], rtol=0, atol=1e-8)
                assert np.allclose(st[0, 0, 3:], s[0, 3:6], rtol=0, atol=1e-11)


def catalogue_sample(n, seed, near_only=False):
    cat = GOLDEN["strack_20240705"]
    g = cat[np.sort(np.random.default_rng(seed).choice(len(cat), n, replace=False))]
    return g[near_earth(g)] if near_only else g


def test_production_matches_oracle(mzb):
    g = catalogue_sample(1500, 11)
    jd = 2460497.0
    pj, _ = mzb.make_sgp4_polyjectory(g, jd, jd + 1.0)
    r = oracle.sgp4_polyjectory(g, jd, jd + 1.0)
    assert np.array_equal(pj.status, r["status"])
    ne = near_earth(g)
    a = pj.arrays
    assert np.allclose([pj.epoch[0], pj.epoch[1]], r["epoch"], rtol=0, atol=0)
    # Same steps (the Keplerian step sizes agree to rounding): the same
    # segment ends for nearly every object; a bisection decided by a
    # rounding-level difference at the error threshold changes a few.
    ns_g, ns_r = a["traj_offsets"][ne, 1], r["traj_offsets"][ne, 1]
    n_same = 0
    for k in np.nonzero(ne)[0]:
        n = int(a["traj_offsets"][k, 1])
        if n == 0 or n != int(r["traj_offsets"][k, 1]):
            continue
        tg = a["time"][int(a["time_offsets"][k]):][:n + 1]
        tr = r["time"][int(r["time_offsets"][k]):][:n + 1]
        n_same += bool(np.max(np.abs(tg - tr)) <= 1e-11)
    assert n_same >= 0.99 * int(np.sum(ns_r > 0)), (n_same, int(np.sum(ns_r > 0)))
    # Where the steps are the same, the two polyjectories agree to the
    # rounding of the propagators (a few segments of every such object, at
    # random times).
    rng = np.random.default_rng(9)
    max_dr = max_dv = 0.0
    for k in np.nonzero(ne)[0][:400]:
        n = int(a["traj_offsets"][k, 1])
        if n == 0 or n != int(r["traj_offsets"][k, 1]):
            continue
        tg = a["time"][int(a["time_offsets"][k]):][:n + 1]
        tr = r["time"][int(r["time_offsets"][k]):][:n + 1]
        if np.max(np.abs(tg - tr)) > 1e-11:
            continue
        cg = a["traj"][int(a["traj_offsets"][k, 0]):][:n * 133].reshape(n, 19, 7)
        cr = r["traj"][int(r["traj_offsets"][k, 0]):][:n * 133].reshape(n, 19, 7)
        for sg in rng.choice(n, min(n, 4), replace=False):
            # The same instant in both (the step starts differ by rounding).
            t_abs = rng.uniform(max(tg[sg], tr[sg]), min(tg[sg + 1], tr[sg + 1]))
            hg, hr = t_abs - tg[sg], t_abs - tr[sg]
            d = np.array([np.polyval(cg[sg, ::-1, v], hg) - np.polyval(cr[sg, ::-1, v], hr) for v in range(6)])
            max_dr = max(max_dr, float(np.abs(d[:3]).max()))
            max_dv = max(max_dv, float(np.abs(d[3:]).max()))
    assert max_dr <= 1e-8 and max_dv <= 1e-11, (max_dr, max_dv)
    # Against the propagator, at the production's own accuracy: positions
    # within its 1e-7 km acceptance threshold (deep space: the reference's
    # 1e-6 km of its deep-space case); velocities, which the error estimate
    # does not bound, within 1e-9 km/s.
    check_against_propagator(pj_arrays(pj), g, jd, np.random.default_rng(5), 1e-7, 1e-9, per_seg=1,
                             deep_atol=(1e-6, 1e-9))
    print(f"{ne.sum()} near-Earth objects: {int(ns_g.sum())} segments; {n_same} with the oracle's step ends "
          f"to 1e-11 d; GPU vs oracle states max |dr| {max_dr:.2e} km, |dv| {max_dv:.2e} km/s")


def test_screening_of_a_produced_catalogue(mzb):
    # 2,500 element sets of the reference's catalogue, produced on the GPU
    # over half a day, screened on the GPU and by the oracle at 5 km: every
    # step bit-exact (boxes, codes, order, trees, pairs) and the same
    # conjunction records.
    g = catalogue_sample(2500, 13)
    jd = 2460497.0
    pj, _ = mzb.make_sgp4_polyjectory(g, jd, jd + 0.5)
    res = mzb.conjunctions(pj, 5.0, 3.0 / 1440.0)
    r = oracle.run(pj, 5.0, 3.0 / 1440.0)
    assert_dense_equal(res, r)
    assert_trees_pairs_equal(res, r)
    assert np.array_equal(res.conjunctions.view(np.uint8), r["conjunctions"].view(np.uint8))
    x = mzb.conjunctions(pj, 5.0, 3.0 / 1440.0, form="mixed")
    assert np.array_equal(x.conjunctions.view(np.uint8), r["conjunctions"].view(np.uint8))
