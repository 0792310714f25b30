"""SGP4 polyjectory production, CPU side.

* The oracle's restatement of make_sgp4_polyjectory, driven by the
  reference's own SGP4 propagator compiled in place, reproduces that
  propagator at random times inside every segment within the reference's
  own tolerances (1e-8 km and 1e-11 km/s; 1e-7 / 1e-6 km and 1e-10 km/s for
  its deep-space cases): the checks of mizuba/test/
  test_make_sgp4_polyjectory.py:32-330 on the reference's own element sets
  (tests/golden/gpes.npz).
* The C ABI's argument checks and messages (test_make_sgp4_polyjectory.py:
  443-610) run before any device work, so they are tested here.
"""

import numpy as np
import pytest

import oracle

GOLDEN = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "gpes.npz")
JD0 = 2460669.0


def tsince_min(g, jd_begin, tau):
    """Minutes from the element set's epoch of the polyjectory times tau
    (days from jd_begin; no leap second inside these spans)."""
    return (((jd_begin - g["epoch_jd1"]) - g["epoch_jd2"]) + tau) * 1440.0


def check_against_propagator(pj_arrays, gpes, jd_begin, rng, pos_atol=1e-8, vel_atol=1e-11, per_seg=5,
                             deep_atol=None):
    """Every segment of every object with data, at per_seg random times:
    the interpolated state against the reference propagator.  With several
    element sets per object, the set in force is the last one whose epoch is
    at or before the time (the first one before that).  deep_atol: (pos,
    vel) tolerances for deep-space objects, if they differ."""
    toff, tmoff = pj_arrays["traj_offsets"], pj_arrays["time_offsets"]
    ids = np.unique(gpes["norad_id"])
    n_checked = 0
    for k, nid in enumerate(ids):
        ns = int(toff[k, 1])
        if ns == 0:
            continue
        sets = gpes[gpes["norad_id"] == nid]
        patol, vatol = pos_atol, vel_atol
        if deep_atol is not None and oracle.sgp4_ref_is_deep_space(sets[:1])[0]:
            patol, vatol = deep_atol
        cf = pj_arrays["traj"][int(toff[k, 0]):int(toff[k, 0]) + ns * 133].reshape(ns, 19, 7)
        tm = pj_arrays["time"][int(tmoff[k]):int(tmoff[k]) + ns + 1]
        for s in range(ns):
            h = rng.uniform(0, tm[s + 1] - tm[s], per_seg)
            tau = tm[s] + h
            ep = (sets["epoch_jd1"] - jd_begin) + sets["epoch_jd2"]
            which = np.clip(np.searchsorted(ep, tau, side="right") - 1, 0, len(sets) - 1)
            for q in range(per_seg):
                g = sets[which[q]:which[q] + 1]
                st, err = oracle.sgp4_ref(g, [tsince_min(g[0], jd_begin, tau[q])])
                assert err[0, 0] == 0
                vals = np.array([np.polyval(cf[s, ::-1, v], h[q]) for v in range(7)])
                assert np.all(np.abs(vals[:3] - st[0, 0, :3]) <= patol), (nid, s, vals[:3] - st[0, 0, :3])
                assert np.all(np.abs(vals[3:6] - st[0, 0, 3:]) <= vatol), (nid, s, vals[3:6] - st[0, 0, 3:])
                assert abs(vals[6] - np.linalg.norm(st[0, 0, :3])) <= patol
                n_checked += 1
    return n_checked


# The reference's cases (test_make_sgp4_polyjectory.py:69-330): element
# sets, span, tolerances (the deep-space sets have larger ones there too).
CASES = {
    "single_gpe": (2460669.0, 2460670.0, 1e-8, 1e-11),
    "single_gpe_ds": (2460669.0, 2460670.0, 1e-7, 1e-10),
    "syncom_gpe": (2460666.5, 2460676.5, 1e-6, 1e-10),
    "multi_gpes": (2460669.0, 2460670.0, 1e-8, 1e-11),
    "iss_gpes": (2460667.0, 2460684.0, 1e-8, 1e-11),
}


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_production_reproduces_reference_propagator(name):
    if oracle.sgp4_ref_lib() is None:
        pytest.skip("the reference's SGP4 propagator was not built (reference tree absent)")
    g = GOLDEN[name]
    jd0, jd1, patol, vatol = CASES[name]
    r = oracle.sgp4_polyjectory(g, jd0, jd1)
    assert np.all(r["status"] == 0)
    # The trajectories start exactly at the polyjectory epoch.
    assert np.all(r["time"][r["time_offsets"][r["traj_offsets"][:, 1] > 0].astype(np.int64)] == 0.0)
    n = check_against_propagator(r, g, jd0, np.random.default_rng(42), patol, vatol)
    assert n >= 5 * 100


def test_oracle_production_catalogue_sample():
    # 150 element sets of the reference's 26,389-object catalogue, half a
    # day, at the production's own accuracy: positions within its 1e-7 km
    # acceptance threshold (deep space: 1e-6 km, the reference's tolerance
    # for its deep-space case); velocities, which the error estimate does not
    # bound, within 1e-9 km/s.
    if oracle.sgp4_ref_lib() is None:
        pytest.skip("the reference's SGP4 propagator was not built (reference tree absent)")
    cat = GOLDEN["strack_20240705"]
    sel = np.sort(np.random.default_rng(7).choice(len(cat), 150, replace=False))
    g = cat[sel]
    jd = 2460497.0
    r = oracle.sgp4_polyjectory(g, jd, jd + 0.5)
    assert np.mean(r["status"] == 0) > 0.9
    check_against_propagator(r, g, jd, np.random.default_rng(3), 1e-7, 1e-9, per_seg=2, deep_atol=(1e-6, 1e-9))


@pytest.fixture(scope="module")
def L():
    from mizuba_b200 import _native, build

    build.build_cuda()
    return _native.core()


def test_argument_checks(L):
    # mizuba/test/test_make_sgp4_polyjectory.py:443-610: messages of the
    # reference, raised before any device work.
    from mizuba_b200 import make_sgp4_polyjectory

    g = GOLDEN["multi_gpes"].copy()
    with pytest.raises(ValueError, match="Invalid Julian date interval "):
        make_sgp4_polyjectory(g, JD0 + 1, JD0)
    with pytest.raises(ValueError, match="Invalid Julian date interval "):
        make_sgp4_polyjectory(g, float("nan"), JD0)
    with pytest.raises(ValueError, match="Invalid Julian date interval "):
        make_sgp4_polyjectory(g, JD0, float("inf"))
    with pytest.raises(ValueError, match="cannot be NaN"):
        make_sgp4_polyjectory(g, JD0, JD0 + 1, reentry_radius=float("nan"))
    with pytest.raises(ValueError, match=r"The reentry radius \(2\) must be less than the exit radius \(1\)"):
        make_sgp4_polyjectory(g, JD0, JD0 + 1, reentry_radius=2.0, exit_radius=1.0)
    with pytest.raises(ValueError, match="requires a non-empty array of GPEs in input"):
        make_sgp4_polyjectory(g[:0], JD0, JD0 + 1)
    bad = g.copy()
    bad["bstar"][3] = float("inf")
    with pytest.raises(ValueError, match="the 'bstar' of the GPE at index 3 is not finite"):
        make_sgp4_polyjectory(bad, JD0, JD0 + 1)
    bad = g.copy()
    bad["epoch_jd2"][0] = float("nan")
    with pytest.raises(ValueError, match="the 'epoch_jd2' of the GPE at index 0 is not finite"):
        make_sgp4_polyjectory(bad, JD0, JD0 + 1)
    with pytest.raises(ValueError, match="is not sorted correctly"):
        make_sgp4_polyjectory(g[::-1].copy(), JD0, JD0 + 1)
    dup = np.concatenate([g[:1], g[:1]])
    with pytest.raises(ValueError, match="Two GPEs with identical NORAD ID 5 and epoch"):
        make_sgp4_polyjectory(dup, JD0, JD0 + 1)
    with pytest.raises(TypeError, match="must all be floats or ints"):
        make_sgp4_polyjectory(g, "a", JD0 + 1)
    with pytest.raises(TypeError, match="the dtype must be 'gpe_dtype'"):
        make_sgp4_polyjectory(np.zeros(3), JD0, JD0 + 1)
