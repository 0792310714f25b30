"""The mixed form against the oracle and the plain form (needs a B200).

Mixed form: FMA-native FP64 enclosures widened by an a-posteriori rounding
bound, FP32 broad phase, an FMA-native FP64 prefilter of the narrow phase
whose survivors are recomputed with the reference formulation.  Required:
the oracle's conjunction set with |dTCA| <= 1e-6 s and relative dDCA <=
1e-9 (records within 1e-9 of the threshold may appear on one side only) --
in fact the records equal the plain form's bit for bit; boxes that contain
the plain form's boxes; every plain-form pair whose two boxes overlap
present among the mixed pairs (a superset of the true overlaps).
"""

import numpy as np
import pytest

import cases
import oracle
from parity import conj_match

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mzb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mizuba_b200

    return mizuba_b200


def overlap(a, b):
    return np.all((a[..., 1, :] >= b[..., 0, :]) & (a[..., 0, :] <= b[..., 1, :]), axis=-1)


def check_mixed(mzb, pj, thresh, interval, otypes=None):
    p = mzb.conjunctions(pj, thresh, interval, otypes=otypes)
    x = mzb.conjunctions(pj, thresh, interval, otypes=otypes, form="mixed")
    r = oracle.run(pj, thresh, interval, otypes=otypes)
    # boxes contain the plain boxes (no-data objects stay infinite)
    pa, xa = p.aabbs[:, :-1], x.aabbs[:, :-1]
    fin = np.isfinite(pa[:, :, 0, 0])
    assert np.array_equal(fin, np.isfinite(xa[:, :, 0, 0]))
    assert np.all(xa[:, :, 0][fin] <= pa[:, :, 0][fin]) and np.all(xa[:, :, 1][fin] >= pa[:, :, 1][fin])
    # true overlaps of the plain form are among the mixed pairs
    for k in range(p.n_cd_steps):
        bp, bx = p.get_aabb_collisions(k), x.get_aabb_collisions(k)
        if len(bp) == 0:
            continue
        ov = overlap(pa[k, bp["i"]], pa[k, bp["j"]])
        need = set(zip(bp["i"][ov].tolist(), bp["j"][ov].tolist()))
        assert need <= set(zip(bx["i"].tolist(), bx["j"].tolist())), k
        assert np.all(bx["i"] < bx["j"])
    # same conjunctions as the oracle, within tolerance, and the plain form's
    # records bit for bit (the survivors of the prefilter are recomputed with
    # the reference formulation)
    n, border, dt, dd = conj_match(x.conjunctions, r["conjunctions"], thresh)
    assert n + len([b for b in border if b[0] == "oracle-only"]) == len(r["conjunctions"])
    assert np.array_equal(x.conjunctions.view(np.uint8), p.conjunctions.view(np.uint8))
    # The screen drops items whose distance provably stays above the
    # threshold, so root finding runs on a subset of the plain form's items.
    assert x.np_report[0] >= p.np_report[0]
    assert x.np_report[2] <= p.np_report[2] and x.np_report[5] <= p.np_report[5]
    c, sv = x.narrow_split
    assert x.np_report[0] >= c >= sv >= x.np_report[2] and p.narrow_split == (0, 0)
    return p, x, r


@pytest.mark.parametrize("case", [2, 4, 6])
def test_mixed_cd_begin_end(mzb, case):
    pj, _ = cases.cd_begin_end_pj(case)
    _, x, _ = check_mixed(mzb, pj, 1e-6, 2.0 / 3.0)
    c = x.conjunctions
    assert len(c) >= 1 and abs(c["tca"][0] - 1.0) < 1e-12 and abs(c["dca"][0]) < 1e-12


@pytest.mark.parametrize("shift", [0.0, 1.1])
def test_mixed_boundary(mzb, shift):
    _, x, _ = check_mixed(mzb, cases.boundary_incoming_pj(shift), 0.25, 0.03)
    c = x.conjunctions
    assert len(c) == 1 and abs(c["tca"][0] - (0.9 + shift)) < 1e-12 and abs(c["dca"][0] - 0.2) < 1e-12


@pytest.mark.parametrize("seed", [1, 2])
def test_mixed_random_ragged(mzb, seed):
    check_mixed(mzb, cases.random_linear_pj(300, seed=seed, box=20.0, speed=20.0), 1.5, 0.05)


def test_mixed_clusters(mzb):
    check_mixed(mzb, cases.clustered_pj(21), 0.5, 0.05)


def test_mixed_catalogue_c1_full_day(mzb):
    from mizuba_b200 import synth

    pj = synth.workload("c1_1k_1d")
    p, x, r = check_mixed(mzb, pj, 5.0, 3.0 / 1440.0)
    assert len(r["conjunctions"]) > 0


def test_mixed_orders(mzb):
    from mizuba_b200 import synth

    for order in (7, 25):
        pj = synth.build_polyjectory(synth.elements_for("c1_1k_1d")[:120], 0.05, order=order)
        check_mixed(mzb, pj, 50.0, 3.0 / 1440.0)


def test_form_argument(mzb):
    with pytest.raises(ValueError, match="unknown screening form"):
        mzb.conjunctions(cases.planar_circ_pj(), 0.1, 0.1, form="fast")
