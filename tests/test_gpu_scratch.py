"""Batch scratch cached between screening calls: repeated calls of either
form reuse it (no growth once the largest call has run), results stay those
of the oracle, and the cache can be handed back to the pool."""

import numpy as np
import pytest

import cases
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mzb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mizuba_b200

    return mizuba_b200


def _same(a, b):
    assert np.array_equal(a.srt_idx, b.srt_idx)
    assert np.array_equal(a.conjunctions.view(np.uint8), b.conjunctions.view(np.uint8))
    for k in range(a.n_cd_steps):
        assert np.array_equal(a.get_bvh_tree(k).view(np.uint8), b.get_bvh_tree(k).view(np.uint8))
        assert np.array_equal(a.get_aabb_collisions(k), b.get_aabb_collisions(k))


def test_scratch_reuse_across_forms(mzb):
    # The mixed form's boxes contain the plain form's, so trees, pairs and
    # narrow-phase counters differ between the forms; each form is checked
    # against its own first call (and the plain form against the oracle),
    # the conjunctions against each other.
    pj = cases.random_linear_pj(600, seed=17, box=15.0, speed=8.0)
    r = oracle.run(pj, 1.0, 0.05)
    # The cache is per device and process: start from an empty one, since
    # earlier calls (other tests) may have sized it for larger inputs.
    mzb.release_scratch()
    assert mzb.scratch_bytes() == 0
    first = {"mixed": mzb.conjunctions(pj, 1.0, 0.05, form="mixed")}
    assert mzb.scratch_bytes() > 0
    first["plain"] = mzb.conjunctions(pj, 1.0, 0.05, form="plain")
    # Once each form has run (the plain form keeps an item queue, the mixed
    # form screens items as it finds them), later calls of either form
    # allocate nothing: the cache does not grow.
    held = mzb.scratch_bytes()
    seq = [(f, mzb.conjunctions(pj, 1.0, 0.05, form=f)) for f in ("mixed", "plain", "mixed", "plain")]
    assert mzb.scratch_bytes() == held
    assert first["plain"].np_report == r["np_report"]
    assert np.array_equal(first["plain"].conjunctions.view(np.uint8), first["mixed"].conjunctions.view(np.uint8))
    for f, g in seq:
        _same(g, first[f])
        assert g.np_report == first[f].np_report
    mzb.release_scratch()
    assert mzb.scratch_bytes() == 0
    again = mzb.conjunctions(pj, 1.0, 0.05, form="mixed")
    _same(again, first["mixed"])
    assert 0 < mzb.scratch_bytes() <= held


def test_concurrent_calls_share_or_bypass_cache(mzb):
    # Two host threads screen at the same time on one device: one holds the
    # device's cached scratch, the other finds it taken and allocates its own
    # buffers.  Both must give the sequential results.
    import threading

    pjs = [cases.random_linear_pj(500, seed=41, box=15.0, speed=8.0), cases.clustered_pj(5)]
    args = [(1.0, 0.05), (0.5, 0.05)]
    seq = [mzb.conjunctions(pj, *a, form="mixed") for pj, a in zip(pjs, args)]
    for _ in range(3):
        got = [None, None]
        errs = []

        def work(k):
            try:
                got[k] = mzb.conjunctions(pjs[k], *args[k], form="mixed")
            except Exception as e:  # reported below
                errs.append(e)

        ts = [threading.Thread(target=work, args=(k,)) for k in range(2)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        assert not errs, errs
        for k in range(2):
            _same(got[k], seq[k])
            assert got[k].np_report == seq[k].np_report
