"""The drop-in conjunctions object's data files (mizuba/detect_conjunctions.cpp:92-126,
:466-534; mizuba/conjunctions.cpp:139-247; mizuba/test/test_conjunctions.py:496-583),
written by mzb_result_write_files straight from HBM."""

import gc
import os
import stat

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

FILES = ("aabbs", "srt_aabbs", "mcodes", "srt_mcodes", "vidx", "bvh", "bp", "conjunctions")


@pytest.fixture(scope="module")
def mzb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mizuba_b200

    return mizuba_b200


def test_files_match_device_results(mzb, tmp_path):
    pj = cases.random_linear_pj(300, seed=5, box=20.0, speed=10.0)
    d = mzb.device_conjunctions(pj, 1.0, 0.05)
    data_dir = tmp_path / "data_dir"
    c = mzb.conjunctions(pj, 1.0, 0.05, data_dir=data_dir)
    p = c.data_dir
    assert p == os.path.realpath(data_dir) and os.stat(p).st_mode & 0o777 == 0o700
    assert sorted(os.listdir(p)) == sorted(FILES)
    for nm in FILES:
        assert stat.S_IMODE(os.stat(os.path.join(p, nm)).st_mode) == stat.S_IRUSR
    S, N = c.n_cd_steps, pj.n_objs
    assert os.path.getsize(os.path.join(p, "aabbs")) == S * (N + 1) * 32
    assert os.path.getsize(os.path.join(p, "vidx")) == S * N * 4
    for nm in ("aabbs", "srt_aabbs", "mcodes", "srt_mcodes", "srt_idx", "cd_end_times", "conjunctions"):
        a, b = getattr(c, nm), getattr(d, nm)
        assert not a.flags.writeable
        assert a.tobytes() == b.tobytes(), nm
    for s in range(S):
        assert c.get_bvh_tree(s).tobytes() == d.get_bvh_tree(s).tobytes()
        assert c.get_aabb_collisions(s).tobytes() == d.get_aabb_collisions(s).tobytes()
    assert len(c.conjunctions) > 0 and c.np_report == d.np_report
    c.hint_release()
    assert np.array_equal(c.srt_idx, d.srt_idx)
    # The directory stays while arrays from it live, then goes.
    keep = c.get_aabb_collisions(0)
    del c, a, b
    gc.collect()
    assert os.path.isdir(p)
    del keep
    gc.collect()
    assert not os.path.exists(p)


def test_data_dir_rules(mzb, tmp_path):
    pj = cases.planar_circ_pj()
    d = tmp_path / "exists"
    d.mkdir()
    with pytest.raises(RuntimeError, match="Error while creating the directory"):
        mzb.conjunctions(pj, conj_thresh=0.1, conj_det_interval=0.01, data_dir=d)
    mzb.conjunctions(pj, conj_thresh=0.1, conj_det_interval=0.01, data_dir="")
    t = tmp_path / "tmp"
    t.mkdir()
    c = mzb.conjunctions(pj, conj_thresh=0.1, conj_det_interval=0.01, tmpdir=t)
    assert any(t.iterdir())
    del c
    gc.collect()
    assert not any(t.iterdir())


def test_sentinels_without_pairs_or_conjunctions(mzb, tmp_path):
    # All objects secondaries: no broad-phase pairs and no conjunctions.
    pj = cases.random_linear_pj(50, seed=3)
    c = mzb.conjunctions(pj, 1.0, 0.05, otypes=[2] * 50, data_dir=tmp_path / "d")
    p = c.data_dir
    assert os.path.getsize(os.path.join(p, "bp")) == 8
    with open(os.path.join(p, "bp"), "rb") as f:
        assert f.read() == bytes(8)
    assert os.path.getsize(os.path.join(p, "conjunctions")) == 1
    assert len(c.conjunctions) == 0
    assert all(len(c.get_aabb_collisions(s)) == 0 for s in range(c.n_cd_steps))
