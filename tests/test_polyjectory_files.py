"""Polyjectory storage: data directories, persistence, mount, from_datafiles
and detach (mizuba/polyjectory.cpp:70-1040; the behaviour checked by
mizuba/test/test_polyjectory.py:350-722 and :1300-1660).  No GPU needed."""

import gc
import os
import stat
import struct

import numpy as np
import pytest

from mizuba_b200 import polyjectory, set_tmpdir, get_tmpdir

STATE = np.zeros((1, 8, 7))


def _pj(**kw):
    return polyjectory(trajs=[STATE, STATE[1:]], times=[np.array([0.0, 1.0]), np.array([], dtype=float)],
                       status=np.array([0, 0], dtype=np.int32), **kw)


def _datafiles(tmp_path):
    traj = tmp_path / "traj"
    np.full((42,), 0.0).tofile(traj)
    time = tmp_path / "time"
    np.array([0.0, 1.0, 1.1]).tofile(time)
    return traj, time


def test_files_and_descriptor(tmp_path):
    d = tmp_path / "d"
    pj = polyjectory(trajs=[np.full((2, 4, 7), 3.0), np.zeros((0, 4, 7)), np.ones((1, 4, 7))],
                     times=[[0.0, 0.5, 1.0], [], [0.25, 2.0]], status=[1, 2, 3], epoch=10.0, epoch2=1e-20,
                     data_dir=d)
    assert pj.data_dir == d.resolve()
    assert sorted(os.listdir(d)) == ["desc", "status", "time", "time_offsets", "traj", "traj_offsets"]
    for nm in os.listdir(d):
        assert stat.S_IMODE(os.stat(d / nm).st_mode) == stat.S_IRUSR
    raw = (d / "desc").read_bytes()
    assert len(raw) == 48
    version, persist, n, op1, maxT, e1, e2 = struct.unpack("<I?3xQI4xddd", raw)
    assert (version, persist, n, op1, maxT, e1, e2) == (0, False, 3, 4, 2.0, 10.0, 1e-20)
    assert np.array_equal(np.fromfile(d / "traj_offsets", dtype=np.uint64).reshape(3, 2), [[0, 2], [56, 0], [56, 1]])
    assert np.array_equal(np.fromfile(d / "time_offsets", dtype=np.uint64), [0, 3, 3])
    assert np.array_equal(np.fromfile(d / "status", dtype=np.int32), [1, 2, 3])
    assert np.array_equal(np.fromfile(d / "time"), [0.0, 0.5, 1.0, 0.25, 2.0])
    assert pj.epoch == (10.0, 1e-20) and pj.maxT == 2.0 and pj.poly_order == 3 and not pj.persist
    tr, tm, st = pj[0]
    assert tr.shape == (2, 4, 7) and np.all(tr == 3.0) and not tr.flags.writeable and st == 1
    assert pj[1][0].shape == (0, 4, 7) and pj[1][1].shape == (0,)
    pj.hint_release()
    del tr, tm
    pj.detach()
    assert not d.exists()


def test_epoch_normalisation():
    pj = _pj(epoch=1.0, epoch2=2.0**-60)
    assert pj.epoch == (1.0, 2.0**-60)
    pj = _pj(epoch=2.0**-60, epoch2=1.0)
    assert pj.epoch == (1.0, 2.0**-60)


def test_custom_data_dir(tmp_path):
    d = tmp_path / "data_dir"
    d.mkdir()
    with pytest.raises(RuntimeError, match="Error while creating the directory"):
        _pj(data_dir=d)
    d2 = (tmp_path / "data_dir2").resolve()
    pj = _pj(data_dir=d2)
    assert pj.data_dir == d2
    pj.detach()
    assert not d2.exists()
    traj, time = _datafiles(tmp_path)
    d3 = (tmp_path / "data_dir3").resolve()
    pj = polyjectory.from_datafiles(traj_file=traj, time_file=time, order=2,
                                    traj_offsets=np.array([(0, 2)], dtype=polyjectory.traj_offset), status=[1],
                                    data_dir=d3)
    assert pj.data_dir == d3 and not traj.exists()
    assert pj[0][0].shape == (2, 3, 7) and np.array_equal(pj[0][1], [0.0, 1.0, 1.1]) and pj.maxT == 1.1
    pj.detach()
    assert not d3.exists()
    _pj(data_dir="")
    with pytest.raises(ValueError, match="cannot be provided at the same time"):
        _pj(data_dir="", tmpdir="")


def test_persist_and_mount(tmp_path):
    d = (tmp_path / "data_dir").resolve()
    pj = _pj(persist=True, data_dir=d)
    assert pj.persist and d.is_dir()
    pj.detach()
    assert d.is_dir()
    m = polyjectory.mount(d)
    assert np.all(m[0][0] == STATE) and np.all(m[0][1] == [0.0, 1.0])
    assert m[1][0].shape == (0, 8, 7) and m[1][1].shape == (0,)
    m.detach()
    assert d.is_dir()
    tmp = _pj()
    with pytest.raises(ValueError, match=": the data is not persistent"):
        polyjectory.mount(tmp.data_dir)
    with pytest.raises(ValueError, match=r"could not be canonicalised \(does it exist\?\)"):
        polyjectory.mount(tmp_path / "foobar")
    (tmp_path / "afile").write_bytes(b"")
    with pytest.raises(ValueError, match="the path is not a directory"):
        polyjectory.mount(tmp_path / "afile")
    traj, time = _datafiles(tmp_path)
    d2 = (tmp_path / "d2").resolve()
    pj = polyjectory.from_datafiles(traj_file=traj, time_file=time, order=2,
                                    traj_offsets=np.array([(0, 2)], dtype=polyjectory.traj_offset), status=[1],
                                    data_dir=d2, persist=True)
    pj.detach()
    assert d2.is_dir() and polyjectory.mount(d2).maxT == 1.1


def test_detached_throw():
    pj = _pj()
    pj.detach()
    pj.detach()
    assert pj.is_detached
    for attr, args in (("n_objs", None), ("maxT", None), ("epoch", None), ("poly_order", None),
                       ("data_dir", None), ("status", None), ("persist", None), ("__getitem__", (0,)),
                       ("state_eval", (0.0,)), ("state_meval", ([0.0],))):
        with pytest.raises(ValueError, match="Cannot operate on a detached polyjectory"):
            a = getattr(pj, attr)
            a(*args)


def test_dir_removal_keeps_mapping():
    state = np.full((1, 8, 7), 42.0)
    pj = polyjectory(trajs=[state, state[1:]], times=[np.array([0.0, 1.0]), np.array([], dtype=float)],
                     status=np.array([0, 0], dtype=np.int32))
    import shutil

    shutil.rmtree(pj.data_dir)
    assert not pj.data_dir.exists()
    assert np.all(pj[0][0] == state) and np.all(pj[0][1] == [0.0, 1.0])


def test_views_keep_the_directory():
    pj = _pj()
    d = pj.data_dir
    view = pj[0][0]
    pj.detach()
    gc.collect()
    assert d.exists()
    del view
    gc.collect()
    assert not d.exists()


def test_tmpdir(tmp_path):
    t = tmp_path / "t"
    t.mkdir()
    pj = _pj(tmpdir=t)
    assert any(t.iterdir()) and pj.data_dir.name.startswith("mizuba_polyjectory-")
    pj.detach()
    assert not any(t.iterdir())
    orig = get_tmpdir()
    try:
        set_tmpdir(t)
        pj = _pj()
        assert pj.data_dir.parent == t.resolve()
        pj.detach()
    finally:
        set_tmpdir(orig)


def test_from_datafiles_errors(tmp_path):
    traj, time = _datafiles(tmp_path)
    to = np.array([(0, 2)], dtype=polyjectory.traj_offset)

    def err(msg, exc=ValueError, **kw):
        args = dict(traj_file=traj, time_file=time, order=2, traj_offsets=to, status=[1])
        args.update(kw)
        with pytest.raises(exc) as e:
            polyjectory.from_datafiles(**args)
        assert msg in str(e.value), str(e.value)

    err("must have 1 dimension, but the number of dimensions is 2", traj_offsets=np.zeros((1, 1), dtype=to.dtype))
    err("Invalid polynomial order 1 specified", order=1)
    err("the vector cannot be empty", traj_offsets=np.zeros(0, dtype=to.dtype), status=[])
    err("the expected size is 1, but the actual size is 2", status=[1, 2])
    err("The initial epoch of a polyjectory must be finite", epoch=float("inf"))
    err("could not be canonicalised", traj_file=tmp_path / "nope")
    err("are the same file", time_file=traj)
    err("the initial offset value must be zero but it is 1 instead",
        traj_offsets=np.array([(1, 2)], dtype=to.dtype))
    err("is inconsistent with the offset and number of steps of the previous object",
        traj_offsets=np.array([(0, 1), (22, 1)], dtype=to.dtype), status=[1, 1])
    err("All the trajectories in a polyjectory have a number of steps equal to zero",
        traj_offsets=np.array([(0, 0)], dtype=to.dtype))
    err("the expected size in bytes is 168 but the actual size is 336 instead",
        traj_offsets=np.array([(0, 1)], dtype=to.dtype))
    assert traj.exists() is False  # moved into the (removed) data directory
