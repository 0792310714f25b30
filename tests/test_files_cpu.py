"""Data directories of the drop-in conjunctions object, on the host side
(mizuba/detail/file_utils.cpp:95-202, mizuba/tmpdir.cpp, mizuba/core.cpp:69-86,
mizuba/test/test_conjunctions.py:496-583).  No GPU needed."""

import gc
import os

import numpy as np
import pytest

from mizuba_b200 import get_tmpdir, set_tmpdir
from mizuba_b200._files import DataDir as _DataDir, MappedFile as _MappedFile, create_data_dir


def _mk(data_dir, tmpdir):
    return create_data_dir(data_dir, tmpdir, "mizuba_conjunctions")


def test_user_data_dir(tmp_path):
    d = tmp_path / "data_dir"
    p = _mk(d, None)
    assert os.path.isdir(p) and p == os.path.realpath(d)
    assert os.stat(p).st_mode & 0o777 == 0o700
    with pytest.raises(RuntimeError, match="Error while creating the directory"):
        _mk(d, None)


def test_temp_dirs(tmp_path):
    p = _mk(None, tmp_path)
    assert os.path.dirname(p) == os.path.realpath(tmp_path)
    assert os.path.basename(p).startswith("mizuba_conjunctions-")
    assert len(os.path.basename(p)) == len("mizuba_conjunctions-xxxx-xxxx-xxxx-xxxx")
    # An empty data_dir means "not given" (test_conjunctions.py:532-534).
    q = _mk("", tmp_path)
    assert os.path.dirname(q) == os.path.realpath(tmp_path) and q != p
    with pytest.raises(ValueError, match="Unable to canonicalise the path to the temporary dir"):
        _mk(None, tmp_path / "missing")


def test_global_tmpdir(tmp_path):
    orig = get_tmpdir()
    try:
        set_tmpdir(tmp_path)
        assert get_tmpdir() == os.fspath(tmp_path)
        p = _mk(None, None)
        assert os.path.dirname(p) == os.path.realpath(tmp_path)
        # An explicit tmpdir overrides the global one.
        other = tmp_path / "other"
        other.mkdir()
        assert os.path.dirname(_mk(None, other)) == os.path.realpath(other)
        set_tmpdir("")
        assert get_tmpdir() is None
        set_tmpdir(None)
        assert get_tmpdir() is None
    finally:
        set_tmpdir(orig)


def test_mapped_views_keep_the_directory(tmp_path):
    p = _mk(None, tmp_path)
    data = np.arange(24, dtype=np.uint64)
    with open(os.path.join(p, "mcodes"), "wb") as f:
        f.write(data.tobytes())
    with open(os.path.join(p, "conjunctions"), "wb") as f:
        f.write(b"\0")
    owner = _DataDir(p)
    mf = _MappedFile(owner, "mcodes")
    a = mf.array(np.uint64, 24, (4, 6))
    assert not a.flags.writeable and np.array_equal(a.ravel(), data)
    with pytest.raises(ValueError):
        a[0, 0] = 1
    empty = _MappedFile(owner, "conjunctions").array(np.uint8, 0)
    assert empty.size == 0 and not empty.flags.writeable
    mf.advise_dontneed()
    row = a[2]
    del owner, mf, a, empty
    gc.collect()
    assert os.path.isdir(p) and row[0] == 12
    del row
    gc.collect()
    assert not os.path.exists(p)
