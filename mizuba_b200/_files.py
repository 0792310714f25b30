"""Data directories and memory-mapped files shared by polyjectories and
conjunctions objects (mizuba/detail/file_utils.cpp, mizuba/tmpdir.cpp).

A data directory is created readable by its owner only, either at a
user-given path or under a temporary directory with a
``<prefix>-XXXX-XXXX-XXXX-XXXX`` name.  Its files are mapped read-only;
arrays made from a mapping keep it, and through it the directory, alive.
A directory that is not persistent is removed once nothing uses it any
more."""

from __future__ import annotations

import mmap
import os
import secrets
import shutil
import tempfile
import threading
import weakref

import numpy as np

_tmpdir_lock = threading.Lock()
_tmpdir = os.environ.get("MIZUBA_TMPDIR") or None


def get_tmpdir():
    """The global directory for temporary data directories (None = the
    system's; mizuba/tmpdir.cpp:63-68, mizuba/core.cpp:69-76)."""
    with _tmpdir_lock:
        return _tmpdir


def set_tmpdir(path):
    """Sets the global temporary directory; None or "" resets it
    (mizuba/tmpdir.cpp:70-75, mizuba/core.cpp:77-86)."""
    global _tmpdir
    with _tmpdir_lock:
        _tmpdir = None if path is None or os.fspath(path) == "" else os.fspath(path)


def create_data_dir(data_dir, tmpdir, prefix):
    """create_dir_0700 / create_temp_dir (mizuba/detail/file_utils.cpp:95-202):
    a new directory readable by its owner only; returns its canonical path."""
    if data_dir is not None and os.fspath(data_dir) != "":
        path = os.fspath(data_dir)
        try:
            os.mkdir(path, 0o700)
        except FileExistsError:
            raise RuntimeError(
                f"Error while creating the directory '{path}': the directory already exists"
            ) from None
        os.chmod(path, 0o700)
        return os.path.realpath(path)
    if tmpdir is not None and os.fspath(tmpdir) != "":
        base = os.fspath(tmpdir)
    else:
        base = get_tmpdir() or tempfile.gettempdir()
    try:
        base = os.path.realpath(base, strict=True)
    except OSError:
        raise ValueError(
            f"Unable to canonicalise the path to the temporary dir '{base}' (does it exist?)"
        ) from None
    for _ in range(10):
        path = os.path.join(base, prefix + "-" + "-".join(secrets.token_hex(2) for _ in range(4)))
        try:
            os.mkdir(path, 0o700)
        except FileExistsError:
            continue
        except OSError:
            break
        os.chmod(path, 0o700)
        return path
    raise ValueError(f"Unable to create a unique temporary directory in the path '{base}'")


def write_read_only(path, data: np.ndarray):
    """Writes a new file (which must not exist) with the array's bytes and
    leaves it readable by its owner only (dump_vector_to_file,
    mizuba/polyjectory.cpp:328-344)."""
    fd = os.open(path, os.O_WRONLY | os.O_CREAT | os.O_EXCL | os.O_CLOEXEC, 0o600)
    try:
        mv = memoryview(np.ascontiguousarray(data)).cast("B")
        off = 0
        while off < len(mv):
            off += os.write(fd, mv[off:off + (1 << 30)])
    finally:
        os.close(fd)
    os.chmod(path, 0o400)


class DataDir:
    """Owns a data directory.  Unless ``keep`` is set, the directory is
    removed when this object is collected, i.e. once its owner and every
    array mapped from its files are gone."""

    def __init__(self, path, keep=False):
        self.path = path
        self.keep = keep
        if not keep:
            weakref.finalize(self, shutil.rmtree, path, True)


class MappedFile:
    """One file of a data directory mapped read-only.  Arrays made from it
    keep it (and through it the data directory) alive."""

    def __init__(self, owner: DataDir, name: str):
        self._owner = owner
        self.path = os.path.join(owner.path, name)
        self.size = os.path.getsize(self.path)
        self._mm = None
        if self.size:
            with open(self.path, "rb") as f:
                self._mm = mmap.mmap(f.fileno(), 0, access=mmap.ACCESS_READ)

    def __buffer__(self, flags):
        return memoryview(self._mm if self._mm is not None else b"")

    def __release_buffer__(self, view):
        view.release()

    def array(self, dtype, count, shape=None):
        if count == 0:
            a = np.zeros(0, dtype=dtype)
            a.setflags(write=False)
        else:
            a = np.frombuffer(self, dtype=dtype, count=count)
        return a.reshape(shape) if shape is not None else a

    def advise_dontneed(self):
        # advise_dontneed (mizuba/detail/file_utils.cpp:421-470).
        if self._mm is None:
            return
        self._mm.madvise(mmap.MADV_DONTNEED)
        fd = os.open(self.path, os.O_RDONLY | os.O_CLOEXEC)
        try:
            os.posix_fadvise(fd, 0, 0, os.POSIX_FADV_DONTNEED)
        finally:
            os.close(fd)
