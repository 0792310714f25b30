"""Host-side polyjectory container.

Mirrors ``mizuba.polyjectory`` (mizuba/expose_polyjectory.cpp:126-300,
mizuba/polyjectory.cpp:70-1040): the same constructors (from lists of
per-object arrays, ``from_datafiles``, ``mount``), argument names,
validation order and error messages, the per-object view
``pj[i] -> (traj[n_steps, order + 1, 7], times[n_steps + 1], status)``, and
the same storage: a private data directory (the user's ``data_dir``, or a
``mizuba_polyjectory-XXXX-XXXX-XXXX-XXXX`` directory under ``tmpdir``, the
global temporary directory or the system's) holding the files ``desc``,
``traj_offsets``, ``time_offsets``, ``traj``, ``time`` and ``status`` in
mizuba's layout, mapped read-only.  The directory is removed when the
polyjectory and every array taken from it are gone, unless ``persist`` is
set; a persistent directory can be opened again with ``mount``, including
one that mizuba itself wrote.

``from_arrays`` (an extension) adopts flat arrays in memory without a data
directory unless one is asked for.  The flat arrays are what the C ABI
uploads to the GPU; ``state_eval`` / ``state_meval`` run there.
"""

from __future__ import annotations

import os
import pathlib
import struct

import numpy as np

from ._files import DataDir, MappedFile, create_data_dir, write_read_only

__all__ = ["polyjectory"]

# Per-object trajectory offset: offset (in doubles) into the traj file and
# number of steps (polyjectory::traj_offset, mizuba/polyjectory.hpp:83-93).
TRAJ_OFFSET = np.dtype([("offset", "<u8"), ("n_steps", "<u8")])

# The descriptor file (polyjectory_impl::descriptor, mizuba/polyjectory.cpp:88-108):
# version (unsigned), persist (bool), n_objs (size_t), order + 1 (uint32),
# maxT, epoch, epoch2 (double), in the x86-64 layout of that struct.
_DESC = struct.Struct("<I?3xQI4xddd")
_PJ_VERSION = 0
_PJ_FILES = ("desc", "traj_offsets", "time_offsets", "traj", "time", "status")


def _two_sum(a, b):
    """Knuth's error-free sum: the normalised double-length (hi, lo) of
    a + b (hilo_to_dfloat, mizuba/detail/dfloat_utils.hpp:34-51)."""
    s = a + b
    bp = s - a
    ap = s - bp
    lo = (a - ap) + (b - bp)
    if not (np.isfinite(s) and np.isfinite(lo)):
        raise ValueError(
            f"The normalisation of the double-length number with components ({_fmt(a)}, {_fmt(b)}) "
            "produced a non-finite result"
        )
    return float(s), float(lo)


def _fmt(x: float) -> str:
    return repr(float(x))


class polyjectory:
    """Piecewise-polynomial trajectories of a set of objects."""

    traj_offset = TRAJ_OFFSET

    def __init__(self, trajs, times, status, epoch=0.0, epoch2=0.0, data_dir=None, persist=False, tmpdir=None):
        trajs = [np.asarray(t, dtype=np.float64) for t in trajs]
        times = [np.asarray(t, dtype=np.float64) for t in times]
        status = np.asarray(status, dtype=np.int32)

        for t in trajs:
            if t.ndim != 3:
                raise ValueError(
                    "A trajectory array must have 3 dimensions, but instead "
                    f"{t.ndim} dimension(s) were detected"
                )
            if t.shape[2] != 7:
                raise ValueError(
                    "A trajectory array must have a size of 7 in the third dimension, "
                    f"but instead a size of {t.shape[2]} was detected"
                )
        for t in times:
            if t.ndim != 1:
                raise ValueError(
                    "A time array must have 1 dimension, but instead "
                    f"{t.ndim} dimension(s) were detected"
                )
        if status.ndim != 1:
            raise ValueError(
                "A status array must have 1 dimension, but instead "
                f"{status.ndim} dimension(s) were detected"
            )

        if data_dir is not None and tmpdir is not None:
            raise ValueError(
                "The 'data_dir' and 'tmpdir' construction arguments cannot be provided at the same time"
            )
        n_objs = len(trajs)
        if n_objs == 0:
            raise ValueError(
                "Cannot initialise a polyjectory object from an empty list of trajectories"
            )
        if n_objs != len(times):
            raise ValueError(
                "In the construction of a polyjectory, the number of objects deduced from "
                f"the list of trajectories ({n_objs}) is inconsistent with the number of "
                f"objects deduced from the list of times ({len(times)})"
            )
        if n_objs != status.shape[0]:
            raise ValueError(
                "In the construction of a polyjectory, the number of objects deduced from "
                f"the list of trajectories ({n_objs}) is inconsistent with the number of "
                f"objects deduced from the status list ({status.shape[0]})"
            )
        if not np.isfinite(epoch):
            raise ValueError(
                "The initial epoch of a polyjectory must be finite, but instead a value "
                f"of {_fmt(epoch)} was provided"
            )
        if not np.isfinite(epoch2):
            raise ValueError(
                "The second component of the initial epoch of a polyjectory must be "
                f"finite, but instead a value of {_fmt(epoch2)} was provided"
            )

        hi, lo = _two_sum(float(epoch), float(epoch2))
        path = create_data_dir(data_dir, tmpdir, "mizuba_polyjectory")
        try:
            self._build(trajs, times, status, hi, lo, path, bool(persist))
        except BaseException:
            import shutil

            shutil.rmtree(path, ignore_errors=True)
            raise

    def _build(self, trajs, times, status, hi, lo, path, persist):
        n_objs = len(trajs)
        op1 = trajs[0].shape[1]
        if op1 < 3:
            raise ValueError(
                "The trajectory polynomial order for the first object is less than 2 - "
                "this is not allowed"
            )
        for i, t in enumerate(trajs[1:], start=1):
            if t.shape[1] != op1:
                raise ValueError(
                    f"The trajectory polynomial order for the object at index {i} is "
                    "inconsistent with the polynomial order deduced from the first "
                    f"object ({op1 - 1})"
                )
        steps = np.array([t.shape[0] for t in trajs], dtype=np.uint64)
        if int(steps.sum()) == 0:
            raise ValueError(
                "All the trajectories in a polyjectory have a number of steps equal to "
                "zero: this is not allowed"
            )
        for i, (tr, tm) in enumerate(zip(trajs, times)):
            if tm.shape[0] == 0:
                if tr.shape[0] != 0:
                    raise ValueError(
                        f"The trajectory of the object at index {i} has a nonzero number "
                        "of steps but no associated time data"
                    )
            elif tm.shape[0] - 1 != tr.shape[0]:
                raise ValueError(
                    f"The number of steps for the trajectory of the object at index {i} "
                    f"is {tr.shape[0]}, but the number of times is {tm.shape[0]} (the "
                    "number of times must be equal to the number of steps + 1)"
                )
        for i, (tr, tm) in enumerate(zip(trajs, times)):
            if not np.all(np.isfinite(tr)):
                raise ValueError(
                    f"A non-finite value was found in the trajectory at index {i}"
                )
            if not np.all(np.isfinite(tm)):
                raise ValueError(
                    f"A non-finite time coordinate was found for the object at index {i}"
                )
            if np.any(tm < 0):
                raise ValueError(
                    f"A negative time coordinate was found for the object at index {i}"
                )
            if tm.shape[0] > 1 and not np.all(tm[1:] > tm[:-1]):
                raise ValueError(
                    f"The sequence of times for the object at index {i} is not "
                    "monotonically increasing"
                )

        per_obj = steps * np.uint64(op1 * 7)
        traj_off = np.zeros((n_objs, 2), dtype=np.uint64)
        traj_off[1:, 0] = np.cumsum(per_obj)[:-1]
        traj_off[:, 1] = steps
        tsz = np.array([t.shape[0] for t in times], dtype=np.uint64)
        time_off = np.zeros(n_objs, dtype=np.uint64)
        time_off[1:] = np.cumsum(tsz)[:-1]
        traj = np.concatenate([t.reshape(-1) for t in trajs]) if n_objs else np.zeros(0)
        time = np.concatenate(times) if n_objs else np.zeros(0)
        _store(path, traj, traj_off, time, time_off, status, op1, _max_time(time, traj_off, time_off), hi, lo,
               persist)
        self._attach(path, keep=persist)

    @classmethod
    def from_arrays(cls, traj, traj_offsets, time, time_offsets, status, order, epoch=0.0, epoch2=0.0,
                    data_dir=None, persist=False, tmpdir=None, traj_checked=False):
        """Adopts flat arrays already in the mizuba layout (vectorised checks).
        Without ``data_dir``, ``persist`` or ``tmpdir`` the data stay in
        memory and there is no data directory.  ``traj_checked``: the
        trajectory values were already found finite where they were made
        (the GPU SGP4 production checks them on the device), so the scan is
        skipped."""
        self = cls.__new__(cls)
        traj = np.ascontiguousarray(traj, dtype=np.float64)
        traj_offsets = np.ascontiguousarray(traj_offsets, dtype=np.uint64).reshape(-1, 2)
        time = np.ascontiguousarray(time, dtype=np.float64)
        time_offsets = np.ascontiguousarray(time_offsets, dtype=np.uint64)
        status = np.ascontiguousarray(status, dtype=np.int32)
        if order < 2:
            raise ValueError(
                "The trajectory polynomial order for the first object is less than 2 - "
                "this is not allowed"
            )
        if not traj_checked and not np.all(np.isfinite(traj)):
            raise ValueError("A non-finite value was found in the trajectory data")
        if not np.all(np.isfinite(time)) or np.any(time < 0):
            raise ValueError("Invalid time data")
        hi, lo = _two_sum(float(epoch), float(epoch2))
        maxT = _max_time(time, traj_offsets, time_offsets)
        if data_dir is None and tmpdir is None and not persist:
            self._set(traj, traj_offsets, time, time_offsets, status, int(order), hi, lo, maxT, None, False)
            return self
        path = create_data_dir(data_dir, tmpdir, "mizuba_polyjectory")
        try:
            _store(path, traj, traj_offsets, time, time_offsets, status, int(order) + 1, maxT, hi, lo,
                   bool(persist))
            self._attach(path, keep=bool(persist))
        except BaseException:
            import shutil

            shutil.rmtree(path, ignore_errors=True)
            raise
        return self

    @staticmethod
    def from_datafiles(traj_file, time_file, order, traj_offsets, status, epoch=0.0, epoch2=0.0, data_dir=None,
                       persist=False, tmpdir=None):
        """A polyjectory over existing data files, which are moved into its data
        directory (polyjectory.cpp:650-948, expose_polyjectory.cpp:216-249)."""
        to = np.asarray(traj_offsets)
        if to.ndim != 1:
            raise ValueError(
                "The array of trajectory offsets passed to 'from_datafiles()' must have 1 dimension, but the "
                f"number of dimensions is {to.ndim} instead"
            )
        if to.dtype.names:
            to = np.stack([to["offset"].astype(np.uint64), to["n_steps"].astype(np.uint64)], axis=1)
        else:
            to = to.astype(np.uint64).reshape(-1, 2)
        status = np.asarray(status, dtype=np.int32).reshape(-1)
        if data_dir is not None and tmpdir is not None:
            raise ValueError(
                "The 'data_dir' and 'tmpdir' construction arguments cannot be provided at the same time"
            )
        order = int(order)
        if order < 2 or order == 2**32 - 1:
            raise ValueError(f"Invalid polynomial order {order} specified during the construction of a polyjectory")
        op1 = order + 1
        n = to.shape[0]
        if n == 0:
            raise ValueError(
                "Invalid trajectory offsets vector passed to the constructor of a polyjectory: the vector cannot "
                "be empty"
            )
        if status.shape[0] != n:
            raise ValueError(
                "Invalid status vector passed to the constructor of a polyjectory: the expected size is "
                f"{n}, but the actual size is {status.shape[0]}"
            )
        if not np.isfinite(epoch):
            raise ValueError(
                "The initial epoch of a polyjectory must be finite, but instead a value "
                f"of {_fmt(epoch)} was provided"
            )
        if not np.isfinite(epoch2):
            raise ValueError(
                "The second component of the initial epoch of a polyjectory must be "
                f"finite, but instead a value of {_fmt(epoch2)} was provided"
            )
        hi, lo = _two_sum(float(epoch), float(epoch2))
        try:
            traj_path = os.path.realpath(os.fspath(traj_file), strict=True)
            time_path = os.path.realpath(os.fspath(time_file), strict=True)
        except OSError:
            raise ValueError(
                "Invalid data file(s) passed to the constructor of a polyjectory: the path(s) could not be "
                "canonicalised"
            ) from None
        if traj_path == time_path:
            raise ValueError(
                "Invalid data file(s) passed to the constructor of a polyjectory: the trajectory data file and "
                "the time data file are the same file"
            )
        steps = to[:, 1]
        offs = to[:, 0]
        if offs[0] != 0:
            raise ValueError(
                "Invalid trajectory offsets vector passed to the constructor of a polyjectory: the initial "
                f"offset value must be zero but it is {int(offs[0])} instead"
            )
        for i in range(1, n):
            if offs[i] < offs[i - 1]:
                raise ValueError(
                    "Invalid trajectory offsets vector passed to the constructor of a polyjectory: the offset "
                    f"of the object at index {i} is less than the offset of the previous object"
                )
            if int(offs[i]) - int(offs[i - 1]) != int(steps[i - 1]) * op1 * 7:
                raise ValueError(
                    "Inconsistent data detected in the trajectory offsets vector passed to the constructor of a "
                    f"polyjectory: the offset of the object at index {i} is inconsistent with the offset and "
                    "number of steps of the previous object"
                )
        n_traj = int(steps.sum()) * op1 * 7
        tsz = steps + (steps != 0).astype(np.uint64)
        n_time = int(tsz.sum())
        if n_traj == 0:
            raise ValueError(
                "All the trajectories in a polyjectory have a number of steps equal to zero: this is not allowed"
            )
        time_off = np.zeros(n, dtype=np.uint64)
        time_off[1:] = np.cumsum(tsz)[:-1]
        path = create_data_dir(data_dir, tmpdir, "mizuba_polyjectory")
        self = polyjectory.__new__(polyjectory)
        try:
            write_read_only(os.path.join(path, "traj_offsets"), to)
            write_read_only(os.path.join(path, "time_offsets"), time_off)
            write_read_only(os.path.join(path, "status"), status)
            tp, mp = os.path.join(path, "traj"), os.path.join(path, "time")
            os.rename(traj_path, tp)
            os.rename(time_path, mp)
            if not os.path.isfile(tp):
                raise ValueError(
                    "Invalid trajectory data file passed to the constructor of a polyjectory: the file is not a "
                    "regular file"
                )
            if not os.path.isfile(mp):
                raise ValueError(
                    "Invalid time data file passed to the constructor of a polyjectory: the file is not a regular "
                    "file"
                )
            os.chmod(tp, 0o400)
            os.chmod(mp, 0o400)
            for nm, p, want in (("trajectory", tp, n_traj * 8), ("time", mp, n_time * 8)):
                got = os.path.getsize(p)
                if got != want:
                    raise ValueError(
                        f"Invalid {nm} data file passed to the constructor of a polyjectory: the expected size in "
                        f"bytes is {want} but the actual size is {got} instead"
                    )
            dd = DataDir(path, keep=True)
            traj = MappedFile(dd, "traj").array(np.float64, n_traj)
            time = MappedFile(dd, "time").array(np.float64, n_time)
            _check_values(traj, to, time, time_off, op1)
            maxT = _max_time(time, to, time_off)
            del traj, time, dd
            with open(os.path.join(path, "desc"), "wb") as f:
                f.write(_DESC.pack(_PJ_VERSION, bool(persist), n, op1, maxT, hi, lo))
            os.chmod(os.path.join(path, "desc"), 0o400)
            self._attach(path, keep=bool(persist))
        except BaseException:
            import shutil

            shutil.rmtree(path, ignore_errors=True)
            raise
        return self

    @staticmethod
    def mount(data_dir):
        """Opens the persistent polyjectory stored in ``data_dir``
        (polyjectory.cpp:188-240 and :956-982)."""
        try:
            path = os.path.realpath(os.fspath(data_dir), strict=True)
        except OSError:
            raise ValueError(
                f"Error while trying to mount a polyjectory on path '{os.fspath(data_dir)}': the path could not "
                "be canonicalised (does it exist?)"
            ) from None
        if not os.path.isdir(path):
            raise ValueError(f"Cannot mount a polyjectory on path '{path}': the path is not a directory")
        with open(os.path.join(path, "desc"), "rb") as f:
            raw = f.read(_DESC.size)
        version = struct.unpack_from("<I", raw)[0]
        if version != _PJ_VERSION:
            raise ValueError(
                "Version mismatch when trying to mount() a polyjectory: the current polyjectory version is "
                f"{_PJ_VERSION}, while the polyjectory in the data dir '{path}' has a version number of {version}"
            )
        if not _DESC.unpack(raw)[1]:
            raise ValueError(
                f"Cannot mount() a polyjectory on the the data dir '{path}': the data is not persistent"
            )
        self = polyjectory.__new__(polyjectory)
        self._attach(path, keep=True)
        return self

    def _attach(self, path, keep):
        """Maps the files of the data directory at ``path``."""
        dd = DataDir(path, keep=keep)
        f = {nm: MappedFile(dd, nm) for nm in _PJ_FILES}
        with open(f["desc"].path, "rb") as fh:
            _, persist, n, op1, maxT, hi, lo = _DESC.unpack(fh.read(_DESC.size))
        traj_off = f["traj_offsets"].array(np.uint64, 2 * n, (n, 2))
        time_off = f["time_offsets"].array(np.uint64, n)
        traj = f["traj"].array(np.float64, f["traj"].size // 8)
        time = f["time"].array(np.float64, f["time"].size // 8)
        status = f["status"].array(np.int32, n)
        self._set(traj, traj_off, time, time_off, status, op1 - 1, hi, lo, maxT, dd, bool(persist))
        self._files = f

    def _set(self, traj, traj_off, time, time_off, status, order, hi, lo, maxT, dd, persist):
        self._traj = traj
        self._traj_off = traj_off
        self._time = time
        self._time_off = time_off
        self._status = status
        self._order = int(order)
        self._epoch = (hi, lo)
        self._maxT = float(maxT)
        self._n = int(traj_off.shape[0])
        self._dd = dd
        self._persist = persist
        self._files = {}
        self._detached = False
        for a in (self._traj, self._traj_off, self._time, self._time_off, self._status):
            if a.flags.writeable:
                a.setflags(write=False)

    def _check(self):
        if getattr(self, "_detached", True):
            raise ValueError("Cannot operate on a detached polyjectory")

    def detach(self):
        """Releases this object's hold on the data (polyjectory::detach,
        polyjectory.cpp:984-987): a non-persistent data directory is removed
        once no array taken from it is left."""
        for nm in ("_traj", "_traj_off", "_time", "_time_off", "_status", "_files", "_dd", "_device"):
            self.__dict__.pop(nm, None)
        self._detached = True

    @property
    def is_detached(self):
        return getattr(self, "_detached", True)

    def hint_release(self):
        """Tells the OS that the pages of the mapped files may be dropped
        (polyjectory::hint_release, polyjectory.cpp:992-1004)."""
        self._check()
        for f in self._files.values():
            f.advise_dontneed()

    @property
    def data_dir(self):
        self._check()
        return None if self._dd is None else pathlib.Path(self._dd.path)

    @property
    def persist(self):
        self._check()
        return self._persist

    # --- reference property names
    @property
    def n_objs(self) -> int:
        self._check()
        return self._n

    @property
    def maxT(self) -> float:
        self._check()
        return self._maxT

    @property
    def epoch(self):
        self._check()
        return self._epoch

    @property
    def poly_order(self) -> int:
        self._check()
        return self._order

    @property
    def status(self):
        self._check()
        return self._status

    def __getitem__(self, i):
        self._check()
        i = int(i)
        if i < 0 or i >= self._n:
            raise IndexError(
                f"Invalid object index {i} specified - the total number of objects in "
                f"the polyjectory is only {self._n}"
            )
        off, ns = (int(x) for x in self._traj_off[i])
        op1 = self._order + 1
        tr = self._traj[off : off + ns * op1 * 7].reshape(ns, op1, 7)
        t0 = int(self._time_off[i])
        tm = self._time[t0 : t0 + (ns + 1 if ns > 0 else 0)]
        return tr, tm, int(self._status[i])

    # --- flat arrays (mizuba layout), consumed by the C ABI
    @property
    def arrays(self):
        self._check()
        return dict(
            traj=self._traj,
            traj_offsets=self._traj_off,
            time=self._time,
            time_offsets=self._time_off,
            n_objs=self._n,
            order=self._order,
            maxT=self._maxT,
        )

    # --- state evaluation on the GPU (polyjectory::state_eval / state_meval,
    # mizuba/polyjectory.cpp:1092-1366; argument handling of the Python
    # exposure, mizuba/expose_polyjectory.cpp:65-98 and 308-530)
    def state_eval(self, time, out=None, obj_idx=None):
        """State (x, y, z, vx, vy, vz, r) of every object, or of the objects in
        ``obj_idx``, at ``time`` (a scalar, or one time per evaluated object).
        Returns ``out`` (shape ``(n, 7)``), NaN where an object has no data."""
        self._check()
        # Check order of the reference's exposure: selector, output array,
        # then the time array.
        sel = _eval_selector(obj_idx)
        tm_arr = None
        if not isinstance(time, (float, int, np.floating, np.integer)):
            tm_arr = _as_f64(time)
        if out is not None:
            _check_out(out, "state_eval")
            if out.ndim != 2:
                raise ValueError(
                    "The output array passed to state_eval() must have 2 dimensions, but the number of "
                    f"dimensions is {out.ndim} instead"
                )
            if out.shape[1] != 7:
                raise ValueError(
                    "The output array passed to state_eval() must have a size of 7 in the second dimension, "
                    f"but the size in the second dimension is {out.shape[1]} instead"
                )
            _check_overlap(out, tm_arr, sel, obj_idx, "state_eval")
        else:
            out = np.empty((self._n if sel is None else sel.shape[0], 7))
        if tm_arr is not None:
            _check_cc(tm_arr, "The time array passed to state_eval() must be C contiguous and properly aligned")
            if tm_arr.ndim != 1:
                raise ValueError(
                    "The time array passed to state_eval() must have 1 dimension, but the number of "
                    f"dimensions is {tm_arr.ndim} instead"
                )
        from .conjunctions import _raise, to_device

        dev = to_device(self)
        if tm_arr is None:
            tbuf = np.array([float(time)])
            tm_ptr, tm_size = tbuf.ctypes.data, -1
        else:
            tm_ptr, tm_size = tm_arr.ctypes.data, tm_arr.shape[0]
        rc = dev._L.mzb_pj_state_eval(dev._h, out.ctypes.data, out.shape[0], tm_ptr, tm_size,
                                      None if sel is None else sel.ctypes.data,
                                      -1 if sel is None else sel.shape[0])
        if rc != 0:
            _raise(dev._L, rc)
        return out

    def state_meval(self, time, out=None, obj_idx=None):
        """States at several times per object: ``time`` is 1-D (the same times
        for every evaluated object) or 2-D (one row per evaluated object).
        Returns ``out`` (shape ``(n, n_times, 7)``)."""
        self._check()
        sel = _eval_selector(obj_idx)
        tm = _as_f64(time)
        _check_cc(tm, "The time array passed to state_meval() must be C contiguous and properly aligned")
        if tm.ndim not in (1, 2):
            raise ValueError(
                "The time array passed to state_meval() must have either 1 or 2 dimensions, but the number of "
                f"dimensions is {tm.ndim} instead"
            )
        n_t = tm.shape[0] if tm.ndim == 1 else tm.shape[1]
        if out is not None:
            _check_out(out, "state_meval")
            if out.ndim != 3:
                raise ValueError(
                    "The output array passed to state_meval() must have 3 dimensions, but the number of "
                    f"dimensions is {out.ndim} instead"
                )
            if out.shape[2] != 7:
                raise ValueError(
                    "The output array passed to state_meval() must have a size of 7 in the third dimension, "
                    f"but the size in the third dimension is {out.shape[2]} instead"
                )
            _check_overlap(out, tm, sel, obj_idx, "state_meval")
        else:
            out = np.empty((self._n if sel is None else sel.shape[0], n_t, 7))
        from .conjunctions import _raise, to_device

        dev = to_device(self)
        rc = dev._L.mzb_pj_state_meval(dev._h, out.ctypes.data, out.shape[0], out.shape[1], tm.ctypes.data,
                                       tm.ndim, tm.shape[0], tm.shape[1] if tm.ndim == 2 else 0,
                                       None if sel is None else sel.ctypes.data,
                                       -1 if sel is None else sel.shape[0])
        if rc != 0:
            _raise(dev._L, rc)
        return out


def _as_f64(a):
    """A float64 array view of ``a``: float64 arrays as they are (so that
    layout checks see them), anything else converted."""
    if isinstance(a, np.ndarray) and a.dtype == np.float64:
        return a
    return np.asarray(a, dtype=np.float64)


def _check_cc(a, msg):
    if not (a.flags.c_contiguous and a.flags.aligned):
        raise ValueError(msg)


def _check_out(out, fn):
    if not isinstance(out, np.ndarray) or out.dtype != np.float64:
        raise TypeError(f"The output array passed to {fn}() must be a NumPy array of float64")
    if not out.flags.writeable:
        raise ValueError(f"The output array passed to {fn}() must be writeable")
    _check_cc(out, f"The output array passed to {fn}() must be C contiguous and properly aligned")


def _check_overlap(out, tm, sel, obj_idx, fn):
    # The output may not share memory with the inputs (the time array and
    # the selector may share memory with each other).
    if tm is not None and np.may_share_memory(out, tm):
        raise ValueError(
            f"Potential memory overlap detected between the output array passed to {fn}() and the time array"
        )
    if sel is not None and isinstance(obj_idx, np.ndarray) and np.may_share_memory(out, sel):
        raise ValueError(
            f"Potential memory overlap detected between the output array passed to {fn}() and the array of "
            "object indices"
        )


def _eval_selector(obj_idx):
    """The object selector as a 1-D uintp array, or None (all objects)."""
    if obj_idx is None:
        return None
    if isinstance(obj_idx, (int, np.integer)):
        if int(obj_idx) < 0:
            raise OverflowError("can't convert negative int to unsigned")
        return np.array([int(obj_idx)], dtype=np.uintp)
    if isinstance(obj_idx, np.ndarray) and obj_idx.dtype == np.uintp:
        sel = obj_idx
    else:
        sel = np.asarray(obj_idx)
        if sel.dtype.kind == "i" and sel.size and sel.min() < 0:
            raise OverflowError("can't convert negative int to unsigned")
        sel = sel.astype(np.uintp)
    _check_cc(sel, "The selector array passed to state_eval() must be C contiguous and properly aligned")
    if sel.ndim != 1:
        raise ValueError(
            "The selector array passed to state_eval() must have 1 dimension, but the number of dimensions "
            f"is {sel.ndim} instead"
        )
    return sel


def _max_time(time, traj_off, time_off):
    """Duration of the longest trajectory: the largest last time point."""
    steps = traj_off[:, 1]
    nz = steps > 0
    if not np.any(nz):
        return 0.0
    last = (time_off[nz] + steps[nz]).astype(np.int64)
    return float(time[last].max())


def _check_values(traj, traj_off, time, time_off, op1):
    """The per-object data checks of the constructors (polyjectory.cpp:553-605,
    :870-932), in object order."""
    bad_traj = ~np.isfinite(traj)
    bad_time = ~np.isfinite(time)
    for i in range(traj_off.shape[0]):
        off, ns = int(traj_off[i, 0]), int(traj_off[i, 1])
        if ns and bad_traj[off:off + ns * op1 * 7].any():
            raise ValueError(f"A non-finite value was found in the trajectory at index {i}")
        t0 = int(time_off[i])
        tm = time[t0:t0 + ns + (1 if ns else 0)]
        if bad_time[t0:t0 + tm.shape[0]].any():
            raise ValueError(f"A non-finite time coordinate was found for the object at index {i}")
        if np.any(tm < 0):
            raise ValueError(f"A negative time coordinate was found for the object at index {i}")
        if tm.shape[0] > 1 and not np.all(tm[1:] > tm[:-1]):
            raise ValueError(
                f"The sequence of times for the object at index {i} is not monotonically increasing"
            )


def _store(path, traj, traj_off, time, time_off, status, op1, maxT, hi, lo, persist):
    """Writes the data files of a polyjectory (polyjectory.cpp:143-171 and
    :528-618), each readable by its owner only."""
    write_read_only(os.path.join(path, "traj_offsets"), np.ascontiguousarray(traj_off, dtype=np.uint64))
    write_read_only(os.path.join(path, "time_offsets"), np.ascontiguousarray(time_off, dtype=np.uint64))
    write_read_only(os.path.join(path, "status"), np.ascontiguousarray(status, dtype=np.int32))
    write_read_only(os.path.join(path, "traj"), np.ascontiguousarray(traj, dtype=np.float64))
    write_read_only(os.path.join(path, "time"), np.ascontiguousarray(time, dtype=np.float64))
    desc = np.frombuffer(_DESC.pack(_PJ_VERSION, bool(persist), int(traj_off.shape[0]), int(op1), float(maxT),
                                    float(hi), float(lo)), dtype=np.uint8)
    write_read_only(os.path.join(path, "desc"), desc)
