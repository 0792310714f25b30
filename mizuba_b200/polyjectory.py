"""Host-side polyjectory container.

Mirrors the in-memory constructor of ``mizuba.polyjectory``
(mizuba/expose_polyjectory.cpp:126-215, mizuba/polyjectory.cpp:352-619): the
same argument names, the same validation order and error messages, and the
same per-object view ``pj[i] -> (traj[n_steps, order + 1, 7], times[n_steps + 1],
status)`` (mizuba/polyjectory.cpp:1006-1036).

The data are held as four flat arrays in mizuba's on-disk layout
(mizuba/polyjectory.cpp:91-107): ``traj`` (all objects' segments
concatenated, each ``[order + 1][7]`` row-major), ``traj_offsets`` (per object
``(offset in doubles, n_steps)``), ``time`` and ``time_offsets``.  These
arrays are what the C ABI uploads to the GPU.
"""

from __future__ import annotations

import numpy as np

__all__ = ["polyjectory"]


def _fmt(x: float) -> str:
    return repr(float(x))


class polyjectory:
    """Piecewise-polynomial trajectories of a set of objects."""

    def __init__(self, trajs, times, status, epoch=0.0, epoch2=0.0):
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
        self._init_arrays(
            np.ascontiguousarray(traj),
            traj_off,
            np.ascontiguousarray(time),
            time_off,
            status.copy(),
            op1 - 1,
            epoch,
        )

    @classmethod
    def from_arrays(cls, traj, traj_offsets, time, time_offsets, status, order, epoch=0.0):
        """Adopts flat arrays already in the mizuba layout (vectorised checks)."""
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
        if not np.all(np.isfinite(traj)):
            raise ValueError("A non-finite value was found in the trajectory data")
        if not np.all(np.isfinite(time)) or np.any(time < 0):
            raise ValueError("Invalid time data")
        self._init_arrays(traj, traj_offsets, time, time_offsets, status, int(order), epoch)
        return self

    def _init_arrays(self, traj, traj_off, time, time_off, status, order, epoch):
        self._traj = traj
        self._traj_off = traj_off
        self._time = time
        self._time_off = time_off
        self._status = status
        self._order = int(order)
        self._epoch = float(epoch)
        n = traj_off.shape[0]
        steps = traj_off[:, 1]
        nz = steps > 0
        last = time_off[nz] + steps[nz]
        self._maxT = float(time[last.astype(np.int64)].max()) if np.any(nz) else 0.0
        for a in (self._traj, self._traj_off, self._time, self._time_off, self._status):
            a.setflags(write=False)
        self._n = n

    # --- reference property names
    @property
    def n_objs(self) -> int:
        return self._n

    @property
    def maxT(self) -> float:
        return self._maxT

    @property
    def epoch(self):
        return (self._epoch, 0.0)

    @property
    def poly_order(self) -> int:
        return self._order

    @property
    def status(self):
        return self._status

    def __getitem__(self, i):
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
