"""SGP4 polyjectories built on the GPU: the drop-in for mizuba's
``make_sgp4_polyjectory`` (mizuba/_sgp4_polyjectory.py:100-233 and
mizuba/make_sgp4_polyjectory.cpp:1461-1603), through the C ABI's
``mzb_make_sgp4_polyjectory``.

The element sets are general perturbations sets with mizuba's ``gpe_dtype``
fields; the result is a ``polyjectory`` whose time unit is days from
``jd_begin`` (converted to TAI), positions in km and velocities in km/s
(TEME), plus the sorted unique NORAD IDs, one per object.
"""

from __future__ import annotations

import ctypes as ct
from enum import IntEnum

import numpy as np

from . import _native
from .polyjectory import polyjectory

# mizuba's gpe_dtype (the gpe struct of mizuba/make_sgp4_polyjectory.hpp).
gpe_dtype = np.dtype([("norad_id", "<u8"), ("epoch_jd1", "<f8"), ("epoch_jd2", "<f8"), ("n0", "<f8"),
                      ("e0", "<f8"), ("i0", "<f8"), ("node0", "<f8"), ("omega0", "<f8"), ("m0", "<f8"),
                      ("bstar", "<f8")])


class sgp4_pj_status(IntEnum):
    """Per-object status codes (mizuba/_sgp4_polyjectory.py:35-55)."""

    OK = 0
    SGP4_ERROR_MEAN_ECC = 1
    SGP4_ERROR_MEAN_MEAN_MOTION = 2
    SGP4_ERROR_PERT_ECC = 3
    SGP4_ERROR_SEMI_LATUS_RECTUM = 4
    SGP4_DECAY = 6
    ERROR_NONFINITE = 10
    REENTRY = 11
    EXIT = 12
    ERROR_SMALL_STEP = 13
    ERROR_INTERPOLATION = 14


def _raise(L, rc):
    msg = L.mzb_last_error().decode()
    if rc == 1:
        raise ValueError(msg)
    if rc == 2:
        raise IndexError(msg)
    raise RuntimeError(msg)


def _as_gpes(gpes):
    """The element sets as a contiguous gpe_dtype array.  Accepts a NumPy
    array of gpe_dtype, or a table with the gpe_dtype columns (a pandas
    DataFrame or a mapping of column arrays), as the reference accepts a
    polars DataFrame (mizuba/_sgp4_polyjectory.py:160-180)."""
    if isinstance(gpes, np.ndarray):
        if gpes.dtype != gpe_dtype:
            raise TypeError(
                "When passing the 'gpes' argument to make_sgp4_polyjectory() as a NumPy array, the dtype must be "
                f"'gpe_dtype', but it is '{gpes.dtype}' instead"
            )
        return np.ascontiguousarray(gpes)
    cols = getattr(gpes, "columns", None)
    if cols is not None or isinstance(gpes, dict):
        out = np.zeros(len(gpes[gpe_dtype.names[0]]), dtype=gpe_dtype)
        for name in gpe_dtype.names:
            out[name] = np.asarray(gpes[name])
        return out
    raise TypeError(
        "The 'gpes' argument to make_sgp4_polyjectory() must be either a dataframe or a NumPy array, but it is of "
        f"type '{type(gpes)}' instead"
    )


def make_sgp4_polyjectory(gpes, jd_begin, jd_end, reentry_radius=0.0, exit_radius=float("inf"), data_dir=None,
                          persist=False, tmpdir=None):
    """Interpolates the element sets over [jd_begin, jd_end) (UTC Julian
    dates) with order-18 polynomials on the GPU.  ``gpes`` must be sorted by
    NORAD ID and then by epoch; each NORAD ID becomes one object.  Returns
    ``(polyjectory, norad_ids)``; ``polyjectory.status`` holds each object's
    ``sgp4_pj_status``."""
    if any(not isinstance(x, (float, int)) for x in (jd_begin, jd_end, reentry_radius, exit_radius)):
        raise TypeError(
            "The jd_begin, jd_end, reentry_radius and exit_radius arguments to make_sgp4_polyjectory() must all "
            "be floats or ints"
        )
    arr = _as_gpes(gpes)
    L = _native.core()
    h = ct.c_void_p()
    rc = L.mzb_make_sgp4_polyjectory(arr.ctypes.data if len(arr) else None, len(arr), float(jd_begin),
                                     float(jd_end), float(reentry_radius), float(exit_radius), ct.byref(h))
    if rc != 0:
        _raise(L, rc)
    try:
        sz = (ct.c_uint64 * 4)()
        L.mzb_sgp4_pj_sizes(h, ct.addressof(sz))
        n_objs, n_traj, n_time, order = (int(x) for x in sz)
        ep = (ct.c_double * 3)()
        L.mzb_sgp4_pj_epoch(h, ct.addressof(ep))
        traj = np.empty(n_traj)
        toff = np.empty((n_objs, 2), dtype=np.uint64)
        time = np.empty(n_time)
        tmoff = np.empty(n_objs, dtype=np.uint64)
        status = np.empty(n_objs, dtype=np.int32)
        rc = L.mzb_sgp4_pj_copy(h, traj.ctypes.data, toff.ctypes.data, time.ctypes.data, tmoff.ctypes.data,
                                status.ctypes.data)
        if rc != 0:
            _raise(L, rc)
        tm = (ct.c_double * 2)()
        L.mzb_sgp4_pj_timing(h, ct.addressof(tm))
    finally:
        L.mzb_sgp4_pj_free(h)
    if not np.any(toff[:, 1]):
        raise ValueError(
            "All the trajectories in a polyjectory have a number of steps equal to zero: this is not allowed"
        )
    # The coefficients were checked for finiteness on the device.
    pj = polyjectory.from_arrays(traj, toff, time, tmoff, status, order, ep[0], ep[1], data_dir=data_dir,
                                 persist=persist, tmpdir=tmpdir, traj_checked=True)
    pj.production_ms = {"interpolation": float(tm[0]), "layout": float(tm[1])}
    return pj, np.unique(arr["norad_id"])


def sgp4_propagate(gpes, tsince):
    """Batched SGP4/SDP4 on the GPU: every element set at every time
    (minutes from its own epoch).  Returns (states [n][t][6] in km, km/s;
    error codes [n][t])."""
    arr = _as_gpes(gpes)
    t = np.ascontiguousarray(tsince, dtype=np.float64).ravel()
    out = np.empty((len(arr), len(t), 6))
    err = np.empty((len(arr), len(t)), dtype=np.int32)
    if len(arr) and len(t):
        L = _native.core()
        rc = L.mzb_sgp4_propagate(arr.ctypes.data, len(arr), t.ctypes.data, len(t), out.ctypes.data,
                                  err.ctypes.data)
        if rc != 0:
            _raise(L, rc)
    return out, err
