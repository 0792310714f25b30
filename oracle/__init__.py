"""CPU oracle for the conjunction-detection path (test infrastructure).

Loads ``oracle/_build/liboracle.so`` (the C++ restatement in ``oracle.cpp``)
through ctypes.  Only the test suite, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this package, always as the checker or
the timed CPU baseline, never as part of the product path.
"""

from __future__ import annotations

import ctypes as ct
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
_LIB = None

BVH_NODE = np.dtype(
    [("begin", "<u4"), ("end", "<u4"), ("left", "<i4"), ("right", "<i4"),
     ("lb", "<f4", (4,)), ("ub", "<f4", (4,))]
)
AABB_COLLISION = np.dtype([("i", "<u4"), ("j", "<u4")])
CONJ = np.dtype(
    [("i", "<u4"), ("j", "<u4"), ("tca", "<f8"), ("dca", "<f8"),
     ("ri", "<f8", (3,)), ("vi", "<f8", (3,)), ("rj", "<f8", (3,)), ("vj", "<f8", (3,))]
)


def _lib():
    global _LIB
    if _LIB is None:
        path = HERE / "_build" / "liboracle.so"
        if not path.exists():
            from . import build as _b

            _b.build()
        L = ct.CDLL(str(path))
        P = ct.c_void_p
        L.mzo_run.restype = ct.c_int
        L.mzo_run.argtypes = [P, P, P, P, ct.c_uint64, ct.c_uint32, ct.c_double, ct.c_double,
                              ct.c_double, P, ct.c_uint64, ct.c_uint64, ct.c_int,
                              ct.POINTER(ct.c_void_p)]
        L.mzo_last_error.restype = ct.c_char_p
        for name in ("mzo_n_cd_steps", "mzo_n_run", "mzo_conj_size"):
            getattr(L, name).restype = ct.c_uint64
            getattr(L, name).argtypes = [P]
        for name in ("mzo_bvh_size", "mzo_bp_size"):
            getattr(L, name).restype = ct.c_uint64
            getattr(L, name).argtypes = [P, ct.c_uint64]
        for name in ("mzo_aabbs", "mzo_srt_aabbs", "mzo_mcodes", "mzo_srt_mcodes", "mzo_srt_idx",
                     "mzo_cd_end_times", "mzo_conj"):
            getattr(L, name).restype = P
            getattr(L, name).argtypes = [P]
        for name in ("mzo_bvh", "mzo_bp"):
            getattr(L, name).restype = P
            getattr(L, name).argtypes = [P, ct.c_uint64]
        L.mzo_np_report.argtypes = [P, P]
        L.mzo_free.argtypes = [P]
        L.mzo_state_eval.restype = ct.c_int
        L.mzo_state_eval.argtypes = [P, P, P, P, ct.c_uint32, P, P, ct.c_uint64, P]
        L.mzo_validate_global_aabbs.restype = ct.c_int
        L.mzo_validate_global_aabbs.argtypes = [P, ct.c_uint64]
        L.mzo_verify_bvh_tree.restype = ct.c_int
        L.mzo_verify_bvh_tree.argtypes = [P, P, ct.c_uint64, P, ct.c_uint64]
        L.mzo_verify_broad_phase.restype = ct.c_int
        L.mzo_verify_broad_phase.argtypes = [P, ct.c_uint64, P, P, ct.c_uint64, ct.c_int,
                                             ct.POINTER(ct.c_uint64)]
        _LIB = L
    return _LIB


def _arr(ptr, dtype, count):
    if count == 0:
        return np.zeros(0, dtype=dtype)
    buf = (ct.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=count).copy()


def run(pj, conj_thresh, conj_det_interval, otypes=None, step_begin=0, step_end=None,
        n_threads=None):
    """Runs the oracle over conjunction steps [step_begin, step_end).

    ``pj`` is a ``mizuba_b200.polyjectory`` (only its flat arrays are read).
    Returns a dict with the reference outputs for the steps that ran.
    Raises ValueError with the reference's message on invalid input.
    """
    L = _lib()
    a = pj.arrays if hasattr(pj, "arrays") else pj
    if n_threads is None:
        n_threads = os.cpu_count() or 1
    if step_end is None:
        step_end = 2**63
    ot = None
    if otypes is not None:
        ot = np.ascontiguousarray(otypes, dtype=np.int32)
    h = ct.c_void_p()
    rc = L.mzo_run(a["traj"].ctypes.data, a["traj_offsets"].ctypes.data, a["time"].ctypes.data,
                   a["time_offsets"].ctypes.data, a["n_objs"], a["order"], a["maxT"],
                   float(conj_thresh), float(conj_det_interval),
                   None if ot is None else ot.ctypes.data, step_begin, step_end, n_threads,
                   ct.byref(h))
    if rc != 0:
        raise ValueError(L.mzo_last_error().decode())
    try:
        N = a["n_objs"]
        nr = L.mzo_n_run(h)
        out = {"n_cd_steps": L.mzo_n_cd_steps(h), "n_run": nr, "step_begin": step_begin}
        out["aabbs"] = _arr(L.mzo_aabbs(h), np.float32, nr * (N + 1) * 8).reshape(nr, N + 1, 2, 4)
        out["srt_aabbs"] = _arr(L.mzo_srt_aabbs(h), np.float32, nr * (N + 1) * 8).reshape(nr, N + 1, 2, 4)
        out["mcodes"] = _arr(L.mzo_mcodes(h), np.uint64, nr * N).reshape(nr, N)
        out["srt_mcodes"] = _arr(L.mzo_srt_mcodes(h), np.uint64, nr * N).reshape(nr, N)
        out["srt_idx"] = _arr(L.mzo_srt_idx(h), np.uint32, nr * N).reshape(nr, N)
        out["cd_end_times"] = _arr(L.mzo_cd_end_times(h), np.float64, nr)
        out["bvh"] = [_arr(L.mzo_bvh(h, s), BVH_NODE, L.mzo_bvh_size(h, s)) for s in range(nr)]
        out["bp"] = [_arr(L.mzo_bp(h, s), AABB_COLLISION, L.mzo_bp_size(h, s)) for s in range(nr)]
        out["conjunctions"] = _arr(L.mzo_conj(h), CONJ, L.mzo_conj_size(h))
        rep = (ct.c_ulonglong * 7)()
        L.mzo_np_report(h, ct.addressof(rep))
        out["np_report"] = tuple(int(x) for x in rep)
        return out
    finally:
        L.mzo_free(h)


def state_eval(pj, objs, tms):
    """States of objects ``objs[k]`` at times ``tms[k]`` (pj_eval_obj_state,
    mizuba/polyjectory.cpp:1092-1159): an array (len(objs), 7), NaN where an
    object has no data.  Raises ValueError on a non-finite time."""
    L = _lib()
    a = pj.arrays if hasattr(pj, "arrays") else pj
    objs = np.ascontiguousarray(objs, dtype=np.uint64).ravel()
    tms = np.ascontiguousarray(tms, dtype=np.float64).ravel()
    assert objs.shape == tms.shape
    out = np.empty((objs.shape[0], 7))
    rc = L.mzo_state_eval(a["traj"].ctypes.data, a["traj_offsets"].ctypes.data, a["time"].ctypes.data,
                          a["time_offsets"].ctypes.data, a["order"], objs.ctypes.data, tms.ctypes.data,
                          objs.shape[0], out.ctypes.data)
    if rc != 0:
        raise ValueError(L.mzo_last_error().decode())
    return out


def morton_ref(fields):
    """Encodes (k, 4) uint16 field values with mizuba's own Morton encoder.

    Returns None when ``oracle/_ref/morton_ref`` was not built (the reference
    tree is not mounted on this machine)."""
    exe = HERE / "_ref" / "morton_ref"
    if not exe.exists():
        return None
    f = np.asarray(fields, dtype=np.uint64).reshape(-1, 4)
    inp = "\n".join(" ".join(str(int(v)) for v in row) for row in f) + "\n"
    res = subprocess.run([str(exe)], input=inp.encode(), capture_output=True, check=True)
    return np.array([int(x) for x in res.stdout.split()], dtype=np.uint64)


# ---- The reference's debug verifiers (mizuba builds them into debug builds
# as assertions), as checks on one step's outputs from any implementation.

def validate_global_aabbs(aabbs_step):
    """Row n_objs of a step's ``aabbs`` ([n_objs + 1][2][4] float32) is the
    min/max of the object boxes (detect_conjunctions_aabbs.cpp:260-282).
    Raises AssertionError naming the failed check."""
    L = _lib()
    a = np.ascontiguousarray(aabbs_step, dtype=np.float32)
    if L.mzo_validate_global_aabbs(a.ctypes.data, a.shape[0] - 1) != 0:
        raise AssertionError(L.mzo_last_error().decode())


def verify_bvh_tree(srt_mcodes_step, srt_aabbs_step, tree):
    """Structure, ranges, split prefixes, breadth-first numbering and node
    boxes of one step's tree (detect_conjunctions_bvh.cpp:60-255)."""
    L = _lib()
    m = np.ascontiguousarray(srt_mcodes_step, dtype=np.uint64)
    a = np.ascontiguousarray(srt_aabbs_step, dtype=np.float32)
    t = np.ascontiguousarray(tree)
    assert t.dtype.itemsize == 48
    if L.mzo_verify_bvh_tree(m.ctypes.data, a.ctypes.data, m.shape[0], t.ctypes.data if len(t) else None,
                             len(t)) != 0:
        raise AssertionError(L.mzo_last_error().decode())


def verify_broad_phase(aabbs_step, pairs, otypes=None, n_threads=None):
    """Every pair of overlapping boxes (N^2 test, otype filter) is in the
    step's sorted, unique pair list (detect_conjunctions_broad_phase.cpp:
    50-137).  Returns the number of true box overlaps."""
    L = _lib()
    a = np.ascontiguousarray(aabbs_step, dtype=np.float32)
    n = a.shape[0] - 1
    p = np.ascontiguousarray(pairs)
    ot = None if otypes is None else np.ascontiguousarray(otypes, dtype=np.int32)
    cnt = ct.c_uint64(0)
    rc = L.mzo_verify_broad_phase(a.ctypes.data, n, None if ot is None else ot.ctypes.data,
                                  p.ctypes.data if len(p) else None, len(p), n_threads or os.cpu_count() or 1,
                                  ct.byref(cnt))
    if rc != 0:
        raise AssertionError(L.mzo_last_error().decode())
    return int(cnt.value)


# ---- SGP4: the reference's own propagator compiled in place
# (oracle/_ref/libsgp4_ref.so, from mizuba/detail/sgp4) and the CPU
# restatement of make_sgp4_polyjectory driven by it.

_SGP4_REF = None


def sgp4_ref_lib():
    """The reference's SGP4 propagator, or None where it was not built (the
    reference tree was absent when the checkers were built)."""
    global _SGP4_REF
    if _SGP4_REF is None:
        path = HERE / "_ref" / "libsgp4_ref.so"
        if not path.exists():
            return None
        L = ct.CDLL(str(path))
        P = ct.c_void_p
        d = ct.c_double
        L.mzr_sgp4.argtypes = [P] * 8 + [ct.c_uint64, P, ct.c_uint64, P, P]
        L.mzr_sgp4_is_deep_space.restype = ct.c_int
        L.mzr_sgp4_is_deep_space.argtypes = [d] * 8
        L.mzr_sgp4_new.restype = P
        L.mzr_sgp4_new.argtypes = [d] * 8 + [P, P]
        L.mzr_sgp4_at.restype = ct.c_int
        L.mzr_sgp4_at.argtypes = [P, d, P, P]
        L.mzr_sgp4_delete.argtypes = [P]
        _SGP4_REF = L
    return _SGP4_REF


def _epoch_1950(gpes):
    """Days from 1950 Jan 0.0 as sgp4init takes them: the double-length epoch
    minus 2433281.5, rounded to a double (make_sgp4_polyjectory.cpp:719-745)."""
    hi = gpes["epoch_jd1"] + gpes["epoch_jd2"]
    lo = gpes["epoch_jd2"] - (hi - gpes["epoch_jd1"])
    return (hi - 2433281.5) + lo


def sgp4_ref(gpes, tsince):
    """The reference propagator: states [n][t][6] (km, km/s) and error codes
    [n][t] of each element set at tsince minutes from its epoch."""
    L = sgp4_ref_lib()
    g = np.ascontiguousarray(gpes)
    t = np.ascontiguousarray(tsince, dtype=np.float64).ravel()
    out = np.zeros((len(g), len(t), 6))
    err = np.zeros((len(g), len(t)), dtype=np.int32)
    cols = [np.ascontiguousarray(_epoch_1950(g))] + [np.ascontiguousarray(g[f], dtype=np.float64)
                                                     for f in ("n0", "e0", "i0", "node0", "omega0", "m0", "bstar")]
    L.mzr_sgp4(*[c.ctypes.data for c in cols], len(g), t.ctypes.data, len(t), out.ctypes.data, err.ctypes.data)
    return out, err


def sgp4_ref_is_deep_space(gpes):
    L = sgp4_ref_lib()
    ep = _epoch_1950(gpes)
    return np.array([bool(L.mzr_sgp4_is_deep_space(float(ep[k]), *(float(gpes[f][k]) for f in
                     ("n0", "e0", "i0", "node0", "omega0", "m0", "bstar")))) for k in range(len(gpes))])


def sgp4_polyjectory(gpes, jd_begin, jd_end, reentry_radius=0.0, exit_radius=float("inf")):
    """CPU restatement of make_sgp4_polyjectory on the reference propagator:
    dict with traj, traj_offsets, time, time_offsets, status, epoch (hi, lo).
    Returns None when the reference propagator was not built."""
    R = sgp4_ref_lib()
    if R is None:
        return None
    L = _lib()
    P = ct.c_void_p
    if not getattr(L, "_sgp4_set", False):
        L.mzo_sgp4_polyjectory.restype = ct.c_int
        L.mzo_sgp4_polyjectory.argtypes = [P, ct.c_uint64, ct.c_double, ct.c_double, ct.c_double, ct.c_double,
                                           P, P, P, ct.POINTER(ct.c_void_p)]
        L.mzo_sgp4_last_error.restype = ct.c_char_p
        for nm in ("mzo_sgp4_pj_n_objs", "mzo_sgp4_pj_traj_size", "mzo_sgp4_pj_time_size"):
            getattr(L, nm).restype = ct.c_uint64
            getattr(L, nm).argtypes = [P]
        L.mzo_sgp4_pj_copy.argtypes = [P] * 7
        L.mzo_sgp4_pj_free.argtypes = [P]
        L._sgp4_set = True
    g = np.ascontiguousarray(gpes)
    fn = [ct.cast(getattr(R, nm), P).value for nm in ("mzr_sgp4_new", "mzr_sgp4_at", "mzr_sgp4_delete")]
    h = ct.c_void_p()
    rc = L.mzo_sgp4_polyjectory(g.ctypes.data, len(g), float(jd_begin), float(jd_end), float(reentry_radius),
                                float(exit_radius), *fn, ct.byref(h))
    if rc != 0:
        raise ValueError(L.mzo_sgp4_last_error().decode())
    try:
        n = L.mzo_sgp4_pj_n_objs(h)
        out = {"traj": np.empty(L.mzo_sgp4_pj_traj_size(h)), "traj_offsets": np.empty((n, 2), dtype=np.uint64),
               "time": np.empty(L.mzo_sgp4_pj_time_size(h)), "time_offsets": np.empty(n, dtype=np.uint64),
               "status": np.empty(n, dtype=np.int32), "epoch": np.empty(2)}
        L.mzo_sgp4_pj_copy(h, out["traj"].ctypes.data, out["traj_offsets"].ctypes.data, out["time"].ctypes.data,
                           out["time_offsets"].ctypes.data, out["status"].ctypes.data, out["epoch"].ctypes.data)
    finally:
        L.mzo_sgp4_pj_free(h)
    return out
