"""ctypes bindings of the in-tree native libraries."""

from __future__ import annotations

import ctypes as ct
import threading

from . import build as _build

_lock = threading.Lock()
_PJGEN = None
_CORE = None


def pjgen():
    global _PJGEN
    with _lock:
        if _PJGEN is None:
            path = _build.LIB / "libmzb_pjgen.so"
            if not path.exists():
                _build.build_pjgen()
            L = ct.CDLL(str(path))
            P = ct.c_void_p
            L.mzb_pjgen_build.restype = P
            L.mzb_pjgen_build.argtypes = [P, ct.c_uint64, ct.c_double, ct.c_double, ct.c_uint32, ct.c_int]
            for nm in ("mzb_pjgen_traj_size", "mzb_pjgen_time_size"):
                getattr(L, nm).restype = ct.c_uint64
                getattr(L, nm).argtypes = [P]
            for nm in ("mzb_pjgen_traj", "mzb_pjgen_time", "mzb_pjgen_traj_off",
                       "mzb_pjgen_time_off", "mzb_pjgen_status"):
                getattr(L, nm).restype = P
                getattr(L, nm).argtypes = [P]
            for nm in ("mzb_pjgen_max_err", "mzb_pjgen_maxT"):
                getattr(L, nm).restype = ct.c_double
                getattr(L, nm).argtypes = [P]
            L.mzb_pjgen_free.argtypes = [P]
            _PJGEN = L
    return _PJGEN


def core():
    """The CUDA library (libmizuba_b200.so).  Raises if it is not built:
    there is no CPU fallback for the screening path."""
    global _CORE
    with _lock:
        if _CORE is None:
            path = _build.LIB / "libmizuba_b200.so"
            if not path.exists():
                raise RuntimeError(
                    f"{path} is missing: build it with `python -m mizuba_b200.build` "
                    "(the conjunction screen runs only on the CUDA path)"
                )
            L = ct.CDLL(str(path))
            P = ct.c_void_p
            u64 = ct.c_uint64
            L.mzb_last_error.restype = ct.c_char_p
            L.mzb_pj_create.restype = ct.c_int
            L.mzb_pj_create.argtypes = [P, u64, P, P, u64, P, u64, ct.c_uint32, ct.c_double,
                                        ct.POINTER(ct.c_void_p)]
            L.mzb_pj_free.argtypes = [P]
            L.mzb_pj_create_async.restype = ct.c_int
            L.mzb_pj_create_async.argtypes = [P, u64, P, P, u64, P, u64, ct.c_uint32, ct.c_double, ct.c_uint32,
                                              ct.POINTER(ct.c_void_p)]
            L.mzb_pj_upload_wait.restype = ct.c_int
            L.mzb_pj_upload_wait.argtypes = [P]
            L.mzb_conjunctions.restype = ct.c_int
            L.mzb_conjunctions.argtypes = [P, ct.c_double, ct.c_double, P, P, ct.POINTER(ct.c_void_p)]
            L.mzb_conjunctions_stream.restype = ct.c_int
            L.mzb_conjunctions_stream.argtypes = [P, ct.c_double, ct.c_double, P, P, P, ct.POINTER(ct.c_void_p)]
            L.mzb_result_free.argtypes = [P]
            for nm in ("mzb_result_n_cd_steps", "mzb_result_n_objs", "mzb_result_n_tree_nodes",
                       "mzb_result_n_bp", "mzb_result_n_conj", "mzb_result_step_begin",
                       "mzb_result_n_steps_run", "mzb_result_n_launches", "mzb_result_broad_visits"):
                getattr(L, nm).restype = u64
                getattr(L, nm).argtypes = [P]
            for nm in ("mzb_result_copy_aabbs", "mzb_result_copy_srt_aabbs", "mzb_result_copy_mcodes",
                       "mzb_result_copy_srt_mcodes", "mzb_result_copy_srt_idx",
                       "mzb_result_copy_cd_end_times", "mzb_result_tree_offsets",
                       "mzb_result_copy_trees", "mzb_result_bp_offsets", "mzb_result_copy_bp",
                       "mzb_result_copy_conj"):
                getattr(L, nm).restype = ct.c_int
                getattr(L, nm).argtypes = [P, P]
            L.mzb_measure_fp64_rate.restype = ct.c_int
            L.mzb_measure_fp64_rate.argtypes = [P]
            L.mzb_scratch_release.restype = ct.c_int
            L.mzb_scratch_release.argtypes = []
            L.mzb_scratch_bytes.restype = ct.c_uint64
            L.mzb_scratch_bytes.argtypes = []
            L.mzb_result_write_files.restype = ct.c_int
            L.mzb_result_write_files.argtypes = [P, ct.c_char_p]
            L.mzb_pj_state_eval.restype = ct.c_int
            L.mzb_pj_state_eval.argtypes = [P, P, u64, P, ct.c_int64, P, ct.c_int64]
            L.mzb_pj_state_meval.restype = ct.c_int
            L.mzb_pj_state_meval.argtypes = [P, P, u64, u64, P, ct.c_uint32, u64, u64, P, ct.c_int64]
            L.mzb_result_np_report.argtypes = [P, P]
            L.mzb_result_narrow_split.argtypes = [P, P]
            L.mzb_result_stage_ms.argtypes = [P, P]
            L.mzb_make_sgp4_polyjectory.restype = ct.c_int
            L.mzb_make_sgp4_polyjectory.argtypes = [P, u64, ct.c_double, ct.c_double, ct.c_double, ct.c_double,
                                                    ct.POINTER(ct.c_void_p)]
            L.mzb_sgp4_pj_sizes.argtypes = [P, P]
            L.mzb_sgp4_pj_epoch.argtypes = [P, P]
            L.mzb_sgp4_pj_copy.restype = ct.c_int
            L.mzb_sgp4_pj_copy.argtypes = [P, P, P, P, P, P]
            L.mzb_sgp4_pj_free.argtypes = [P]
            L.mzb_sgp4_pj_timing.argtypes = [P, P]
            L.mzb_sgp4_propagate.restype = ct.c_int
            L.mzb_sgp4_propagate.argtypes = [P, u64, P, u64, P, P]
            _CORE = L
    return _CORE


class MzbOpts(ct.Structure):
    _fields_ = [("steps_per_batch", ct.c_uint32), ("form", ct.c_uint32),
                ("step_begin", ct.c_uint64), ("step_end", ct.c_uint64),
                ("bvh_threads", ct.c_uint32), ("broad_walk", ct.c_uint32),
                ("sort_threads", ct.c_uint32), ("reserved", ct.c_uint32)]


class MzbHostOutputs(ct.Structure):
    _fields_ = [("aabbs", ct.c_void_p), ("srt_aabbs", ct.c_void_p), ("mcodes", ct.c_void_p),
                ("srt_mcodes", ct.c_void_p), ("srt_idx", ct.c_void_p), ("cd_end_times", ct.c_void_p),
                ("trees", ct.c_void_p), ("trees_cap", ct.c_uint64)]
