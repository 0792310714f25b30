"""``conjunctions``: the drop-in for ``mizuba.conjunctions``.

Same constructor (``pj, conj_thresh, conj_det_interval, otypes=None,
data_dir=None, tmpdir=None``; mizuba/expose_conjunctions.cpp:83-101), same
argument checks and messages (mizuba/conjunctions.cpp:263-332), same
read-only properties and accessors (mizuba/expose_conjunctions.cpp:99-203):
``n_cd_steps``, ``aabbs``, ``cd_end_times``, ``srt_aabbs``, ``mcodes``,
``srt_mcodes``, ``srt_idx``, ``get_bvh_tree(i)``, ``get_aabb_collisions(i)``,
``conjunctions``, ``otypes``, ``conj_thresh``, ``conj_det_interval``,
``hint_release()`` and the ``bvh_node`` / ``aabb_collision`` / ``conj``
dtypes.  The computation runs on the GPU through the C ABI of
``libmizuba_b200.so``.

As in mizuba, the results live in files of a private data directory (the
user's ``data_dir``, or a fresh ``mizuba_conjunctions-XXXX-XXXX-XXXX-XXXX``
directory under ``tmpdir``, the global temporary directory of
``set_tmpdir`` / ``MIZUBA_TMPDIR``, or the system's), written by the library
straight from HBM, and the accessors return read-only views of the
memory-mapped files.  The directory is removed when the object and every
array taken from it are gone (mizuba/conjunctions.cpp:70-247).

``device_conjunctions`` is the same computation with the results left in HBM
and copied to host arrays on first access (no files).
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _native
from ._files import DataDir, MappedFile, create_data_dir, get_tmpdir, set_tmpdir  # noqa: F401
from .polyjectory import polyjectory

BVH_NODE = np.dtype(
    [("begin", "<u4"), ("end", "<u4"), ("left", "<i4"), ("right", "<i4"),
     ("lb", "<f4", (4,)), ("ub", "<f4", (4,))]
)
AABB_COLLISION = np.dtype([("i", "<u4"), ("j", "<u4")])
CONJ = np.dtype(
    [("i", "<u4"), ("j", "<u4"), ("tca", "<f8"), ("dca", "<f8"),
     ("ri", "<f8", (3,)), ("vi", "<f8", (3,)), ("rj", "<f8", (3,)), ("vj", "<f8", (3,))]
)


def _raise(L, rc):
    msg = L.mzb_last_error().decode()
    if rc == 1:
        raise ValueError(msg)
    if rc == 2:
        raise IndexError(msg)
    raise RuntimeError(msg)


class device_polyjectory:
    """A polyjectory uploaded to HBM (``mzb_pj_create``)."""

    def __init__(self, pj: polyjectory):
        L = _native.core()
        a = pj.arrays
        h = ct.c_void_p()
        rc = L.mzb_pj_create(a["traj"].ctypes.data, a["traj"].size, a["traj_offsets"].ctypes.data,
                             a["time"].ctypes.data, a["time"].size, a["time_offsets"].ctypes.data,
                             a["n_objs"], a["order"], a["maxT"], ct.byref(h))
        if rc != 0:
            _raise(L, rc)
        self._h = h
        self._L = L
        self.n_objs = a["n_objs"]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.mzb_pj_free(h)
            self._h = None


def release_scratch() -> None:
    """Returns the batch scratch that screening calls keep cached on the
    current CUDA device (sized by the largest call so far) to the driver's
    stream-ordered pool.  Waits for a call in progress on the device."""
    L = _native.core()
    rc = L.mzb_scratch_release()
    if rc:
        _raise(L, rc)


def scratch_bytes() -> int:
    """Bytes of batch scratch cached on the current CUDA device."""
    return int(_native.core().mzb_scratch_bytes())


def to_device(pj: polyjectory) -> device_polyjectory:
    dev = getattr(pj, "_device", None)
    if dev is None:
        dev = device_polyjectory(pj)
        pj._device = dev
    return dev


class device_conjunctions:
    """Conjunction screening with the results left in HBM: the arrays are
    copied to the host on first access.  Same arguments as ``conjunctions``
    except the data directory ones."""

    bvh_node = BVH_NODE
    aabb_collision = AABB_COLLISION
    conj = CONJ

    def __init__(self, pj, conj_thresh, conj_det_interval, otypes=None, steps_per_batch=0, step_range=None,
                 form="plain", tuning=None):
        n = pj.n_objs
        ot = None
        if otypes is not None:
            ot = np.ascontiguousarray(otypes, dtype=np.int32).reshape(-1)
            if ot.shape[0] != n:
                raise ValueError(
                    "Invalid array of object types passed to the constructor of a conjunctions "
                    f"objects: the expected size is {n}, but the actual size is {ot.shape[0]} instead"
                )
        L = _native.core()
        dev = to_device(pj) if isinstance(pj, polyjectory) else pj
        opts = _native.MzbOpts()
        opts.steps_per_batch = int(steps_per_batch)
        if form not in ("plain", "mixed"):
            raise ValueError(f"unknown screening form {form!r}: expected 'plain' or 'mixed'")
        opts.form = 1 if form == "mixed" else 0
        opts.bvh_threads = int((tuning or {}).get("bvh_threads", 0))
        opts.broad_walk = int((tuning or {}).get("broad_walk", 0))
        opts.sort_threads = int((tuning or {}).get("sort_threads", 0))
        if step_range is not None:
            # A shard of the time axis: per-step outputs cover only these steps.
            opts.step_begin, opts.step_end = (int(x) for x in step_range)
        h = ct.c_void_p()
        rc = L.mzb_conjunctions(dev._h, float(conj_thresh), float(conj_det_interval),
                                None if ot is None else ot.ctypes.data, ct.byref(opts), ct.byref(h))
        if rc != 0:
            _raise(L, rc)
        self._L = L
        self._h = h
        self._n = n
        self._thresh = float(conj_thresh)
        self._interval = float(conj_det_interval)
        self._otypes = np.ones(n, dtype=np.int32) if ot is None else ot.copy()
        self._otypes.setflags(write=False)
        self._S_total = int(L.mzb_result_n_cd_steps(h))
        self._S = int(L.mzb_result_n_steps_run(h))
        self.step_begin = int(L.mzb_result_step_begin(h))
        self._cache = {}
        self._keepalive = dev

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.mzb_result_free(h)
            self._h = None

    # ------------------------------------------------------------ helpers
    def _fetch(self, key, fn, dtype, shape):
        arr = self._cache.get(key)
        if arr is None:
            arr = np.empty(shape, dtype=dtype)
            if arr.size:
                rc = getattr(self._L, fn)(self._h, arr.ctypes.data)
                if rc != 0:
                    _raise(self._L, rc)
            arr.setflags(write=False)
            self._cache[key] = arr
        return arr

    def _trees(self):
        if "trees" not in self._cache:
            os_ = np.empty((self._S, 2), dtype=np.uint64)
            self._L.mzb_result_tree_offsets(self._h, os_.ctypes.data)
            tot = int(os_[:, 1].sum())
            t = np.empty(tot, dtype=BVH_NODE)
            if tot:
                rc = self._L.mzb_result_copy_trees(self._h, t.ctypes.data)
                if rc != 0:
                    _raise(self._L, rc)
            t.setflags(write=False)
            self._cache["trees"] = (os_, t)
        return self._cache["trees"]

    def _bp(self):
        if "bp" not in self._cache:
            os_ = np.empty((self._S, 2), dtype=np.uint64)
            self._L.mzb_result_bp_offsets(self._h, os_.ctypes.data)
            tot = int(self._L.mzb_result_n_bp(self._h))
            b = np.empty(tot, dtype=AABB_COLLISION)
            if tot:
                rc = self._L.mzb_result_copy_bp(self._h, b.ctypes.data)
                if rc != 0:
                    _raise(self._L, rc)
            b.setflags(write=False)
            self._cache["bp"] = (os_, b)
        return self._cache["bp"]

    # ------------------------------------------------------ reference API
    @property
    def n_cd_steps(self):
        return self._S_total

    @property
    def aabbs(self):
        return self._fetch("aabbs", "mzb_result_copy_aabbs", np.float32, (self._S, self._n + 1, 2, 4))

    @property
    def srt_aabbs(self):
        return self._fetch("srt_aabbs", "mzb_result_copy_srt_aabbs", np.float32,
                           (self._S, self._n + 1, 2, 4))

    @property
    def mcodes(self):
        return self._fetch("mcodes", "mzb_result_copy_mcodes", np.uint64, (self._S, self._n))

    @property
    def srt_mcodes(self):
        return self._fetch("srt_mcodes", "mzb_result_copy_srt_mcodes", np.uint64, (self._S, self._n))

    @property
    def srt_idx(self):
        return self._fetch("srt_idx", "mzb_result_copy_srt_idx", np.uint32, (self._S, self._n))

    @property
    def cd_end_times(self):
        return self._fetch("cd_end_times", "mzb_result_copy_cd_end_times", np.float64, (self._S,))

    def get_bvh_tree(self, i):
        if i >= self._S:
            raise IndexError(
                f"Cannot fetch the BVH tree for the conjunction timestep at index {i}: the total "
                f"number of conjunction steps is only {self._S}"
            )
        os_, t = self._trees()
        o, s = int(os_[i, 0]), int(os_[i, 1])
        return t[o:o + s]

    def get_aabb_collisions(self, i):
        if i >= self._S:
            raise IndexError(
                f"Cannot fetch the list of AABB collisions for the conjunction timestep at index {i}: "
                f"the total number of conjunction steps is only {self._S}"
            )
        os_, b = self._bp()
        o, s = int(os_[i, 0]), int(os_[i, 1])
        return b[o:o + s]

    @property
    def conjunctions(self):
        n = int(self._L.mzb_result_n_conj(self._h))
        return self._fetch("conj", "mzb_result_copy_conj", CONJ, (n,))

    @property
    def otypes(self):
        return self._otypes

    @property
    def conj_thresh(self):
        return self._thresh

    @property
    def conj_det_interval(self):
        return self._interval

    def hint_release(self):
        self._cache.clear()

    # ------------------------------------------------------------- extras
    @property
    def np_report(self):
        out = (ct.c_uint64 * 7)()
        self._L.mzb_result_np_report(self._h, ct.addressof(out))
        return tuple(int(x) for x in out)

    @property
    def narrow_split(self):
        """Mixed form: (items past the distance screen, items past the FMA
        prefilter); zeros for the plain form."""
        out = (ct.c_uint64 * 2)()
        self._L.mzb_result_narrow_split(self._h, ct.addressof(out))
        return tuple(int(x) for x in out)

    @property
    def n_launches(self):
        return int(self._L.mzb_result_n_launches(self._h))

    @property
    def broad_visits(self):
        """Tree-node visits of the broad-phase walk (default walk only)."""
        return int(self._L.mzb_result_broad_visits(self._h))

    @property
    def stage_ms(self):
        out = (ct.c_double * 8)()
        self._L.mzb_result_stage_ms(self._h, ct.addressof(out))
        keys = ("aabb", "morton_sort", "bvh", "broad", "narrow", "roots", "conj_sort", "total")
        return dict(zip(keys, (float(x) for x in out)))

_FILES = ("aabbs", "srt_aabbs", "mcodes", "srt_mcodes", "vidx", "bvh", "bp", "conjunctions")


class conjunctions:
    """Conjunction screening of a polyjectory (the drop-in for
    ``mizuba.conjunctions``).  ``steps_per_batch``, ``step_range`` (a shard of
    the time axis) and ``form`` ("plain": the reference's FP64 arithmetic;
    "mixed": enclosing boxes and an FP64 prefilter with the same conjunction
    records) are extensions."""

    bvh_node = BVH_NODE
    aabb_collision = AABB_COLLISION
    conj = CONJ

    def __init__(self, pj, conj_thresh, conj_det_interval, otypes=None, data_dir=None, tmpdir=None,
                 steps_per_batch=0, step_range=None, form="plain", tuning=None):
        if data_dir is not None and tmpdir is not None:
            raise ValueError(
                "The 'data_dir' and 'tmpdir' construction arguments cannot be provided at the same time"
            )
        d = device_conjunctions(pj, conj_thresh, conj_det_interval, otypes=otypes,
                                steps_per_batch=steps_per_batch, step_range=step_range, form=form, tuning=tuning)
        L = d._L
        path = create_data_dir(data_dir, tmpdir, "mizuba_conjunctions")
        owner = DataDir(path)
        rc = L.mzb_result_write_files(d._h, path.encode())
        if rc != 0:
            _raise(L, rc)
        S, N = d._S, d._n
        self._n = N
        self._S = S
        self._S_total = d._S_total
        self.step_begin = d.step_begin
        self._thresh = d._thresh
        self._interval = d._interval
        self._otypes = d._otypes
        self._np_report = d.np_report
        self._narrow_split = d.narrow_split
        self._n_launches = d.n_launches
        self._stage_ms = d.stage_ms
        self._cd_end = d.cd_end_times
        tos = np.empty((S, 2), dtype=np.uint64)
        L.mzb_result_tree_offsets(d._h, tos.ctypes.data)
        bos = np.empty((S, 2), dtype=np.uint64)
        L.mzb_result_bp_offsets(d._h, bos.ctypes.data)
        n_bp = int(L.mzb_result_n_bp(d._h))
        n_conj = int(L.mzb_result_n_conj(d._h))
        del d  # the device result is released: from here on the files hold the data
        self._tree_off, self._bp_off = tos, bos
        self._dir = owner
        self._files = {nm: MappedFile(owner, nm) for nm in _FILES}
        f = self._files
        self._aabbs = f["aabbs"].array(np.float32, S * (N + 1) * 8, (S, N + 1, 2, 4))
        self._srt_aabbs = f["srt_aabbs"].array(np.float32, S * (N + 1) * 8, (S, N + 1, 2, 4))
        self._mcodes = f["mcodes"].array(np.uint64, S * N, (S, N))
        self._srt_mcodes = f["srt_mcodes"].array(np.uint64, S * N, (S, N))
        self._srt_idx = f["vidx"].array(np.uint32, S * N, (S, N))
        self._trees = f["bvh"].array(BVH_NODE, int(tos[:, 1].sum()) if S else 0)
        self._bp = f["bp"].array(AABB_COLLISION, n_bp)
        # A single byte in the conjunctions file means none (conjunctions.cpp:204-213).
        self._conj = f["conjunctions"].array(CONJ, n_conj if f["conjunctions"].size > 1 else 0)

    # ------------------------------------------------------ reference API
    @property
    def n_cd_steps(self):
        return self._S_total

    @property
    def aabbs(self):
        return self._aabbs

    @property
    def srt_aabbs(self):
        return self._srt_aabbs

    @property
    def mcodes(self):
        return self._mcodes

    @property
    def srt_mcodes(self):
        return self._srt_mcodes

    @property
    def srt_idx(self):
        return self._srt_idx

    @property
    def cd_end_times(self):
        return self._cd_end

    def get_bvh_tree(self, i):
        if i >= self._S:
            raise IndexError(
                f"Cannot fetch the BVH tree for the conjunction timestep at index {i}: the total "
                f"number of conjunction steps is only {self._S}"
            )
        o, s = int(self._tree_off[i, 0]), int(self._tree_off[i, 1])
        return self._trees[o:o + s]

    def get_aabb_collisions(self, i):
        if i >= self._S:
            raise IndexError(
                f"Cannot fetch the list of AABB collisions for the conjunction timestep at index {i}: "
                f"the total number of conjunction steps is only {self._S}"
            )
        o, s = int(self._bp_off[i, 0]), int(self._bp_off[i, 1])
        return self._bp[o:o + s]

    @property
    def conjunctions(self):
        return self._conj

    @property
    def otypes(self):
        return self._otypes

    @property
    def conj_thresh(self):
        return self._thresh

    @property
    def conj_det_interval(self):
        return self._interval

    def hint_release(self):
        """Tells the OS that the mapped files' pages may be dropped
        (conjunctions::hint_release, mizuba/conjunctions.cpp:466-476)."""
        for f in self._files.values():
            f.advise_dontneed()

    # ------------------------------------------------------------- extras
    @property
    def data_dir(self):
        return self._dir.path

    @property
    def np_report(self):
        return self._np_report

    @property
    def narrow_split(self):
        return self._narrow_split

    @property
    def n_launches(self):
        return self._n_launches

    @property
    def stage_ms(self):
        return dict(self._stage_ms)
