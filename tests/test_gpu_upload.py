"""mzb_pj_create_async: trajectories uploaded by time chunk while the
screening runs batch by batch (gathered by a kernel from pinned memory,
packed by host threads for the copy engine from pageable memory) give
exactly the results of the synchronous upload (every output byte), for even
and odd orders + 1 (padded rows), with more chunks than batches and the
reverse, and with chunks larger than a staging piece (runs split across
pieces, inside one object's range too)."""

import ctypes as ct

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mizuba_b200 import _native

    return _native.core()


def _pinned(a):
    import torch

    t = torch.empty(max(a.nbytes, 1), dtype=torch.uint8, pin_memory=True)
    v = t.numpy()[: a.nbytes].view(a.dtype).reshape(a.shape)
    v[...] = a
    return t, v


def _create(L, a, fn, traj, *extra):
    h = ct.c_void_p()
    rc = getattr(L, fn)(traj.ctypes.data, a["traj"].size, a["traj_offsets"].ctypes.data, a["time"].ctypes.data,
                        a["time"].size, a["time_offsets"].ctypes.data, a["n_objs"], a["order"], a["maxT"], *extra,
                        ct.byref(h))
    assert rc == 0, L.mzb_last_error()
    return h


def _outputs(L, pj_h, thresh, interval, spb, form):
    from mizuba_b200 import _native

    opts = _native.MzbOpts()
    opts.steps_per_batch = spb
    opts.form = form
    h = ct.c_void_p()
    assert L.mzb_conjunctions(pj_h, thresh, interval, None, ct.byref(opts), ct.byref(h)) == 0, L.mzb_last_error()
    S, N = int(L.mzb_result_n_cd_steps(h)), int(L.mzb_result_n_objs(h))
    out = {}
    for name, fn, nb in (("aabbs", "mzb_result_copy_aabbs", S * (N + 1) * 32),
                         ("srt_aabbs", "mzb_result_copy_srt_aabbs", S * (N + 1) * 32),
                         ("mcodes", "mzb_result_copy_mcodes", S * N * 8),
                         ("srt_mcodes", "mzb_result_copy_srt_mcodes", S * N * 8),
                         ("srt_idx", "mzb_result_copy_srt_idx", S * N * 4),
                         ("trees", "mzb_result_copy_trees", int(L.mzb_result_n_tree_nodes(h)) * 48),
                         ("bp", "mzb_result_copy_bp", int(L.mzb_result_n_bp(h)) * 8),
                         ("conj", "mzb_result_copy_conj", int(L.mzb_result_n_conj(h)) * 120)):
        buf = np.zeros(max(nb, 1), np.uint8)
        assert getattr(L, fn)(h, buf.ctypes.data) == 0, name
        out[name] = buf[:nb].tobytes()
    L.mzb_result_free(h)
    return out


def _cases():
    from mizuba_b200 import synth

    return [
        # order 3: 4 coefficients per row, no padding
        ("linear", lambda: cases.random_linear_pj(400, seed=31, box=20.0, speed=10.0), 1.0, 0.03, 0),
        # order 18: 19 coefficients, padded to 20 (mixed form)
        ("catalogue", lambda: synth.workload("c1_1k_1d", n_objs=400, span_days=0.1), 5.0, 3.0 / 1440.0, 1),
    ]


@pytest.mark.parametrize("chunks,spb", [(5, 4), (3, 16), (1, 0)])
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_async_upload_matches_sync(L, case, chunks, spb):
    _, make, thresh, interval, form = case
    a = make().arrays
    ref_h = _create(L, a, "mzb_pj_create", a["traj"])
    ref = _outputs(L, ref_h, thresh, interval, 0, form)
    L.mzb_pj_free(ref_h)
    keep, traj = _pinned(a["traj"])
    h = _create(L, a, "mzb_pj_create_async", traj, chunks)
    got = _outputs(L, h, thresh, interval, spb, form)
    assert L.mzb_pj_upload_wait(h) == 0
    L.mzb_pj_free(h)
    del keep
    for k in ref:
        assert got[k] == ref[k], k


def test_async_upload_pageable(L):
    a = cases.random_linear_pj(200, seed=5).arrays
    ref_h = _create(L, a, "mzb_pj_create", a["traj"])
    ref = _outputs(L, ref_h, 1.0, 0.05, 0, 0)
    L.mzb_pj_free(ref_h)
    # A pageable copy, kept alive until the upload has finished (the call
    # returns before the data is read).
    traj = np.array(a["traj"])
    h = _create(L, a, "mzb_pj_create_async", traj, 4)
    assert L.mzb_pj_upload_wait(h) == 0
    del traj
    got = _outputs(L, h, 1.0, 0.05, 3, 0)
    L.mzb_pj_free(h)
    assert got == ref


def test_state_eval_waits_for_async_upload(L):
    # State evaluation may need any segment: on a polyjectory still being
    # uploaded it must wait for every chunk and give the synchronous result.
    from mizuba_b200 import synth

    a = synth.workload("c1_1k_1d", n_objs=300, span_days=0.1).arrays
    tms = np.linspace(0.0, a["maxT"] * 0.999, 300)
    res = []
    for fn, traj, extra in (("mzb_pj_create", a["traj"], ()), ("mzb_pj_create_async", None, (7,))):
        keep = None
        if traj is None:
            keep, traj = _pinned(a["traj"])
        h = _create(L, a, fn, traj, *extra)
        out = np.zeros((a["n_objs"], 7))
        assert L.mzb_pj_state_eval(h, out.ctypes.data, out.shape[0], tms.ctypes.data, tms.size, None, -1) == 0, \
            L.mzb_last_error()
        L.mzb_pj_free(h)
        del keep
        res.append(out)
    assert res[0].tobytes() == res[1].tobytes()
    assert np.isfinite(res[0]).all()


def test_async_upload_splits_large_chunks(L):
    # Order 18 (1,064 bytes per segment; a 16 MB staging piece holds about
    # 15,700 segments): one object of 40,000 segments and small ones around
    # it, uploaded in one and in three chunks, against the synchronous
    # upload, by state evaluation at every segment's midpoint (bit for bit).
    rng = np.random.default_rng(7)
    order, nseg = 18, [5, 40000, 3, 17000, 1]
    trajs, times = [], []
    for ns in nseg:
        tm = np.linspace(0.0, 1.0, ns + 1)
        trajs.append(rng.normal(0, 1, (ns, order + 1, 7)))
        times.append(tm)
    traj = np.ascontiguousarray(np.concatenate(trajs).reshape(-1))
    per = (order + 1) * 7
    soff = np.cumsum([0] + nseg[:-1]) * per
    toff = np.cumsum([0] + [n + 1 for n in nseg[:-1]])
    a = {"traj": traj, "traj_offsets": np.ascontiguousarray(np.stack([soff, nseg], 1).astype(np.uint64)),
         "time": np.concatenate(times), "time_offsets": toff.astype(np.uint64), "n_objs": len(nseg),
         "order": order, "maxT": 1.0}
    mids = []
    for ns in nseg:
        mids.append((np.arange(ns) + 0.5) / ns)
    tms = np.unique(np.concatenate(mids))[::7]

    def evaluate(h):
        out = np.zeros((len(nseg), tms.size, 7))
        assert L.mzb_pj_state_meval(h, out.ctypes.data, out.shape[0], out.shape[1], tms.ctypes.data, 1, tms.size, 0,
                                    None, -1) == 0, L.mzb_last_error()
        return out

    ref_h = _create(L, a, "mzb_pj_create", a["traj"])
    ref = evaluate(ref_h)
    L.mzb_pj_free(ref_h)
    assert np.isfinite(ref).all()
    keep, pinned = _pinned(a["traj"])
    for chunks, traj_in in ((1, pinned), (3, pinned), (3, a["traj"])):
        h = _create(L, a, "mzb_pj_create_async", traj_in, chunks)
        got = evaluate(h)
        assert L.mzb_pj_upload_wait(h) == 0
        L.mzb_pj_free(h)
        assert got.tobytes() == ref.tobytes(), chunks
    del keep
