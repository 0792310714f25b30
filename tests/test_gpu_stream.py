"""mzb_conjunctions_stream: the per-step arrays and trees streamed to host
memory during the screening equal the result's own copies (several batches,
a shard of the time axis) and an undersized tree buffer is refused."""

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


def _run(L, pj, thresh, interval, steps_per_batch=0, step_range=None, trees_cap=None, form=0):
    from mizuba_b200 import _native, to_device

    dev = to_device(pj)
    opts = _native.MzbOpts()
    opts.steps_per_batch = steps_per_batch
    opts.form = form
    if step_range:
        opts.step_begin, opts.step_end = step_range
    n_cd = int(np.ceil(pj.maxT / interval))
    S = (step_range[1] - step_range[0]) if step_range else n_cd
    N = pj.n_objs
    out = {"aabbs": np.zeros((S, N + 1, 2, 4), np.float32), "srt_aabbs": np.zeros((S, N + 1, 2, 4), np.float32),
           "mcodes": np.zeros((S, N), np.uint64), "srt_mcodes": np.zeros((S, N), np.uint64),
           "srt_idx": np.zeros((S, N), np.uint32), "cd_end_times": np.zeros(S)}
    cap = S * (2 * N - 1) if trees_cap is None else trees_cap
    trees = np.zeros(max(cap, 1) * 48, np.uint8)
    dst = _native.MzbHostOutputs()
    for k, v in out.items():
        setattr(dst, k, v.ctypes.data)
    dst.trees, dst.trees_cap = trees.ctypes.data, cap
    h = ct.c_void_p()
    rc = L.mzb_conjunctions_stream(dev._h, thresh, interval, None, ct.byref(opts), ct.byref(dst), ct.byref(h))
    return rc, h, out, trees


def _check(L, h, out, trees):
    S, N = out["mcodes"].shape
    for k, fn in (("aabbs", "mzb_result_copy_aabbs"), ("srt_aabbs", "mzb_result_copy_srt_aabbs"),
                  ("mcodes", "mzb_result_copy_mcodes"), ("srt_mcodes", "mzb_result_copy_srt_mcodes"),
                  ("srt_idx", "mzb_result_copy_srt_idx"), ("cd_end_times", "mzb_result_copy_cd_end_times")):
        ref = np.zeros_like(out[k])
        assert getattr(L, fn)(h, ref.ctypes.data) == 0
        assert ref.tobytes() == out[k].tobytes(), k
    nt = int(L.mzb_result_n_tree_nodes(h))
    ref = np.zeros(nt * 48, np.uint8)
    assert L.mzb_result_copy_trees(h, ref.ctypes.data) == 0
    assert ref.tobytes() == trees[:nt * 48].tobytes()
    L.mzb_result_free(h)


@pytest.mark.parametrize("spb", [0, 7])
def test_stream_matches_copies(L, spb):
    pj = cases.random_linear_pj(300, seed=13, box=20.0, speed=10.0)
    rc, h, out, trees = _run(L, pj, 1.0, 0.03, steps_per_batch=spb)
    assert rc == 0, L.mzb_last_error()
    _check(L, h, out, trees)


def test_stream_shard_and_mixed(L):
    pj = cases.clustered_pj(6)
    rc, h, out, trees = _run(L, pj, 0.5, 0.05, steps_per_batch=5, step_range=(3, 14), form=1)
    assert rc == 0, L.mzb_last_error()
    _check(L, h, out, trees)


def test_stream_refuses_small_tree_buffer(L):
    pj = cases.random_linear_pj(100, seed=2)
    rc, h, out, trees = _run(L, pj, 1.0, 0.05, trees_cap=10)
    assert rc == 1 and b"nodes of the destination buffer" in L.mzb_last_error()


def test_reserved_option_must_be_zero(L):
    from mizuba_b200 import _native, to_device

    dev = to_device(cases.random_linear_pj(50, seed=3))
    opts = _native.MzbOpts()
    opts.reserved = 1
    h = ct.c_void_p()
    rc = L.mzb_conjunctions(dev._h, 1.0, 0.05, None, ct.byref(opts), ct.byref(h))
    assert rc == 1 and "reserved must be 0" in L.mzb_last_error().decode()
