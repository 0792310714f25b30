"""The allocation-free step sort (mzb_sort_step_noalloc), called through the
C ABI (needs a B200).

The no-alloc entry point serves callers that cannot allocate device memory
where they sort (hosts whose own allocator owns all device memory, or
allocation-free hot loops); its scratch is a fixed array inside the library.
It is checked against the oracle's sort order and gathers, on consecutive
calls (the shared scratch keeps the previous call's contents), on steps with
no-data boxes, at exactly the documented maximum of 524,288 objects, and for
allocating nothing.  This file is collected last so that a failure here
leaves every other test already run.
"""

import ctypes as ct

import numpy as np
import pytest

import cases
import oracle

pytestmark = pytest.mark.gpu

MAX_OBJS = 524288


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mizuba_b200 import _native

    L = _native.core()
    L.mzb_sort_step_noalloc.restype = ct.c_int
    L.mzb_sort_step_noalloc.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_uint64, ct.c_void_p, ct.c_void_p,
                                        ct.c_void_p, ct.c_void_p]
    return L, torch


def sort_on_gpu(L, torch, aabbs, mcodes):
    """One step through mzb_sort_step_noalloc; returns the three outputs."""
    n = mcodes.shape[0]
    dev = torch.device("cuda", 0)
    a = torch.from_numpy(np.ascontiguousarray(aabbs, dtype=np.float32)).to(dev)
    m = torch.from_numpy(np.ascontiguousarray(mcodes, dtype=np.uint64).view(np.int64)).to(dev)
    o_idx = torch.empty(n, dtype=torch.int32, device=dev)
    o_mc = torch.empty(n, dtype=torch.int64, device=dev)
    o_ab = torch.empty((n + 1, 2, 4), dtype=torch.float32, device=dev)
    rc = L.mzb_sort_step_noalloc(a.data_ptr(), m.data_ptr(), n, o_idx.data_ptr(), o_mc.data_ptr(),
                                 o_ab.data_ptr(), None)
    assert rc == 0, L.mzb_last_error().decode()
    torch.cuda.synchronize()
    return (o_idx.cpu().numpy().view(np.uint32), o_mc.cpu().numpy().view(np.uint64), o_ab.cpu().numpy())


def test_matches_oracle_on_consecutive_calls(env):
    L, torch = env
    # Ragged random trajectories: late starts, early ends and empty objects
    # give steps with no-data (infinite) boxes, which sort last.
    pj = cases.random_linear_pj(700, seed=11, box=30.0, speed=20.0)
    r = oracle.run(pj, 1.0, 0.05)
    steps = [k for k in range(r["n_run"]) if np.isinf(r["aabbs"][k, :-1, 0, 0]).any()]
    assert len(steps) >= 2
    # Two calls in a row on different steps, then the first step again.
    for k in (steps[0], steps[-1], steps[0]):
        idx, mc, ab = sort_on_gpu(L, torch, r["aabbs"][k], r["mcodes"][k])
        assert np.array_equal(idx, r["srt_idx"][k])
        assert np.array_equal(mc, r["srt_mcodes"][k])
        assert np.array_equal(ab.view(np.uint32), r["srt_aabbs"][k].view(np.uint32))


def test_at_the_documented_maximum(env):
    L, torch = env
    rng = np.random.default_rng(5)
    n = MAX_OBJS
    lb = rng.uniform(-1e4, 1e4, (n, 4)).astype(np.float32)
    ab = np.empty((n + 1, 2, 4), dtype=np.float32)
    ab[:n, 0] = lb
    ab[:n, 1] = lb + 1.0
    # No-data boxes (as the AABB stage writes them) and their all-ones codes.
    nodata = rng.random(n) < 0.03
    ab[np.nonzero(nodata)[0], 0] = np.inf
    ab[np.nonzero(nodata)[0], 1] = -np.inf
    ab[n, 0] = ab[:n][~nodata, 0].min(axis=0)
    ab[n, 1] = ab[:n][~nodata, 1].max(axis=0)
    # Codes with many ties (ties are ordered by index).
    mc = rng.integers(0, 1 << 20, n, dtype=np.uint64) * np.uint64(0x9E3779B97F4)
    mc[nodata] = np.uint64(2**64 - 1)
    want = np.lexsort((np.arange(n), mc, nodata)).astype(np.uint32)
    idx, smc, sab = sort_on_gpu(L, torch, ab, mc)
    assert np.array_equal(idx, want)
    assert np.array_equal(smc, mc[want])
    assert np.array_equal(sab[:n].view(np.uint32), ab[want].view(np.uint32))
    assert np.array_equal(sab[n].view(np.uint32), ab[n].view(np.uint32))
    # One past the maximum is refused with a clear error.
    t = torch.empty(8, device=torch.device("cuda", 0))
    rc = L.mzb_sort_step_noalloc(t.data_ptr(), t.data_ptr(), n + 1, t.data_ptr(), t.data_ptr(), t.data_ptr(), None)
    assert rc == 1 and b"exceed the capacity" in L.mzb_last_error()


def test_allocates_nothing(env):
    L, torch = env
    pj = cases.random_linear_pj(400, seed=3, box=30.0, speed=20.0)
    r = oracle.run(pj, 1.0, 0.05, step_begin=0, step_end=2)
    dev = torch.device("cuda", 0)
    n = pj.n_objs
    a = torch.from_numpy(np.ascontiguousarray(r["aabbs"][1])).to(dev)
    m = torch.from_numpy(r["mcodes"][1].view(np.int64).copy()).to(dev)
    outs = [torch.empty(n, dtype=torch.int32, device=dev), torch.empty(n, dtype=torch.int64, device=dev),
            torch.empty((n + 1, 2, 4), dtype=torch.float32, device=dev)]

    def call():
        rc = L.mzb_sort_step_noalloc(a.data_ptr(), m.data_ptr(), n, *(o.data_ptr() for o in outs), None)
        assert rc == 0
        torch.cuda.synchronize()

    call()  # the first call on the device looks up the scratch array
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(outs[0].cpu().numpy().view(np.uint32), r["srt_idx"][1])
