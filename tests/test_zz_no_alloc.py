"""The allocation-free step sort (mzb_sort_step_noalloc) against the sort
inside mzb_conjunctions, called through the C ABI (needs a B200).

The no-alloc entry point serves callers that cannot allocate device memory
where they sort (hosts whose own allocator owns all device memory, or
allocation-free hot loops); its scratch is a fixed array inside the library.
This file is collected last so that a failure here leaves every other test
already run.
"""

import ctypes as ct

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def test_sort_step_noalloc_matches_pipeline_sort():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mizuba_b200 import _native, conjunctions

    L = _native.core()
    L.mzb_sort_step_noalloc.restype = ct.c_int
    L.mzb_sort_step_noalloc.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_uint64, ct.c_void_p, ct.c_void_p,
                                        ct.c_void_p, ct.c_void_p]
    pj = cases.random_linear_pj(700, seed=11, box=30.0, speed=20.0)
    ref = conjunctions(pj, 1.0, 0.05)
    n = pj.n_objs
    dev = torch.device("cuda", 0)
    # Two calls in a row on different steps: the shared scratch keeps the
    # first call's contents, which the second must not depend on.
    for step in (3, 12):
        a = torch.from_numpy(np.array(ref.aabbs[step], copy=True)).to(dev)
        m = torch.from_numpy(np.array(ref.mcodes[step], copy=True).view(np.int64)).to(dev)
        o_idx = torch.empty(n, dtype=torch.int32, device=dev)
        o_mc = torch.empty(n, dtype=torch.int64, device=dev)
        o_ab = torch.empty((n + 1, 2, 4), dtype=torch.float32, device=dev)
        rc = L.mzb_sort_step_noalloc(a.data_ptr(), m.data_ptr(), n, o_idx.data_ptr(), o_mc.data_ptr(),
                                     o_ab.data_ptr(), None)
        assert rc == 0, L.mzb_last_error().decode()
        torch.cuda.synchronize()
        assert np.array_equal(o_idx.cpu().numpy().view(np.uint32), ref.srt_idx[step])
        assert np.array_equal(o_mc.cpu().numpy().view(np.uint64), ref.srt_mcodes[step])
        assert np.array_equal(o_ab.cpu().numpy().view(np.uint32), ref.srt_aabbs[step].view(np.uint32))
    # Sizes beyond the built-in scratch are rejected with a clear error.
    rc = L.mzb_sort_step_noalloc(a.data_ptr(), m.data_ptr(), 1 << 22, o_idx.data_ptr(), o_mc.data_ptr(),
                                 o_ab.data_ptr(), None)
    assert rc == 1 and b"exceed the capacity" in L.mzb_last_error()
