"""mzb_pj_create rejects malformed polyjectories before any device work.

The C ABI runs the polyjectory constructor's checks (mizuba/polyjectory.cpp:
460-600) on the host: a NaN, negative or non-increasing time point, offsets
outside the data, an all-empty polyjectory or a maxT that is not the largest
end time return MZB_INVALID_ARGUMENT with the reference's message.  These
checks come before the first device call, so they run here without a GPU.
"""

import ctypes as ct

import numpy as np
import pytest

ORDER = 3
OP1 = ORDER + 1


@pytest.fixture(scope="module")
def L():
    from mizuba_b200 import _native, build

    build.build_cuda()
    return _native.core()


def make(n_steps=(2, 3)):
    """Flat arrays of a small valid polyjectory: object k has n_steps[k]
    segments on the time points 0, 1, 2, ..."""
    traj, toff, time, tmoff = [], [], [], []
    off = 0
    for ns in n_steps:
        toff.append((off, ns))
        traj.append(np.ones(ns * OP1 * 7))
        off += ns * OP1 * 7
        tmoff.append(sum(len(t) for t in time))
        if ns:
            time.append(np.arange(ns + 1, dtype=np.float64))
    return (np.concatenate(traj), np.array(toff, dtype=np.uint64),
            np.concatenate(time) if time else np.zeros(1), np.array(tmoff, dtype=np.uint64))


def create(L, traj, toff, time, tmoff, maxT=None):
    if maxT is None:
        nz = toff[:, 1] > 0
        maxT = float(time[(tmoff[nz] + toff[nz, 1]).astype(np.int64)].max()) if nz.any() else 0.0
    h = ct.c_void_p()
    rc = L.mzb_pj_create(traj.ctypes.data, traj.size, toff.ctypes.data, time.ctypes.data, time.size,
                         tmoff.ctypes.data, len(tmoff), ORDER, maxT, ct.byref(h))
    assert not h.value
    return rc, L.mzb_last_error().decode()


def test_non_finite_time(L):
    traj, toff, time, tmoff = make()
    time[4] = np.nan  # object 1, second time point
    rc, msg = create(L, traj, toff, time, tmoff, maxT=3.0)
    assert rc == 1 and msg == "A non-finite time coordinate was found for the object at index 1"


def test_negative_time(L):
    traj, toff, time, tmoff = make()
    time[0] = -1.0
    rc, msg = create(L, traj, toff, time, tmoff)
    assert rc == 1 and msg == "A negative time coordinate was found for the object at index 0"


@pytest.mark.parametrize("bad", [1.0, 0.5])  # equal to, then below, the previous time point
def test_non_increasing_time(L, bad):
    traj, toff, time, tmoff = make()
    time[5] = bad  # object 1: 0, 1, bad, 3
    rc, msg = create(L, traj, toff, time, tmoff, maxT=3.0)
    assert rc == 1 and msg == "The sequence of times for the object at index 1 is not monotonically increasing"


def test_all_empty(L):
    traj, toff, time, tmoff = make((0, 0))
    rc, msg = create(L, traj, toff, time, tmoff, maxT=0.0)
    assert rc == 1 and "have a number of steps equal to zero" in msg


def test_max_time_mismatch(L):
    traj, toff, time, tmoff = make()
    rc, msg = create(L, traj, toff, time, tmoff, maxT=2.5)
    assert rc == 1 and "does not equal the largest trajectory end time" in msg


def test_offsets_outside_the_data(L):
    traj, toff, time, tmoff = make()
    toff[1, 1] = 4  # one segment more than the data hold
    rc, msg = create(L, traj, toff, time, tmoff, maxT=3.0)
    assert rc == 1 and "invalid trajectory offsets for the object at index 1" in msg
    traj, toff, time, tmoff = make()
    tmoff[1] = time.size - 2  # the time points run past the array
    rc, msg = create(L, traj, toff, time, tmoff, maxT=3.0)
    assert rc == 1 and "invalid time offsets for the object at index 1" in msg


def test_first_failing_object_of_a_large_input(L):
    # 10,000 objects (the checks run in parallel over object ranges): the
    # error reported is the lowest failing index, as in the reference's
    # serial pass, whatever range finds its error first.
    traj, toff, time, tmoff = make([2] * 10000)
    time[int(tmoff[9000]) + 1] = time[int(tmoff[9000])]  # object 9,000: repeated time point
    time[int(tmoff[7000]) + 2] = -np.inf                  # object 7,000: non-finite
    time[int(tmoff[8000])] = -1.0                         # object 8,000: negative
    rc, msg = create(L, traj, toff, time, tmoff, maxT=2.0)
    assert rc == 1 and msg == "A non-finite time coordinate was found for the object at index 7000"
    time[int(tmoff[7000]) + 2] = 2.0
    rc, msg = create(L, traj, toff, time, tmoff, maxT=2.0)
    assert rc == 1 and msg == "A negative time coordinate was found for the object at index 8000"
