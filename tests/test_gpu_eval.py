"""State evaluation on the GPU (polyjectory::state_eval / state_meval,
mizuba/polyjectory.cpp:1092-1366) against the reference's known answers
(mizuba/test/test_polyjectory.py:792-1293) and, bit for bit, against the
oracle's restatement of pj_eval_obj_state on a synthetic catalogue."""

import numpy as np
import pytest

import cases
import oracle

pytestmark = pytest.mark.gpu

ROW0 = [0.89, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0]
ROW0b = [0.88, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0]
ROW1 = [0.20, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0]
ROW1b = [0.21, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0]


@pytest.fixture(scope="module")
def mzb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mizuba_b200

    return mizuba_b200


@pytest.fixture(scope="module")
def pj(mzb):
    return cases.cd_begin_end_pj(1)[0]


def close(a, b):
    return np.allclose(a, b, rtol=0.0, atol=1e-15)


def test_known_answers(pj):
    res = pj.state_eval(time=np.array([0.11, 0.11]))
    assert close(res[0], ROW0) and np.all(np.isnan(res[1]))
    out = np.zeros((2, 7))
    res = pj.state_eval(time=np.array([0.11, 0.11]), out=out)
    assert res is out and close(res[0], ROW0) and np.all(np.isnan(res[1]))
    res = pj.state_meval(time=np.array([0.11, 0.12]))
    assert close(res[0], [ROW0, ROW0b]) and np.all(np.isnan(res[1]))
    out = np.zeros((2, 2, 7))
    res = pj.state_meval(out=out, time=np.array([0.11, 0.12]))
    assert res is out and close(res[0], [ROW0, ROW0b]) and np.all(np.isnan(res[1]))
    res = pj.state_meval(time=np.array([[0.11], [0.12]]))
    assert close(res[0], [ROW0]) and np.all(np.isnan(res[1]))
    res = pj.state_eval(time=np.array([0.11, 0.12] * 1000), obj_idx=[0, 1] * 1000)
    assert close(res[::2], [ROW0] * 1000) and np.all(np.isnan(res[1::2]))
    res = pj.state_meval(time=np.array([0.11, 0.12] * 1000), obj_idx=[0, 1] * 1000)
    assert close(res[::2], [ROW0, ROW0b] * 1000) and np.all(np.isnan(res[1::2]))
    res = pj.state_meval(time=np.array([[0.11, 0.12] * 1000, [1.2, 1.21] * 1000]), obj_idx=[0, 1])
    assert close(res[0], [ROW0, ROW0b] * 1000) and close(res[1], [ROW1, ROW1b] * 1000)
    res = pj.state_meval(time=np.array([[0.11, 0.12] * 1000, [1.2, 1.21] * 1000] * 1000), obj_idx=[0, 1] * 1000)
    assert close(res[::2], [ROW0, ROW0b] * 1000) and close(res[1::2], [ROW1, ROW1b] * 1000)
    res = pj.state_eval(time=np.array([1.2, 1.21]))
    assert np.all(np.isnan(res[0])) and close(res[1], ROW1b)
    res = pj.state_eval(time=np.array([0.11, 1.21]))
    assert close(res[0], ROW0) and close(res[1], ROW1b)
    res = pj.state_eval(time=0.1)
    assert close(res[0], [0.9, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0]) and np.all(np.isnan(res[1]))
    res = pj.state_eval(time=1.2)
    assert np.all(np.isnan(res[0])) and close(res[1], ROW1)
    res = pj.state_eval(time=0.1, obj_idx=0)
    assert res.shape == (1, 7) and close(res, [[0.9, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0]])
    res = pj.state_eval(time=1.2, obj_idx=1)
    assert close(res, [ROW1])


def test_empty_trajectory(mzb, pj):
    p2 = mzb.polyjectory([pj[0][0], np.empty((0, 4, 7))], [pj[0][1], []], [0, 0])
    res = p2.state_eval(time=np.array([0.1, 0.1]))
    assert np.all(np.isnan(res[1])) and not np.any(np.isnan(res[0]))


def test_size_and_value_errors(pj):
    def msg(fn, *a, exc=ValueError, **k):
        with pytest.raises(exc) as e:
            fn(*a, **k)
        return str(e.value)

    assert ("Invalid time array passed to state_eval(): the number of objects is 2 but the size of the array "
            "is 5 (the two numbers must be equal)") in msg(pj.state_eval, time=np.zeros((5,)))
    assert "An non-finite evaluation time of " in msg(pj.state_eval, time=np.full((2,), float("inf")))
    assert "An non-finite evaluation time of " in msg(pj.state_eval, float("nan"))
    assert ("Invalid time array passed to state_eval(): the number of selected objects is 1 but the size of "
            "the array is 2 (the two numbers must be equal)") in msg(pj.state_eval, time=np.array([0.11, 0.11]),
                                                                    obj_idx=1)
    assert ("Invalid object index 2 specified - the total number of objects in the polyjectory is only 2"
            in msg(pj.state_eval, time=0.11, obj_idx=2, exc=IndexError))
    assert ("Invalid object index 45 specified - the total number of objects in the polyjectory is only 2"
            in msg(pj.state_eval, time=0.11, obj_idx=[45], exc=IndexError))
    assert ("Invalid output array passed to state_eval(): the number of objects is 2 but the size of the "
            "first dimension of the array is 3 (the two numbers must be equal)") in msg(
        pj.state_eval, time=0.11, out=np.full((3, 7), 1.0))
    assert ("Invalid output array passed to state_eval(): the number of objects selected for evaluation is 1 "
            "but the size of the first dimension of the array is 3 (the two numbers must be equal)") in msg(
        pj.state_eval, time=0.11, out=np.full((3, 7), 1.0), obj_idx=[1])
    assert ("Invalid output array passed to state_eval(): the number of objects is 2 but the size of the "
            "first dimension of the array is 3 (the two numbers must be equal)") in msg(
        pj.state_eval, time=[0.11, 0.11], out=np.full((3, 7), 1.0))
    assert ("Invalid output array passed to state_eval(): the number of objects selected for evaluation is 1 "
            "but the size of the first dimension of the array is 3 (the two numbers must be equal)") in msg(
        pj.state_eval, time=[0.11, 0.11], out=np.full((3, 7), 1.0), obj_idx=[1])
    assert ("Invalid output array passed to state_meval(): the number of time evaluations per object is 2 "
            "but the size of the second dimension of the array is 4 (the two numbers must be equal)") in msg(
        pj.state_meval, time=[0.11, 0.11], out=np.zeros((3, 4, 7)))
    assert ("Invalid output array passed to state_meval(): the number of selected objects is 1 but the size "
            "of the first dimension of the array is 2 (the two numbers must be equal)") in msg(
        pj.state_meval, time=[0.11, 0.11], out=np.zeros((2, 2, 7)), obj_idx=[1])
    assert ("Invalid output array passed to state_meval(): the number of selected objects is 1 but the size "
            "of the first dimension of the array is 2 (the two numbers must be equal)") in msg(
        pj.state_meval, time=[[0.11, 0.11]], out=np.zeros((2, 2, 7)), obj_idx=[1])
    assert ("Invalid time array passed to state_meval(): the number of selected objects is 1 but the size of "
            "the first dimension of the array is 2 (the two numbers must be equal)") in msg(
        pj.state_meval, time=[[0.11, 0.11], [0.11, 0.11]], out=np.zeros((1, 2, 7)), obj_idx=[1])
    assert ("Invalid output array passed to state_meval(): the number of objects is 2 but the size of the "
            "first dimension of the array is 3 (the two numbers must be equal)") in msg(
        pj.state_meval, time=[0.11, 0.11], out=np.zeros((3, 2, 7)))
    assert ("Invalid output array passed to state_meval(): the number of objects is 2 but the size of the "
            "first dimension of the array is 3 (the two numbers must be equal)") in msg(
        pj.state_meval, time=[[0.11, 0.11]], out=np.zeros((3, 2, 7)))
    assert ("Invalid time array passed to state_meval(): the number of objects is 2 but the size of the "
            "first dimension of the array is 1 (the two numbers must be equal)") in msg(
        pj.state_meval, time=[[0.11, 0.11]], out=np.zeros((2, 2, 7)))
    # No evaluation, no error (an empty selection).
    assert pj.state_eval(time=float("nan"), obj_idx=np.zeros(0, dtype=np.uintp)).shape == (0, 7)


def _catalogue():
    from mizuba_b200 import synth

    return synth.build_polyjectory(synth.elements_for("c1_1k_1d")[:300], 0.25)


def _edge_times(pj, rng, n):
    """Times on segment boundaries, first / last points, outside the data, and
    random interior times, per object."""
    tms = []
    for i in range(pj.n_objs):
        t = pj[i][1]
        if len(t) == 0:
            tms.append(rng.uniform(0, 0.25, n))
            continue
        c = [t[0], t[-1], t[-1] + 1e-3, t[0] - 1e-3, np.nextafter(t[-1], -np.inf)]
        c += list(rng.choice(t, min(4, len(t))))
        c += list(rng.uniform(t[0], t[-1], n - len(c)))
        tms.append(np.array(c[:n]))
    return np.array(tms)


def test_bit_exact_vs_oracle(mzb):
    pj = _catalogue()
    rng = np.random.default_rng(7)
    T = _edge_times(pj, rng, 12)  # [n_objs][12]
    N = pj.n_objs
    # state_meval, 2-D times
    g = pj.state_meval(time=T)
    r = oracle.state_eval(pj, np.repeat(np.arange(N), 12), T.ravel()).reshape(N, 12, 7)
    assert np.array_equal(g, r, equal_nan=True)
    # state_meval, 1-D times shared by a selection with repeats
    sel = rng.integers(0, N, 500).astype(np.uintp)
    t1 = T[0]
    g = pj.state_meval(time=t1, obj_idx=sel)
    r = oracle.state_eval(pj, np.repeat(sel, len(t1)), np.tile(t1, len(sel))).reshape(len(sel), len(t1), 7)
    assert np.array_equal(g, r, equal_nan=True)
    # state_eval, one time per object and a scalar time
    g = pj.state_eval(time=T[:, 3].copy())
    r = oracle.state_eval(pj, np.arange(N), T[:, 3])
    assert np.array_equal(g, r, equal_nan=True)
    g = pj.state_eval(time=0.125)
    r = oracle.state_eval(pj, np.arange(N), np.full(N, 0.125))
    assert np.array_equal(g, r, equal_nan=True)
    assert np.count_nonzero(~np.isnan(g[:, 0])) > N // 2
