"""State evaluation: the oracle against the reference's known answers, and
the argument checks that the Python layer makes before any device work
(mizuba/test/test_polyjectory.py:792-1293; mizuba/expose_polyjectory.cpp:65-98,
308-530).  No GPU needed."""

import numpy as np
import pytest

import cases
import oracle


@pytest.fixture(scope="module")
def pj():
    # test_polyjectory.py:796-846: object 0 moves along x on [0, 0.9],
    # object 1 on [1.1, 2.0].
    return cases.cd_begin_end_pj(1)[0]


def close(a, b):
    return np.allclose(a, b, rtol=0.0, atol=1e-15)


def test_oracle_known_answers(pj):
    out = oracle.state_eval(pj, [0, 1, 0, 1, 1, 0, 1, 0], [0.11, 0.11, 0.12, 1.2, 1.21, 0.1, 0.1, 1.2])
    assert close(out[0], [0.89, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0])
    assert np.all(np.isnan(out[1]))
    assert close(out[2], [0.88, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0])
    assert close(out[3], [0.2, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0])
    assert close(out[4], [0.21, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0])
    assert close(out[5], [0.9, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0])
    assert np.all(np.isnan(out[6])) and np.all(np.isnan(out[7]))


def test_oracle_time_range_edges(pj):
    # First time point: data; last time point and beyond: NaN; a segment
    # boundary belongs to the segment that starts there (upper_bound).
    out = oracle.state_eval(pj, [0, 0, 0, 0, 1], [0.0, 0.9, -0.1, 0.2, 1.1])
    assert close(out[0], [1.0, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0])
    assert np.all(np.isnan(out[1])) and np.all(np.isnan(out[2]))
    assert close(out[3], [0.8, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0])
    assert close(out[4], [0.1, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0])


def test_oracle_empty_trajectory():
    from mizuba_b200 import polyjectory

    base = cases.cd_begin_end_pj(1)[0]
    pj = polyjectory([base[0][0], np.empty((0, 4, 7))], [base[0][1], []], [0, 0])
    out = oracle.state_eval(pj, [1], [0.1])
    assert np.all(np.isnan(out))


def test_oracle_non_finite_time(pj):
    with pytest.raises(ValueError, match="An non-finite evaluation time of "):
        oracle.state_eval(pj, [0], [float("inf")])


# ---- argument checks made before any device work


def test_state_eval_array_checks(pj):
    with pytest.raises(ValueError, match=r"The time array passed to state_eval\(\) must be C contiguous"):
        pj.state_eval(np.zeros((5,))[::2])
    with pytest.raises(ValueError) as e:
        pj.state_eval(np.zeros((5, 5)))
    assert ("The time array passed to state_eval() must have 1 dimension, but the number of dimensions is 2 "
            "instead") in str(e.value)
    with pytest.raises(ValueError, match=r"selector array passed to state_eval\(\) must be C contiguous"):
        pj.state_eval(time=0.11, obj_idx=np.array([0, 0, 0, 0], dtype=np.uintp)[::2])
    with pytest.raises(ValueError) as e:
        pj.state_eval(time=0.11, obj_idx=np.zeros((2, 2)))
    assert ("The selector array passed to state_eval() must have 1 dimension, but the number of dimensions "
            "is 2 instead") in str(e.value)
    with pytest.raises(ValueError, match=r"output array passed to state_eval\(\) must be C contiguous"):
        pj.state_eval(time=0.11, out=np.array([1.0, 2.0, 3.0])[::2])
    with pytest.raises(ValueError) as e:
        pj.state_eval(time=0.11, out=np.full((1,), 1.0))
    assert ("The output array passed to state_eval() must have 2 dimensions, but the number of dimensions "
            "is 1 instead") in str(e.value)
    with pytest.raises(ValueError) as e:
        pj.state_eval(time=0.11, out=np.full((1, 6), 1.0))
    assert ("The output array passed to state_eval() must have a size of 7 in the second dimension, but "
            "the size in the second dimension is 6 instead") in str(e.value)
    out = np.zeros((2, 7))
    with pytest.raises(ValueError, match="Potential memory overlap detected between the output array passed "
                                         r"to state_eval\(\) and the time array"):
        pj.state_eval(time=out[:2], out=out)
    with pytest.raises(ValueError, match="Potential memory overlap detected between the output array passed "
                                         r"to state_eval\(\) and the array of object indices"):
        pj.state_eval(time=[1.1, 1.1], out=out, obj_idx=out[0, :2].view(dtype=np.uintp))


def test_state_meval_array_checks(pj):
    with pytest.raises(ValueError, match=r"The time array passed to state_meval\(\) must be C contiguous"):
        pj.state_meval(time=np.array([0.11, 0.11, 0.11, 0.11])[::2])
    with pytest.raises(ValueError) as e:
        pj.state_meval(time=np.zeros((3, 3, 3)))
    assert ("The time array passed to state_meval() must have either 1 or 2 dimensions, but the number of "
            "dimensions is 3 instead") in str(e.value)
    with pytest.raises(ValueError, match=r"output array passed to state_meval\(\) must be C contiguous"):
        pj.state_meval(time=[0.11, 0.11], out=np.array([1.0, 2.0, 0.3, 0.4])[::2])
    with pytest.raises(ValueError) as e:
        pj.state_meval(time=[0.11, 0.11], out=np.array([1.0, 2.0, 0.3, 0.4]))
    assert ("The output array passed to state_meval() must have 3 dimensions, but the number of dimensions "
            "is 1 instead") in str(e.value)
    with pytest.raises(ValueError) as e:
        pj.state_meval(time=[0.11, 0.11], out=np.zeros((3, 4, 5)))
    assert ("The output array passed to state_meval() must have a size of 7 in the third dimension, but the "
            "size in the third dimension is 5 instead") in str(e.value)
    out = np.zeros((2, 2, 7))
    with pytest.raises(ValueError, match="Potential memory overlap detected between the output array passed "
                                         r"to state_meval\(\) and the time array"):
        pj.state_meval(time=out[0, 0, :2], out=out)
    with pytest.raises(ValueError, match="Potential memory overlap detected between the output array passed "
                                         r"to state_meval\(\) and the array of object indices"):
        pj.state_meval(time=[1.1, 1.1], out=out, obj_idx=out[0, 0, :2].view(dtype=np.uintp))
