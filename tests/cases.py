"""Polyjectory builders for the known-answer cases of mizuba's own test-suite.

Each builder restates, in code of this repository, the input of one reference
test (file:line cited) so that the oracle and the CUDA path can be checked on
exactly the situations the reference pins with exact or near-exact answers.
"""

from __future__ import annotations

import math
import pathlib

import numpy as np

from mizuba_b200.polyjectory import polyjectory


def zero_aabbs_pj():
    """mizuba/test/test_conjunctions.py:586-626 (object fixed at (1, 1, 1))."""
    td = np.zeros((6, 7))
    td[0, :3] = 1.0
    td[0, 6] = math.sqrt(3.0)
    return polyjectory([np.stack([td, td, td])], [[0.0, 1.0, 2.0, 3.0]], [0])


def _unit(axis_vals):
    td = np.zeros((6, 7))
    for k, v in axis_vals.items():
        td[0, k] = v
    return td


def no_traj_data_pj():
    """mizuba/test/test_conjunctions.py:628-692."""
    t0 = _unit({0: 1.0})
    t1 = _unit({0: -1.0})
    t2 = _unit({1: 1.0})
    t3 = _unit({1: -1.0})
    t4 = _unit({2: 1.0})
    t5 = _unit({2: -1.0})
    t6 = np.zeros((6, 7))
    t7 = np.zeros((6, 7))
    t7[0:1] = 1
    trajs = [np.stack([t0])] * 10 + [np.stack([t] * 2) for t in (t0, t1, t2, t3, t4, t5, t6, t7)]
    times = [[0.0, 1.0]] * 10 + [[0.0, 1.0, 2.0]] * 8
    return polyjectory(trajs, times, [0] * 18)


def bvh_single_pj():
    """mizuba/test/test_conjunctions.py:694-716 (one object)."""
    td = np.zeros((6, 7))
    td[1, :] = 0.1
    return polyjectory([td[None]], [[0.0, 1.0]], [0])


def bvh_twins_pj():
    """mizuba/test/test_conjunctions.py:718-728 (two identical objects)."""
    td = np.zeros((6, 7))
    td[1, :] = 0.1
    return polyjectory([td[None], td[None]], [[0.0, 1.0], [0.0, 1.0]], [0, 0])


def bvh_lastbit_pj():
    """mizuba/test/test_conjunctions.py:730-784 (codes differing at the LSB)."""
    ts = [_unit({0: 1.0}), _unit({0: -1.0}), _unit({1: 1.0}), _unit({1: -1.0}),
          _unit({2: 1.0}), _unit({2: -1.0}), np.zeros((6, 7))]
    t7 = np.zeros((6, 7))
    t7[0, :] = 1
    t8 = np.zeros((6, 7))
    t8[0, :] = 1
    t8[0, 0] = 1.0 - 2.1 / 2**16
    ts += [t7, t8]
    return polyjectory([t[None] for t in ts], [[0.0, 1.0]] * 9, [0] * 9)


TM = np.round(np.arange(21) * 0.1, 10)


def _linear(tm_list, sign):
    """Uniform unit-speed motion along x (one segment per 0.1 interval)."""
    out = []
    for tm in tm_list[1:]:
        td = np.zeros((7, 4))
        td[0, 0] = sign * (1.0 - (tm - 0.1))
        td[0, 1] = -sign * 1.0
        td[3, 0] = -sign * 1.0
        out.append(td)
    return np.ascontiguousarray(np.array(out).transpose((0, 2, 1)))


def cd_begin_end_pj(case):
    """mizuba/test/test_conjunctions.py:1071-1324, cases 1..6.

    Objects start at x = +-1 and meet at the origin at t = 1.
    Returns (pj, expected number of conjunctions (None = 'at least one'))."""
    sl = {
        1: (slice(None, 10), slice(11, None), 0),
        2: (slice(None, 12), slice(9, None), 1),
        3: (slice(11, None), slice(12, None), 0),
        4: (slice(9, None), slice(8, None), 1),
        5: (slice(None, 9), slice(None, 8), 0),
        6: (slice(None, 11), slice(None, 12), None),
    }[case]
    t0, t1 = TM[sl[0]], TM[sl[1]]
    pj = polyjectory([_linear(t0, 1.0), _linear(t1, -1.0)], [t0, t1], [0, 0])
    return pj, sl[2]


def boundary_incoming_pj(shift=0.0):
    """mizuba/test/test_boundary_conjunctions.py:24-123."""
    tm0 = np.array([0.0, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9])
    tm1 = np.round(np.arange(14) * 0.1, 10)
    tr = [[], []]
    for tm in tm1[1:]:
        td = np.zeros((7, 4))
        td[0, 0] = 1.0 - (tm - 0.1)
        td[0, 1] = -1.0
        td[3, 0] = -1.0
        if tm <= 0.9:
            tr[0].append(td.T.copy())
        tr[1].append((-td).T.copy())
    return polyjectory([np.array(tr[0]), np.array(tr[1])], [tm0 + shift, tm1 + shift], [0, 0])


def boundary_outgoing_pj(shift=0.0):
    """mizuba/test/test_boundary_conjunctions.py:125-198."""
    tm = np.array([0.0, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9])
    tr = [[], []]
    for t in tm[1:]:
        td = np.zeros((7, 4))
        td[0, 0] = 0.1 + (t - 0.1)
        td[0, 1] = 1.0
        td[3, 0] = 1.0
        tr[0].append(td.T.copy())
        tr[1].append((-td).T.copy())
    return polyjectory([np.array(tr[0]), np.array(tr[1])], [tm + shift, tm + shift], [0, 0])


GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def planar_circ_arrays():
    """The reference's own planar fixture (mizuba/test/_planar_circ.py, used
    by test_conjunctions.py:284-406): one revolution of a unit circular
    orbit in the xy plane as 7 order-20 Taylor segments, stored unchanged in
    tests/golden/planar_circ.npz by tests/golden/make_planar_circ.py."""
    d = np.load(GOLDEN / "planar_circ.npz")
    return d["tcs"].copy(), d["times"].copy()


def planar_circ_pj(shift=0.0):
    tr, tm = planar_circ_arrays()
    return polyjectory([tr], [tm + shift], [0])


def random_linear_pj(n, seed, span=1.0, nseg_max=4, box=10.0, speed=5.0, order=3):
    """Ragged random straight-line objects (segment boundaries at random
    times, some trajectories starting late or ending early, a few empty):
    a property-rich stress input for small sizes."""
    rng = np.random.default_rng(seed)
    trajs, times = [], []
    for i in range(n):
        if rng.random() < 0.05:
            trajs.append(np.zeros((0, order + 1, 7)))
            times.append(np.zeros(0))
            continue
        t_start = 0.0 if rng.random() < 0.8 else rng.uniform(0, span / 2)
        t_end = span if rng.random() < 0.8 else rng.uniform(t_start + span / 10, span)
        ns = int(rng.integers(1, nseg_max + 1))
        cuts = np.sort(rng.uniform(t_start, t_end, ns - 1))
        tm = np.concatenate([[t_start], cuts, [t_end]])
        if np.any(np.diff(tm) <= 0):
            tm = np.linspace(t_start, t_end, ns + 1)
        p0 = rng.uniform(-box, box, 3)
        v = rng.normal(0, speed, 3)
        acc = rng.normal(0, speed, 3)
        segs = []
        for t0 in tm[:-1]:
            c = np.zeros((order + 1, 7))
            dt = t0 - tm[0]
            pos = p0 + v * dt + 0.5 * acc * dt * dt
            vel = v + acc * dt
            c[0, :3] = pos
            c[1, :3] = vel
            c[2, :3] = 0.5 * acc
            c[0, 3:6] = vel
            c[1, 3:6] = acc
            c[0, 6] = np.linalg.norm(pos)
            c[1, 6] = np.dot(pos, vel) / max(np.linalg.norm(pos), 1e-9)
            segs.append(c)
        trajs.append(np.array(segs))
        times.append(tm)
    return polyjectory(trajs, times, [0] * n)


def clustered_pj(seed, n_base=120, n_groups=12, group=6, order=3):
    """Dense clusters: groups of near-identical objects (offsets far below the
    Morton cell, so groups share codes and form multi-object leaves with
    slightly different member boxes) inside a crowded box, so that many
    objects have more than a handful of broad-phase partners."""
    rng = np.random.default_rng(seed)
    base = random_linear_pj(n_base, seed=seed, box=3.0, speed=2.0, order=order)
    trajs, times = [], []
    for i in range(n_base):
        tr, tm, _ = base[i]
        trajs.append(np.array(tr))
        times.append(np.array(tm))
    for g in range(n_groups):
        src = int(rng.integers(0, n_base))
        tr, tm, _ = base[src]
        if tr.shape[0] == 0:
            continue
        for k in range(group):
            t2 = np.array(tr)
            t2[:, 0, :3] += rng.uniform(-1e-6, 1e-6, 3)
            if k % 3 == 0:
                t2[:, 1, :3] *= 1.0 + 1e-7 * k
            trajs.append(t2)
            times.append(np.array(tm))
    return polyjectory(trajs, times, [0] * len(trajs))
