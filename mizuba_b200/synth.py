"""Seeded synthetic catalogues for the conjunction-screening workloads.

The element distributions follow the workload definitions of this project
(seeds 1001-1005): 80 % LEO (perigee altitude U(350, 1500) km,
e = min(|N(0, 0.005)|, 0.05)), 15 % MEO/HEO (e U(0.05, 0.7), same perigee
range), 5 % GEO (a = 42164 km, e = |N(0, 5e-4)|, i U(0, 15 deg)); non-GEO
inclinations are a 1/3 mixture of 53 deg, 97.6 deg and U(0, 180 deg); RAAN,
argument of perigee and mean anomaly U(0, 2 pi); bstar log-uniform in
[1e-5, 1e-3] per earth radius.  Dense shells are circular, 72 planes x N
slots at 550 km / 53 deg, 1100 km / 70 deg and 550 km / 97.6 deg with phase
jitter U(0, 0.5 deg).

The polyjectory itself is built on the host by the C++ builder in
``csrc/pjgen.cpp`` (a Keplerian + J2 + drag model standing in for mizuba's
``make_sgp4_polyjectory``, which needs heyoka).
"""

from __future__ import annotations

import ctypes as ct
import math
import os

import numpy as np

from . import _native
from .polyjectory import polyjectory

RE = 6378.135
DEG = math.pi / 180.0

# name -> (n_objs, shell objects, span days, threshold km, seed, low-perigee fraction)
WORKLOADS = {
    "c1_1k_1d": dict(n=1000, shells=0, days=1.0, thresh=5.0, seed=1001, lowp=0.0),
    "c2_20k_1d": dict(n=20000, shells=0, days=1.0, thresh=5.0, seed=1002, lowp=0.0),
    "c3_20k_shells_1d": dict(n=20000, shells=6000, days=1.0, thresh=10.0, seed=1003, lowp=0.0),
    "c4_30k_7d": dict(n=30000, shells=0, days=7.0, thresh=5.0, seed=1004, lowp=0.05),
    "c5_60k_shells_3d": dict(n=60000, shells=15000, days=3.0, thresh=20.0, seed=1005, lowp=0.0),
}
INTERVAL_DAYS = 3.0 / 1440.0


def base_elements(n, rng, lowp=0.0):
    """(n, 7) array: a [km], e, inc, raan, argp, M0 [rad], bstar."""
    el = np.zeros((n, 7))
    u = rng.random(n)
    n_geo = int(round(0.05 * n))
    n_meo = int(round(0.15 * n))
    kind = np.zeros(n, dtype=np.int64)  # 0 LEO, 1 MEO/HEO, 2 GEO, 3 low perigee
    kind[:n_meo] = 1
    kind[n_meo:n_meo + n_geo] = 2
    n_low = int(round(lowp * n))
    kind[n_meo + n_geo:n_meo + n_geo + n_low] = 3
    rng.shuffle(kind)
    hp = rng.uniform(350.0, 1500.0, n)
    e = np.minimum(np.abs(rng.normal(0.0, 0.005, n)), 0.05)
    e_meo = rng.uniform(0.05, 0.7, n)
    e = np.where(kind == 1, e_meo, e)
    hp = np.where(kind == 3, rng.uniform(200.0, 350.0, n), hp)
    a = (RE + hp) / (1.0 - e)
    geo = kind == 2
    a[geo] = 42164.0
    e[geo] = np.abs(rng.normal(0.0, 5e-4, geo.sum()))
    mix = rng.integers(0, 3, n)
    inc = np.where(mix == 0, 53.0 * DEG, np.where(mix == 1, 97.6 * DEG, rng.uniform(0, math.pi, n)))
    inc[geo] = rng.uniform(0, 15.0 * DEG, geo.sum())
    el[:, 0] = a
    el[:, 1] = e
    el[:, 2] = inc
    el[:, 3] = rng.uniform(0, 2 * math.pi, n)
    el[:, 4] = rng.uniform(0, 2 * math.pi, n)
    el[:, 5] = rng.uniform(0, 2 * math.pi, n)
    bstar = 10.0 ** rng.uniform(-5.0, -3.0, n)
    bstar = np.where(kind == 3, 10.0 ** rng.uniform(-4.0, -3.0, n), bstar)
    el[:, 6] = bstar
    del u
    return el


def shell_elements(n_shell, rng):
    shells = [(550.0, 53.0), (1100.0, 70.0), (550.0, 97.6)]
    per = int(math.ceil(n_shell / 3))
    slots = int(math.ceil(per / 72))
    rows = []
    for alt, inc in shells:
        k = 0
        for p in range(72):
            for s in range(slots):
                if k >= per:
                    break
                m = (s * 360.0 / slots + rng.uniform(0, 0.5)) * DEG
                rows.append([RE + alt, 0.0, inc * DEG, 5.0 * p * DEG, 0.0, m, 1e-5])
                k += 1
    el = np.array(rows[:n_shell])
    return el


def elements_for(name):
    w = WORKLOADS[name]
    rng = np.random.default_rng(w["seed"])
    nb = w["n"] - w["shells"]
    el = base_elements(nb, rng, w["lowp"])
    if w["shells"]:
        el = np.concatenate([el, shell_elements(w["shells"], rng)])
    return el


def build_polyjectory(elements, span_days, order=18, n_threads=None, t_start=0.0):
    """Builds a polyjectory from an (n, 7) element array on the host; the
    trajectories cover [t_start, t_start + span_days] days."""
    L = _native.pjgen()
    el = np.ascontiguousarray(elements, dtype=np.float64)
    n = el.shape[0]
    nt = n_threads or os.cpu_count() or 1
    h = L.mzb_pjgen_build(el.ctypes.data, n, float(t_start), float(span_days), int(order), int(nt))
    try:
        def grab(ptr, dtype, count):
            if count == 0:
                return np.zeros(0, dtype=dtype)
            buf = (ct.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr)
            return np.frombuffer(buf, dtype=dtype, count=count).copy()

        traj = grab(L.mzb_pjgen_traj(h), np.float64, L.mzb_pjgen_traj_size(h))
        time = grab(L.mzb_pjgen_time(h), np.float64, L.mzb_pjgen_time_size(h))
        toff = grab(L.mzb_pjgen_traj_off(h), np.uint64, 2 * n).reshape(n, 2)
        tmoff = grab(L.mzb_pjgen_time_off(h), np.uint64, n)
        status = grab(L.mzb_pjgen_status(h), np.int32, n)
        max_err = L.mzb_pjgen_max_err(h)
    finally:
        L.mzb_pjgen_free(h)
    pj = polyjectory.from_arrays(traj, toff, time, tmoff, status, order)
    pj.fit_error_km = max_err
    return pj


def workload(name, n_objs=None, span_days=None, order=18, t_start=0.0):
    """Polyjectory for a named workload (optionally truncated, or starting
    later on the time axis)."""
    w = WORKLOADS[name]
    el = elements_for(name)
    if n_objs is not None:
        el = el[:n_objs]
    return build_polyjectory(el, span_days or w["days"], order=order, t_start=t_start)
