"""Writes ``planar_circ.npz`` from the fixture the reference ships.

mizuba's own tests drive ``test_main`` (mizuba/test/test_conjunctions.py:
284-406) with ``mizuba/test/_planar_circ.py``: the order-20 Taylor
coefficients (7 segments x 21 coefficients x 7 variables) and the 8 time
points of one revolution of a planar circular Keplerian orbit in
non-dimensional units.  That module holds only numpy array literals; this
script imports it from the reference tree and stores the two arrays
unchanged, so the tests can feed the reference's golden input to the oracle
and to the GPU on machines where the reference tree is absent.

Usage: python tests/golden/make_planar_circ.py [path/to/mizuba/test/_planar_circ.py]
"""

import importlib.util
import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
DEFAULT = pathlib.Path(os.environ.get("MIZUBA_REFERENCE_TREE", "/root/reference")) / "mizuba/test/_planar_circ.py"


def main():
    src = pathlib.Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT
    spec = importlib.util.spec_from_file_location("_planar_circ", src)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    tcs = np.ascontiguousarray(mod._planar_circ_tcs, dtype=np.float64)
    times = np.ascontiguousarray(mod._planar_circ_times, dtype=np.float64)
    assert tcs.shape == (times.shape[0] - 1, 21, 7), (tcs.shape, times.shape)
    np.savez_compressed(HERE / "planar_circ.npz", tcs=tcs, times=times)
    print(f"wrote {HERE / 'planar_circ.npz'}: tcs {tcs.shape}, times {times.shape}")


if __name__ == "__main__":
    main()
