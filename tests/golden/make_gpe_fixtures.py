"""Writes ``gpes.npz`` from the GPE catalogues the reference ships.

mizuba's tests feed ``make_sgp4_polyjectory`` with real general perturbation
element sets stored as parquet files under ``mizuba/test/`` (for instance
test_make_sgp4_polyjectory.py:69-330 with single_gpe, single_gpe_ds,
syncom_gpe, multi_gpes and iss_gpes; strack_20240705 is a 26,389-object
catalogue).  This script reads the ten numeric fields of the reference's
``gpe`` struct (mizuba/make_sgp4_polyjectory.hpp: norad_id, epoch_jd1,
epoch_jd2 as UTC Julian dates, n0 [rad/min], e0, i0, node0, omega0, m0
[rad], bstar [1/earth radii]) from each file, unchanged, and stores them as
one structured array per file, so that the tests and the benchmark can use
the reference's inputs where the reference tree is absent.

Usage: python tests/golden/make_gpe_fixtures.py [path/to/mizuba/test]
"""

import os
import pathlib
import sys

import numpy as np
import pyarrow.parquet as pq

HERE = pathlib.Path(__file__).resolve().parent
DEFAULT = pathlib.Path(os.environ.get("MIZUBA_REFERENCE_TREE", "/root/reference")) / "mizuba" / "test"
FIELDS = ["norad_id", "epoch_jd1", "epoch_jd2", "n0", "e0", "i0", "node0", "omega0", "m0", "bstar"]
GPE_DTYPE = np.dtype([("norad_id", "<u8")] + [(f, "<f8") for f in FIELDS[1:]])
FILES = ["single_gpe", "single_gpe_ds", "syncom_gpe", "multi_gpes", "iss_gpes", "strack_20240705"]


def main():
    src = pathlib.Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT
    out = {}
    for name in FILES:
        t = pq.read_table(src / f"{name}.parquet", columns=FIELDS)
        a = np.zeros(t.num_rows, dtype=GPE_DTYPE)
        for f in FIELDS:
            a[f] = t.column(f).to_numpy()
        out[name] = a
        print(f"{name}: {len(a)} element sets")
    np.savez_compressed(HERE / "gpes.npz", **out)
    print(f"wrote {HERE / 'gpes.npz'} ({(HERE / 'gpes.npz').stat().st_size} bytes)")


if __name__ == "__main__":
    main()
