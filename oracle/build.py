"""Build recipe for the oracle (test infrastructure, never the product).

* ``oracle/_build/liboracle.so``: the C++ restatements in ``oracle.cpp``
  (conjunction screening) and ``sgp4pj_oracle.cpp`` (SGP4 polyjectory
  production), compiled without FMA contraction so that their operation
  order is the one written in the source.
* ``oracle/_ref/morton_ref``: mizuba's own Morton encoder header compiled in
  place from the reference tree by ``morton_ref_harness.cpp``;
* ``oracle/_ref/libsgp4_ref.so``: the SGP4 propagator the reference links
  (``mizuba/detail/sgp4/SGP4.cpp``, Vallado's public code) compiled in place
  with ``sgp4_ref_harness.cpp``.

The two ``_ref`` outputs are built only where the reference tree is present
(``MIZUBA_REFERENCE_TREE``, by default the mount point of this build
machine; the rest of the reference needs heyoka, TBB and Boost and cannot be
built here).  They are checkers for the tests; the built files travel with
the repository to machines without the reference tree.
"""

from __future__ import annotations

import os
import pathlib
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
REF_TREE = pathlib.Path(os.environ.get("MIZUBA_REFERENCE_TREE", "/root/reference"))
REF_DETAIL = REF_TREE / "mizuba" / "detail"


def _stale(out: pathlib.Path, *srcs: pathlib.Path) -> bool:
    return not out.exists() or any(s.stat().st_mtime > out.stat().st_mtime for s in srcs)


def build(force: bool = False) -> pathlib.Path:
    out = HERE / "_build" / "liboracle.so"
    srcs = [HERE / "oracle.cpp", HERE / "sgp4pj_oracle.cpp"]
    out.parent.mkdir(exist_ok=True)
    if force or _stale(out, *srcs):
        subprocess.check_call(
            ["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fPIC", "-shared",
             "-pthread", *map(str, srcs), "-o", str(out)]
        )
    ref_hdr = REF_DETAIL / "mortonND_LUT.h"
    harness = HERE / "morton_ref_harness.cpp"
    ref_out = HERE / "_ref" / "morton_ref"
    if ref_hdr.exists() and (force or _stale(ref_out, harness)):
        ref_out.parent.mkdir(exist_ok=True)
        subprocess.check_call(
            ["g++", "-O2", "-std=c++17", f"-I{REF_DETAIL}", str(harness), "-o", str(ref_out)]
        )
    sgp4_dir = REF_DETAIL / "sgp4"
    sgp4_harness = HERE / "sgp4_ref_harness.cpp"
    sgp4_out = HERE / "_ref" / "libsgp4_ref.so"
    if (sgp4_dir / "SGP4.cpp").exists() and (force or _stale(sgp4_out, sgp4_harness)):
        sgp4_out.parent.mkdir(exist_ok=True)
        subprocess.check_call(
            ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-w", f"-I{sgp4_dir}",
             str(sgp4_harness), str(sgp4_dir / "SGP4.cpp"), "-o", str(sgp4_out)]
        )
    return out


if __name__ == "__main__":
    print(build(force=True))
