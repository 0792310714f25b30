"""Build recipe for the oracle (test infrastructure, never the product).

* ``oracle/_build/liboracle.so``: the C++ restatement in ``oracle.cpp``,
  compiled without FMA contraction so that its operation order is the one
  written in the source.
* ``oracle/_ref/morton_ref``: mizuba's own Morton encoder header compiled in
  place from the reference tree by ``morton_ref_harness.cpp`` (only when the
  reference tree is mounted; the rest of the reference needs heyoka, TBB and
  Boost and cannot be built here).
"""

from __future__ import annotations

import pathlib
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
REF_DETAIL = pathlib.Path("/root/reference/mizuba/detail")


def _stale(out: pathlib.Path, *srcs: pathlib.Path) -> bool:
    return not out.exists() or any(s.stat().st_mtime > out.stat().st_mtime for s in srcs)


def build(force: bool = False) -> pathlib.Path:
    out = HERE / "_build" / "liboracle.so"
    src = HERE / "oracle.cpp"
    out.parent.mkdir(exist_ok=True)
    if force or _stale(out, src):
        subprocess.check_call(
            ["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fPIC", "-shared",
             "-pthread", str(src), "-o", str(out)]
        )
    ref_hdr = REF_DETAIL / "mortonND_LUT.h"
    harness = HERE / "morton_ref_harness.cpp"
    ref_out = HERE / "_ref" / "morton_ref"
    if ref_hdr.exists() and (force or _stale(ref_out, harness)):
        ref_out.parent.mkdir(exist_ok=True)
        subprocess.check_call(
            ["g++", "-O2", "-std=c++17", f"-I{REF_DETAIL}", str(harness), "-o", str(ref_out)]
        )
    return out


if __name__ == "__main__":
    print(build(force=True))
