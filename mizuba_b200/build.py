"""In-tree build of the native libraries (no JIT cache, nothing installed).

* ``_lib/libmizuba_b200.so``: the sm_100a CUDA kernels, the host pipeline and
  the C ABI declared in ``include/mizuba_b200.h``;
* ``_lib/libmzb_pjgen.so``: the host-side synthetic polyjectory builder.
"""

from __future__ import annotations

import os
import pathlib
import subprocess

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "_lib"
NVCC = os.environ.get("NVCC", "nvcc")

CUDA_SOURCES = ["pipeline.cu", "k_aabb.cu", "k_sort.cu", "k_bvh.cu", "k_broad.cu", "k_narrow.cu", "k_eval.cu", "k_probe.cu", "k_sgp4.cu"]
CUDA_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # The plain form reproduces the oracle's operation order exactly: no FMA
    # contraction, IEEE division and square root, denormals kept.
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    f"-I{ROOT / 'include'}", f"-I{CSRC}",
]


def _stale(out: pathlib.Path, srcs) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(pathlib.Path(s).stat().st_mtime > t for s in srcs)


def build_pjgen(force: bool = False) -> pathlib.Path:
    LIB.mkdir(exist_ok=True)
    out = LIB / "libmzb_pjgen.so"
    src = CSRC / "pjgen.cpp"
    if force or _stale(out, [src]):
        subprocess.check_call(["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-pthread",
                               str(src), "-o", str(out)])
    return out


def build_cuda(force: bool = False, jobs: int | None = None) -> pathlib.Path:
    LIB.mkdir(exist_ok=True)
    out = LIB / "libmizuba_b200.so"
    srcs = [CSRC / s for s in CUDA_SOURCES]
    deps = srcs + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "mizuba_b200.h"]
    if not (force or _stale(out, deps)):
        return out
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = objdir / (s.stem + ".o")
        objs.append(o)
        procs.append(subprocess.Popen([NVCC, *CUDA_FLAGS, "-c", str(s), "-o", str(o)]))
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("nvcc failed")
    # The CUDA runtime is linked statically so the library loads without a
    # CUDA toolkit on the library path.
    subprocess.check_call([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-cudart", "static", *map(str, objs), "-o", str(out)])
    return out


def build(force: bool = False) -> None:
    build_pjgen(force)
    build_cuda(force)


if __name__ == "__main__":
    build(force=True)
