"""CPU-side checks of the C ABI boundary (no device calls)."""

import ctypes as ct
import pathlib
import re
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "mizuba_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(mzb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    from mizuba_b200 import build

    return build.build_cuda()  # rebuilds only when a source is newer than the library


def test_library_loads_and_exports_every_declared_symbol(lib_path):
    lib = ct.CDLL(str(lib_path))
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(mzb_[a-z0-9_]+)\b", out))
    assert set(syms) <= exported


def test_no_cpu_fallback_in_product_path():
    # The product package never imports the oracle.
    for p in (ROOT / "mizuba_b200").rglob("*.py"):
        assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\w+)", p.read_text(), re.M), p
