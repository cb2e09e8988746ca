"""The C ABI library loads and exports every symbol include/oneline_cuda.h declares (CPU only)."""
import ctypes
import os
import re

from oneline_b200 import _lib
from oneline_b200.build import build_cuda

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols() -> set[str]:
    text = open(os.path.join(ROOT, "include", "oneline_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(ol_[a-z0-9_]+)\s*\(", text))


def test_library_builds_and_loads():
    path = build_cuda()
    assert os.path.exists(path)
    ctypes.CDLL(path)


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(build_cuda())
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert header_symbols() == set(_lib.SIGNATURES), header_symbols() ^ set(_lib.SIGNATURES)


def test_pattern_validation_mirrors_the_reference():
    """search.rs:41-46: 1..=64 bytes on the drop-in search; errors carry the status."""
    from oneline_b200.gpu import GpuParser
    from oneline_b200 import OnelineError
    import pytest

    for bad in (b"", b"a" * 65):
        with pytest.raises(OnelineError):
            GpuParser._check_pattern(bad, 64)
    assert GpuParser._check_pattern(b"a" * 64, 64) == b"a" * 64
    assert GpuParser._check_pattern(b"a" * 1024, None) == b"a" * 1024
