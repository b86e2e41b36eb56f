"""The C-ABI library builds, loads without a GPU and exports every declared entry point (CPU)."""

from __future__ import annotations

import ctypes
import re
import shutil

import pytest

from conftest import REPO


def _declared() -> set[str]:
    text = (REPO / "include" / "swe_b200.h").read_text()
    return set(re.findall(r"^\s*(?:const\s+)?[a-z0-9_ ]+\**\s*\**(swe_[a-z_0-9]+)\s*\(", text, re.M))


@pytest.fixture(scope="module")
def libpath():
    from hybrid_flood_b200 import build

    if build.is_stale():
        if shutil.which("nvcc") is None and not build.LIB.exists():
            pytest.skip("nvcc unavailable and library not built")
        build.build()
    return build.LIB


def test_header_declares_expected_entry_points():
    from hybrid_flood_b200 import _lib

    assert _declared() == set(_lib.EXPORTS)


def test_library_loads_and_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(str(libpath))
    for name in _declared():
        assert hasattr(lib, name), name
    lib.swe_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.swe_version()


def test_error_path_without_device(libpath):
    """Argument validation runs before any CUDA call and reports through swe_last_error."""
    from hybrid_flood_b200 import _lib

    lib = _lib.load(libpath)
    desc = _lib.DomainDesc()
    desc.rows, desc.cols = 0, 5
    h = ctypes.c_void_p()
    assert lib.swe_domain_create(ctypes.byref(desc), ctypes.byref(h)) == _lib.SWE_ERR_INVALID
    assert "rows and cols" in _lib.last_error()
    with pytest.raises(ValueError):
        _lib.check(_lib.SWE_ERR_INVALID, "x")
    with pytest.raises(RuntimeError):
        _lib.check(_lib.SWE_ERR_MAX_STEPS, "x")


def test_library_is_sm100a_only(libpath):
    """The build flags request sm_100a code only (no PTX for other targets)."""
    from hybrid_flood_b200 import build

    assert build.ARCH_FLAGS == ["-gencode", "arch=compute_100a,code=sm_100a"]
