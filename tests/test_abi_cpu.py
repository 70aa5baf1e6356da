"""The C-ABI library loads without a GPU and exports every entry point that
include/gjxl_b200.h declares (no compute calls here)."""

import ctypes
import re
from pathlib import Path

from gjxl_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "gjxl_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"GJXL_B200_API[^;(]*?\b(gjxl_b200_\w+)\s*\(", text, re.S)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "gjxl_b200_prepare_input" in names and len(names) >= 4


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIBRARY_PATH))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_version_and_error_string_work_without_gpu():
    lib = _lib.load()
    assert lib.gjxl_b200_version() >= 100
    assert lib.gjxl_b200_last_error() is not None


def test_failure_injection_arming_is_validated_without_gpu():
    """gjxl_b200_test_arm_failure is host-only: valid kinds arm and disarm,
    unknown kinds and negative check points are rejected."""
    lib = _lib.load()
    for kind in (1, 2, 3):
        assert lib.gjxl_b200_test_arm_failure(kind, 0) == 0
    assert lib.gjxl_b200_test_arm_failure(0, 1) == 1
    assert lib.gjxl_b200_test_arm_failure(4, 1) == 1
    assert lib.gjxl_b200_test_arm_failure(1, -1) == 1


def test_integration_binding_loads_without_gpu():
    """The reference-side binding (integration/, built with the reference's
    sources when they are present) loads and exports its entry points."""
    import pytest
    path = HEADER.parent.parent / "integration" / "_build" / "libgjxl_b200_encoder.so"
    if not path.exists():
        pytest.skip("integration binding not built (reference sources absent)")
    lib = ctypes.CDLL(str(path))
    assert hasattr(lib, "gjxl_b200_encode_image")
    assert hasattr(lib, "gjxl_b200_integration_last_error")
