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
