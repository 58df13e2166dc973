"""The C ABI library loads and exports every entry point include/vbcsr_b200.h
declares (no compute: runs without a GPU)."""
import re
from pathlib import Path

from vbcsr_b200 import _capi

HEADER = Path(__file__).resolve().parent.parent / "include" / "vbcsr_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(vbg_\w+)\(", text, flags=re.M)))


def test_header_and_binding_agree():
    assert declared_symbols() == _capi.exported_symbols()


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_and_error_string():
    lib = _capi.load()
    assert lib.vbg_version() >= 1
    assert lib.vbg_last_error() is not None
