"""Loads the ``vbcsr_core`` host-core extension built in this package directory
(``python -m vbcsr_b200._build``).  There is no CPU fallback: importing the
Python API without the extension raises."""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
_mod = None


def load():
    global _mod
    if _mod is not None:
        return _mod
    if not any(HERE.glob("vbcsr_core*.so")):
        raise ImportError(
            f"vbcsr_core extension not built in {HERE}; run `python -m vbcsr_b200._build` (needs nvcc and g++)"
        )
    if str(HERE) not in sys.path:
        sys.path.insert(0, str(HERE))
    _mod = importlib.import_module("vbcsr_core")
    return _mod
