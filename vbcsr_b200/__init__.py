"""vbcsr_b200: the VBCSR variable-block sparse hot path on one NVIDIA B200.

Python API (mirrors the reference package ``vbcsr``): :class:`VBCSR`,
:class:`DistVector`, :class:`DistMultiVector`, ``DistGraph``, ``AssemblyMode``;
Chebyshev/KPM helpers in :mod:`vbcsr_b200.utils` and :mod:`vbcsr_b200.kpm`,
McWeeny purification in :mod:`vbcsr_b200.purification`, Chebyshev time
propagation in :mod:`vbcsr_b200.propagation`.

The numeric work runs in the CUDA library ``libvbcsr_b200.so`` (C ABI in
include/vbcsr_b200.h) under the ``vbcsr_core`` host core; both are built in
place by ``python -m vbcsr_b200._build``.  Submodules import lazily, so
``import vbcsr_b200`` works before the extensions exist (the build imports it).
"""
__version__ = "0.1.0"

_LAZY = {
    "VBCSR": ("matrix", "VBCSR"),
    "DistVector": ("vector", "DistVector"),
    "DistMultiVector": ("multivector", "DistMultiVector"),
}


def __getattr__(name):
    if name in _LAZY:
        import importlib

        mod, attr = _LAZY[name]
        return getattr(importlib.import_module(f".{mod}", __name__), attr)
    if name in ("DistGraph", "AssemblyMode", "RedistOp"):
        from . import _core

        return getattr(_core.load(), name)
    raise AttributeError(name)


__all__ = ["VBCSR", "DistVector", "DistMultiVector", "DistGraph", "AssemblyMode", "RedistOp"]
