"""DistVector: the reference's Python vector wrapper (vbcsr/vector.py), on the
B200 core.  ``to_numpy()`` returns a view of the core's host mirror (the
reference's contract, vector.py:98-119); writing through it is seen by the next
device operation."""
from __future__ import annotations

from typing import Any, Union

import numpy as np

Scalar = Union[float, complex, int]


def _core_buffer(core) -> np.ndarray:
    return np.array(core, copy=False)


def _dtype_of(core) -> np.dtype:
    return np.dtype(np.complex128) if "Complex" in type(core).__name__ else np.dtype(np.float64)


class DistVector:
    def __init__(self, core_obj: Any, comm: Any = None):
        self._core = core_obj
        self.dtype = _dtype_of(core_obj)
        self.comm = comm

    def _local(self) -> np.ndarray:
        return _core_buffer(self._core)[: self.local_size]

    @property
    def local_size(self) -> int:
        return self._core.local_size

    @property
    def ghost_size(self) -> int:
        return self._core.ghost_size

    @property
    def full_size(self) -> int:
        return self._core.full_size

    @property
    def ndim(self) -> int:
        return 1

    @property
    def shape(self):
        return (self.local_size,)

    @property
    def size(self) -> int:
        return self.local_size

    def __len__(self) -> int:
        return self.local_size

    def __repr__(self):
        return f"<DistVector of size {self.local_size}, dtype={self.dtype}>"

    def to_numpy(self) -> np.ndarray:
        return self._local()

    def from_numpy(self, arr: np.ndarray) -> None:
        if arr.shape != (self.local_size,):
            raise ValueError(f"Array shape {arr.shape} mismatch. Expected ({self.local_size},)")
        self._local()[:] = arr

    def __array__(self, dtype=None, copy=None):
        a = self.to_numpy()
        return a.astype(dtype) if dtype is not None else a

    def sync_ghosts(self) -> None:
        self._core.sync_ghosts()

    def reduce_ghosts(self) -> None:
        self._core.reduce_ghosts()

    def duplicate(self) -> "DistVector":
        return DistVector(self._core.duplicate(), self.comm)

    def copy(self) -> "DistVector":
        return self.duplicate()

    def set_constant(self, val: Scalar) -> None:
        self._core.set_constant(val)

    def set_random(self, seed: int, normalize: bool = True) -> None:
        self._core.set_random(seed, normalize)

    def scale(self, alpha: Scalar) -> None:
        self._core.scale(alpha)

    def axpy(self, alpha: Scalar, x: "DistVector") -> None:
        if not isinstance(x, DistVector):
            raise TypeError("axpy expects DistVector")
        self._core.axpy(alpha, x._core)

    def axpby(self, alpha: Scalar, x: "DistVector", beta: Scalar) -> None:
        if not isinstance(x, DistVector):
            raise TypeError("axpby expects DistVector")
        self._core.axpby(alpha, x._core, beta)

    def pointwise_mult(self, other: "DistVector") -> None:
        if not isinstance(other, DistVector):
            raise TypeError("pointwise_mult expects DistVector")
        self._core.pointwise_mult(other._core)

    def dot(self, other: "DistVector"):
        if not isinstance(other, DistVector):
            raise TypeError("dot expects DistVector")
        return self._core.dot(other._core)

    # operators (vbcsr/vector.py:191-305)
    def __neg__(self):
        r = self.duplicate()
        r._core.scale(-1.0)
        return r

    def __pos__(self):
        return self

    def __add__(self, other):
        r = self.duplicate()
        r += other
        return r

    def __iadd__(self, other):
        if isinstance(other, DistVector):
            self._core.axpy(1.0, other._core)
        elif np.isscalar(other) or isinstance(other, np.ndarray):
            self._local()[:] += other
        else:
            return NotImplemented
        return self

    def __sub__(self, other):
        r = self.duplicate()
        r -= other
        return r

    def __isub__(self, other):
        if isinstance(other, DistVector):
            self._core.axpy(-1.0, other._core)
        elif np.isscalar(other) or isinstance(other, np.ndarray):
            self._local()[:] -= other
        else:
            return NotImplemented
        return self

    def __mul__(self, other):
        r = self.duplicate()
        r *= other
        return r

    def __imul__(self, other):
        if np.isscalar(other):
            self._core.scale(other)
        elif isinstance(other, DistVector):
            self._core.pointwise_mult(other._core)
        elif isinstance(other, np.ndarray):
            self._local()[:] *= other
        else:
            return NotImplemented
        return self

    def __radd__(self, other):
        return self.__add__(other)

    def __rsub__(self, other):
        r = -self
        r += other
        return r

    def __rmul__(self, other):
        return self.__mul__(other)

    def __truediv__(self, other):
        r = self.duplicate()
        r /= other
        return r

    def __itruediv__(self, other):
        if np.isscalar(other):
            self._core.scale(1.0 / other)
        elif isinstance(other, DistVector):
            self._local()[:] /= other.to_numpy()
        elif isinstance(other, np.ndarray):
            self._local()[:] /= other
        else:
            return NotImplemented
        return self
