"""DistMultiVector: the reference's Python multivector wrapper
(vbcsr/multivector.py) on the B200 core.  Row-major with a padded leading
dimension; ``to_numpy()`` is a strided view of the host mirror."""
from __future__ import annotations

from typing import Any

import numpy as np

from .vector import DistVector, _core_buffer, _dtype_of


class DistMultiVector:
    def __init__(self, core_obj: Any, comm: Any = None):
        self._core = core_obj
        self.dtype = _dtype_of(core_obj)
        self.comm = comm

    def _local(self) -> np.ndarray:
        return _core_buffer(self._core)[: self.local_rows, :]

    @property
    def local_rows(self) -> int:
        return self._core.local_rows

    @property
    def ghost_rows(self) -> int:
        return self._core.ghost_rows

    @property
    def num_vectors(self) -> int:
        return self._core.num_vectors

    @property
    def ndim(self) -> int:
        return 2

    @property
    def shape(self):
        return (self.local_rows, self.num_vectors)

    @property
    def size(self) -> int:
        return self.local_rows * self.num_vectors

    def __len__(self) -> int:
        return self.local_rows

    def __repr__(self):
        return f"<DistMultiVector of shape ({self.local_rows}, {self.num_vectors}), dtype={self.dtype}>"

    def reset_comm_stats(self) -> None:
        self._core.reset_comm_stats()

    @property
    def comm_seconds(self) -> float:
        return self._core.comm_seconds

    @property
    def comm_calls(self) -> int:
        return self._core.comm_calls

    def to_numpy(self) -> np.ndarray:
        return self._local()

    def from_numpy(self, arr: np.ndarray) -> None:
        if arr.shape != (self.local_rows, self.num_vectors):
            raise ValueError(f"Array shape {arr.shape} mismatch. Expected ({self.local_rows}, {self.num_vectors})")
        self._local()[:] = arr

    def __array__(self, dtype=None, copy=None):
        a = self.to_numpy()
        return a.astype(dtype) if dtype is not None else a

    def sync_ghosts(self) -> None:
        self._core.sync_ghosts()

    def reduce_ghosts(self) -> None:
        self._core.reduce_ghosts()

    def duplicate(self) -> "DistMultiVector":
        return DistMultiVector(self._core.duplicate(), self.comm)

    def copy(self) -> "DistMultiVector":
        return self.duplicate()

    def set_constant(self, val) -> None:
        self._core.set_constant(val)

    def set_random(self, seed: int, normalize: bool = True) -> None:
        self._core.set_random(seed, normalize)

    def scale(self, alpha) -> None:
        self._core.scale(alpha)

    def axpy(self, alpha, x: "DistMultiVector") -> None:
        if not isinstance(x, DistMultiVector):
            raise TypeError("axpy expects DistMultiVector")
        self._core.axpy(alpha, x._core)

    def axpby(self, alpha, x: "DistMultiVector", beta) -> None:
        if not isinstance(x, DistMultiVector):
            raise TypeError("axpby expects DistMultiVector")
        self._core.axpby(alpha, x._core, beta)

    def pointwise_mult(self, other) -> None:
        if isinstance(other, DistMultiVector):
            self._core.pointwise_mult(other._core)
        elif isinstance(other, DistVector):
            self._core.pointwise_mult_vec(other._core)
        else:
            raise TypeError("pointwise_mult expects DistMultiVector or DistVector")

    def bdot(self, other: "DistMultiVector") -> list:
        if not isinstance(other, DistMultiVector):
            raise TypeError("bdot expects DistMultiVector")
        return self._core.bdot(other._core)

    # operators (vbcsr/multivector.py:191-274)
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
        if isinstance(other, DistMultiVector):
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
        if isinstance(other, DistMultiVector):
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
        elif isinstance(other, DistMultiVector):
            self._core.pointwise_mult(other._core)
        elif isinstance(other, DistVector):
            self._core.pointwise_mult_vec(other._core)
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
        elif isinstance(other, DistMultiVector):
            self._local()[:] /= other.to_numpy()
        elif isinstance(other, DistVector):
            self._local()[:] /= other.to_numpy()[:, None]
        elif isinstance(other, np.ndarray):
            self._local()[:] /= other
        else:
            return NotImplemented
        return self
