"""Dataset protocols used by unwrap() (reference cuphu/io/_dataset.py:11-37)."""
from __future__ import annotations

from typing import Protocol, runtime_checkable

import numpy as np


@runtime_checkable
class InputDataset(Protocol):
    """Read-only array-like with ``shape``, ``ndim`` and ``__array__``
    (numpy arrays, rasterio readers, h5py datasets)."""

    @property
    def shape(self) -> tuple[int, ...]: ...

    @property
    def ndim(self) -> int: ...

    def __array__(self, dtype: np.dtype | None = None) -> np.ndarray: ...


@runtime_checkable
class OutputDataset(Protocol):
    """Writable array-like with ``shape`` and ``ndim``; written with ``[...]``."""

    @property
    def shape(self) -> tuple[int, ...]: ...

    @property
    def ndim(self) -> int: ...

    def __array__(self, dtype: np.dtype | None = None) -> np.ndarray: ...
