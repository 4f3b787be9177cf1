"""dtype guards shared by the host API.

Positions are fractional coordinates of a box basis (rows are lattice vectors),
nominally in [0, 1); every array the kernels consume is float64.

Error convention follows ``xla_cco/_types.py:34-52`` of the reference: a
non-float64 array raises ``TypeError`` before any device work is issued.
"""

from __future__ import annotations

from typing import Any

import numpy as np


def require_float64(x: Any, name: str) -> None:
    """Raise ``TypeError`` unless ``x`` has dtype float64.

    Accepts NumPy arrays and anything exposing ``dtype`` (torch tensors
    included: ``torch.float64`` is compared by name).
    """
    assert isinstance(name, str), "name must be a string"
    dtype = getattr(x, "dtype", None)
    if dtype is None:
        raise TypeError(f"{name} must be float64, got dtype {dtype}")
    if isinstance(dtype, np.dtype) or isinstance(dtype, type):
        ok = np.dtype(dtype) == np.float64
    else:  # torch.dtype and friends
        ok = str(dtype) in ("torch.float64", "float64")
    if not ok:
        raise TypeError(f"{name} must be float64, got dtype {dtype}")
