"""Periodic simulation box: fractional/Cartesian maps and the reciprocal basis.

Host-side mirror of ``xla_cco/box.py:34-139``. ``basis`` rows are lattice
vectors a_i (density 1: the cubic box is N^(1/d) times the unit basis and
V = N). Reciprocal rows satisfy b_i . a_j = 2 pi delta_ij. Everything here is
small (d x d or N x d) NumPy arithmetic on the host; the kernels only ever see
the volume and the integer k-set.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from xla_cco._types import require_float64


@dataclasses.dataclass(frozen=True)
class Box:
    """Periodic box defined by a (d, d) float64 lattice basis (rows = a_i)."""

    basis: np.ndarray

    def __post_init__(self) -> None:
        require_float64(self.basis, "basis")
        b = np.asarray(self.basis)
        if b.ndim != 2 or b.shape[0] != b.shape[1]:
            raise ValueError(f"basis must be square (d, d), got {b.shape}")

    @property
    def dim(self) -> int:
        """Spatial dimension d."""
        return int(np.asarray(self.basis).shape[0])

    @property
    def volume(self) -> float:
        """Box volume |det(basis)| (``box.py:50-53``)."""
        return float(abs(np.linalg.det(np.asarray(self.basis))))

    def reciprocal(self) -> np.ndarray:
        """Rows b_i with b_i . a_j = 2 pi delta_ij (``box.py:55-58``)."""
        return 2.0 * np.pi * np.linalg.inv(np.asarray(self.basis)).T

    def to_cartesian(self, s: np.ndarray) -> np.ndarray:
        """r = s @ basis (``box.py:60-71``)."""
        require_float64(s, "s")
        return np.asarray(s) @ np.asarray(self.basis)

    def to_fractional(self, r: np.ndarray) -> np.ndarray:
        """s = r @ inv(basis) (``box.py:73-84``)."""
        require_float64(r, "r")
        return np.asarray(r) @ np.linalg.inv(np.asarray(self.basis))

    def cartesian_forces(self, grad_s: np.ndarray) -> np.ndarray:
        """F = -grad_s @ inv(B).T, the C++ force (``box.py:86-97``)."""
        require_float64(grad_s, "grad_s")
        return -np.asarray(grad_s) @ np.linalg.inv(np.asarray(self.basis)).T


def cubic_box(n_particles: int, dim: int) -> Box:
    """Cubic box of side N^(1/d) (density 1, V = N) (``box.py:111-124``)."""
    assert n_particles >= 1, "n_particles must be >= 1"
    assert dim in (1, 2, 3), "dim must be 1, 2 or 3"
    side = float(n_particles) ** (1.0 / dim)
    return Box(basis=np.asarray(side * np.eye(dim), dtype=np.float64))


_BELOW_ONE = float(np.nextafter(1.0, 0.0))


def wrap_fractional(s: np.ndarray) -> np.ndarray:
    """Wrap fractional coordinates into [0, 1) (``box.py:127-139``).

    s - floor(s) rounds to exactly 1.0 for tiny negative s, so the result is
    clamped to the largest double below 1.
    """
    require_float64(s, "s")
    a = np.asarray(s)
    return np.minimum(a - np.floor(a), _BELOW_ONE)
