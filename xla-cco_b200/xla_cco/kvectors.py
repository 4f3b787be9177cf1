"""Host-side construction of the stealthy half-space k-set (bit-exact contract).

Mirror of ``xla_cco/kvectors.py:33-169``. The k-set is the product's only
bit-exact output besides integer bookkeeping, so the floating-point steps are
kept in the same order as the reference (which follows the C++ engine):

* per-axis scan bound ``ceil(K2 |a_i| / 2 pi) + 1`` (``kvectors.py:75-78``);
* half-space rule: the first nonzero component of n is positive (``:119-126``);
* k_j = sum_i n_i recip[i, j] accumulated in index order, |k|^2 likewise
  (``:82-88``), with recip = 2 pi inv(B)^T from ``numpy.linalg.inv``;
* strict shell test K1^2 < |k|^2 < K2^2 (``:89``);
* order by (|k|^2, n_0, n_1, ...) (``:91-93``); unit weights (``:98``).

The scan is written over a flattened index grid rather than a meshgrid stack,
but the arithmetic each surviving row sees is the same sequence of IEEE
operations, which is what the bit-exact tests pin.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass(frozen=True)
class KSet:
    """Half-space k-vectors with K1^2 < |k|^2 < K2^2.

    n: (M, d) int64 reciprocal-basis coefficients; k: (M, d) float64 Cartesian
    vectors; k_sq: (M,) float64 squared moduli; weights: (M,) float64 (ones);
    k_inner, k_outer: the cutoffs K1, K2.
    """

    n: np.ndarray
    k: np.ndarray
    k_sq: np.ndarray
    weights: np.ndarray
    k_inner: float
    k_outer: float


def _check_inputs(basis: np.ndarray, k_inner: float, k_outer: float) -> None:
    """``ValueError`` for a malformed basis or cutoff pair (``kvectors.py:104-116``)."""
    if basis.ndim != 2 or basis.shape[0] != basis.shape[1] or basis.shape[0] < 1:
        raise ValueError(f"basis must be square (d, d), got {basis.shape}")
    finite = bool(np.all(np.isfinite(basis))) and math.isfinite(k_inner)
    if not (finite and math.isfinite(k_outer)):
        raise ValueError("basis and cutoffs must be finite")
    if not 0.0 <= k_inner < k_outer:
        raise ValueError(f"need 0 <= k_inner < k_outer, got {k_inner}, {k_outer}")
    det = float(np.linalg.det(basis))
    if not abs(det) > 0.0 or not math.isfinite(det):
        raise ValueError("basis must have positive |det|")


def _half_space(n: np.ndarray) -> np.ndarray:
    """Mask of rows whose first nonzero coefficient is positive."""
    keep = np.zeros(n.shape[0], dtype=bool)
    open_ = np.ones(n.shape[0], dtype=bool)
    for col in range(n.shape[1]):
        keep |= open_ & (n[:, col] > 0)
        open_ &= n[:, col] == 0
    return keep


def enumerate_kvectors(basis: np.ndarray, k_inner: float, k_outer: float) -> KSet:
    """Enumerate the half-space k-set of a periodic box.

    ``basis`` is (d, d) float64 with lattice vectors as rows; ``k_inner`` and
    ``k_outer`` are the strict cutoffs K1 < K2 (inverse length).
    """
    basis = np.asarray(basis, dtype=np.float64)
    _check_inputs(basis, k_inner, k_outer)
    dim = basis.shape[0]
    recip = 2.0 * math.pi * np.linalg.inv(basis).T
    bound = [
        int(math.ceil(k_outer * float(np.linalg.norm(basis[i])) / (2.0 * math.pi))) + 1
        for i in range(dim)
    ]
    # every integer vector of the box [-b_i, b_i], row-major (last axis fastest)
    sides = [2 * b + 1 for b in bound]
    flat = np.arange(int(np.prod(sides)), dtype=np.int64)
    n = np.empty((flat.size, dim), dtype=np.int64)
    for i in range(dim - 1, -1, -1):
        n[:, i] = flat % sides[i] - bound[i]
        flat //= sides[i]
    n = n[_half_space(n)]
    k = np.zeros((n.shape[0], dim))
    for j in range(dim):
        for i in range(dim):  # fixed summation order (no BLAS reassociation)
            k[:, j] = k[:, j] + n[:, i] * recip[i, j]
    k_sq = np.zeros(n.shape[0])
    for i in range(dim):
        k_sq = k_sq + k[:, i] * k[:, i]
    keep = (k_inner * k_inner < k_sq) & (k_sq < k_outer * k_outer)
    n, k, k_sq = n[keep], k[keep], k_sq[keep]
    keys = tuple(n[:, i] for i in range(dim - 1, -1, -1)) + (k_sq,)
    order = np.lexsort(keys)  # last key primary: |k|^2, then n_0, n_1, ...
    n, k, k_sq = n[order], k[order], k_sq[order]
    return KSet(
        n=n,
        k=k,
        k_sq=k_sq,
        weights=np.ones(n.shape[0]),
        k_inner=float(k_inner),
        k_outer=float(k_outer),
    )


# The C++ engine hard-codes the unit-ball volume for d <= 4 (HyperSphere_C);
# these are those literals rounded to double, as in ``kvectors.py:131-136``.
_UNIT_BALL = {1: 2.0, 2: math.pi, 3: 4.1887902047863909846, 4: 4.9348022005446793094}


def unit_ball_volume(dim: int) -> float:
    """Volume V_d(1) of the unit d-ball, equal to the C++ constants for d <= 4."""
    assert dim >= 1, "dim must be >= 1"
    if dim in _UNIT_BALL:
        return _UNIT_BALL[dim]
    return float(math.pi ** (dim / 2.0) / math.gamma(dim / 2.0 + 1.0))


def k_outer_from_ka(ka: float, phi: float, dim: int) -> float:
    """K2 = Ka / a with a = (phi / V_d(1))^(1/d) (``kvectors.py:152-156``)."""
    assert phi > 0.0 and dim >= 1, "need phi > 0 and dim >= 1"
    a = (phi / unit_ball_volume(dim)) ** (1.0 / dim)
    return float(ka / a)


def ka_from_chi(chi: float, phi: float, dim: int) -> float:
    """Ka = (2^(d+1) d chi Gamma(d/2+1)^2 phi)^(1/d) (``kvectors.py:159-163``)."""
    assert chi >= 0.0 and phi > 0.0 and dim >= 1, "need chi >= 0, phi > 0, dim >= 1"
    arg = 2.0 ** (dim + 1) * dim * chi * math.gamma(dim / 2.0 + 1.0) ** 2 * phi
    return float(arg ** (1.0 / dim))


def chi_from_count(m: int, n_particles: int, dim: int) -> float:
    """chi = M / (d (N - 1)) for M half-space constraints (``kvectors.py:166-169``)."""
    assert n_particles >= 2 and dim >= 1, "need N >= 2 and dim >= 1"
    return float(m / (dim * (n_particles - 1)))
