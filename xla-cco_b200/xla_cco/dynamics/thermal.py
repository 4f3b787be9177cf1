"""Thermal helpers (``src/xla_cco/dynamics/thermal.py:38-153``): kinetic energy
and temperature, Maxwell-Boltzmann velocities, harmonic ground-state draws.

Velocities use the Philox4x32-10 normals of the integrators (stream 9,
index = element) instead of JAX's threefry: same distribution, other draws.
"""

from __future__ import annotations

import math
from typing import Any

import numpy as np

from xla_cco._types import require_float64
from xla_cco.dynamics.integrators import _normal, _philox

_MB_STREAM = 9


def require_key(key: Any) -> None:
    """``TypeError`` unless ``key`` is a uint32 array of shape (2,)."""
    if getattr(key, "dtype", None) != np.uint32 or getattr(key, "shape", ()) != (2,):
        raise TypeError("key must be a raw uint32 PRNG key of shape (2,)")


def maxwell_boltzmann(key: np.ndarray, n: int, d: int, temperature: float,
                      remove_com: bool) -> np.ndarray:  # fmt: skip
    """(n, d) velocities ~ N(0, T) per component; mean removed if ``remove_com``."""
    if n < 1 or d < 1:
        raise ValueError(f"n and d must be positive, got n={n}, d={d}")
    require_key(key)
    xi = _normal(_philox(key, _MB_STREAM, np.arange(n * d))).reshape(n, d)
    v = math.sqrt(float(temperature)) * xi
    if remove_com:
        v = v - np.mean(v, axis=0, keepdims=True)
    return v


def kinetic_energy(v: np.ndarray) -> np.ndarray:
    """sum_j |v_j|^2 / 2 (mass 1); a batch (b, n, d) gives (b,)."""
    require_float64(v, "v")
    assert v.ndim >= 2, "v must have shape (n, d) or (b, n, d)"
    return 0.5 * np.sum(v * v, axis=(-2, -1))


def kinetic_temperature(v: np.ndarray, dof: int) -> np.ndarray:
    """2 KE / dof (dof = d (n - 1) without centre-of-mass motion)."""
    if dof < 1:
        raise ValueError(f"dof must be positive, got {dof}")
    return 2.0 * kinetic_energy(v) / dof


def _cartesian_hessian(energy: Any, s: np.ndarray, basis: np.ndarray) -> np.ndarray:
    """d^2 Phi / dr dr at r = s B: (I x B^-1) H_s (I x B^-1)^T, symmetrised."""
    n, d = s.shape
    if basis.shape != (d, d) or not np.isfinite(basis).all():
        raise ValueError(f"basis must be a finite ({d}, {d}) array")
    inv = np.linalg.inv(basis)
    h_s = np.asarray(energy.hessian(np.ascontiguousarray(s)))
    h = np.einsum("ac,jcle,be->jalb", inv, h_s.reshape(n, d, n, d), inv).reshape(n * d, n * d)
    return 0.5 * (h + h.T)


def harmonic_sample(rng: np.random.Generator, energy: Any, s_gs: np.ndarray, basis: np.ndarray,
                    temperature: float, zero_rel: float = 1e-9) -> np.ndarray:  # fmt: skip
    """Ground state plus a canonical harmonic displacement (Cartesian, unwrapped).

    Modes of the Cartesian Hessian (from the device Hessian) with
    lambda > zero_rel lambda_max get amplitude N(0, T / lambda), drawn with one
    ``rng.standard_normal(k)`` in ascending eigenvalue order; the others none.
    """
    if not (math.isfinite(temperature) and temperature >= 0.0):
        raise ValueError(f"temperature must be finite and >= 0, got {temperature}")
    if not isinstance(rng, np.random.Generator):
        raise TypeError("rng must be a numpy.random.Generator")
    s = np.asarray(s_gs, dtype=np.float64)
    b = np.asarray(basis, dtype=np.float64)
    if s.ndim != 2:
        raise ValueError(f"s_gs must have shape (n, d), got {s.shape}")
    lam, vec = np.linalg.eigh(_cartesian_hessian(energy, s, b))
    if not lam[-1] > 0.0:
        raise ValueError("Hessian has no positive eigenvalue")
    keep = lam > zero_rel * lam[-1]
    amp = np.sqrt(temperature / lam[keep]) * rng.standard_normal(int(keep.sum()))
    return s @ b + (vec[:, keep] @ amp).reshape(s.shape)
