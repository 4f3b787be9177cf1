"""MD containers: settings, tracked waves, per-lane state, snapshots, trace.

Same names, fields and defaults as ``src/xla_cco/dynamics/state.py:44-172``
of the reference. Arrays are NumPy; a batch carries a leading lane axis on
every array of ``MDState`` (the reference vmaps the same containers).

``MDSettings``: ``dt``; ``scheme`` in SCHEMES; ``andersen_p`` and
``andersen_mode`` in ANDERSEN_MODES; ``gamma`` (BAOAB friction);
``remove_com`` (zero total momentum at ``begin_segment``);
``chunk_steps`` (steps per device call); ``wind_every`` (cadence of the
unconstrained waves' densities); ``record_steps`` (absolute steps of the
snapshots, ascending, at most 256); ``record_rho_every`` /
``max_rho_records`` (dense rho trace, 0: off); ``phase_floor`` on
S = |rho|^2 / N; ``drift_tol`` (plain Verlet stops a lane with STATUS_DRIFT
when |E - e0| > drift_tol * d (N - 1) T / 2; inf: no guard).
"""

from __future__ import annotations

import dataclasses
from typing import Optional, Tuple

import numpy as np

SCHEMES: Tuple[str, ...] = ("verlet", "andersen", "baoab")
ANDERSEN_MODES: Tuple[str, ...] = ("count", "bernoulli")


@dataclasses.dataclass(frozen=True)
class MDSettings:
    dt: float = 0.01
    scheme: str = "verlet"
    andersen_p: float = 0.01
    andersen_mode: str = "count"
    gamma: float = 0.0
    remove_com: bool = True
    chunk_steps: int = 10_000
    wind_every: int = 1
    record_steps: Tuple[int, ...] = ()
    record_rho_every: int = 0
    max_rho_records: int = 0
    phase_floor: float = 1e-16
    drift_tol: float = 1e-3


@dataclasses.dataclass(frozen=True)
class Waves:
    """Tracked waves, constrained first: ``n_vectors`` (w, d) coefficients,
    ``kvec`` (w, d) Cartesian (n 2 pi B^-T), ``constrained`` (w,) flags; the
    first ``n_constrained`` rows equal the energy's first n_vectors."""

    n_vectors: np.ndarray
    kvec: np.ndarray
    constrained: np.ndarray
    n_constrained: int


@dataclasses.dataclass
class Snapshots:
    """Snapshots at ``MDSettings.record_steps`` (``step`` -1: empty slot)."""

    step: np.ndarray
    time: np.ndarray
    wind_abs: np.ndarray
    wind_net: np.ndarray
    rho: np.ndarray
    r: np.ndarray
    phi: np.ndarray
    kinetic: np.ndarray
    count: np.ndarray


@dataclasses.dataclass
class RhoTrace:
    """Dense rho of the tracked waves every ``record_rho_every`` steps."""

    rho: np.ndarray
    time: np.ndarray
    count: np.ndarray


@dataclasses.dataclass
class MDState:
    """One lane (or a batch with a leading lane axis): positions, velocities,
    forces, energy, temperature, PRNG key (uint32[2]), step and time, the
    Andersen accumulator, the winding bookkeeping (``rho_prev`` (w, 2),
    ``wind_abs``, ``wind_net``, ``n_valid``), the segment's energy reference
    ``e0`` and largest drift, running sums since the last reset (``n_sum``
    samples), status (STATUS_RUNNING or STATUS_DRIFT) and the buffers."""

    r: np.ndarray
    v: np.ndarray
    f: np.ndarray
    phi: np.ndarray
    temperature: np.ndarray
    key: np.ndarray
    step: np.ndarray
    time: np.ndarray
    reset_acc: np.ndarray
    rho_prev: np.ndarray
    wind_abs: np.ndarray
    wind_net: np.ndarray
    n_valid: np.ndarray
    e0: np.ndarray
    max_drift: np.ndarray
    sum_kinetic: np.ndarray
    sum_phi: np.ndarray
    sum_phi2: np.ndarray
    sum_s: np.ndarray
    n_sum: np.ndarray
    status: np.ndarray
    snap: Snapshots
    trace: RhoTrace


@dataclasses.dataclass
class MDResult:
    """Final batched state, its snapshots and (if recorded) the rho trace."""

    state: MDState
    snapshots: Snapshots
    trace: Optional[RhoTrace]
