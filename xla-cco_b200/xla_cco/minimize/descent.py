"""Adaptive normalized gradient descent (C++ ``StructureOptimization`` rule).

Settings mirror ``xla_cco/minimize/descent.py:52-63`` field for field. The
iteration itself runs on the device (``csrc/cco_opt.cu``, descent update
kernel); this module holds the settings, the single-configuration entry point
and the budget arithmetic the reference exposes.

Per iteration (``descent.py:153-175``): |g|, gn = g/|g| (0 if |g| = 0),
xn = s - gn*step, (f2, g2) = value_and_grad(xn); reject iff
|(f - f2) - step|g|| / (step|g|) > rel_tol (a NaN ratio accepts); the step is
multiplied by ``shrink`` on reject and ``grow`` on accept; ``n_evals`` grows by
2 per iteration (C++ budget semantics). Status precedence (``:92-104``):
energy_tol > zero gradient > step floor > budget (it >= max_evals // 2).
"""

from __future__ import annotations

import dataclasses

import numpy as np

DEFAULT_CHUNK_ITERS: int = 2_000


@dataclasses.dataclass(frozen=True)
class DescentSettings:
    """Adaptive-descent settings (same names and defaults as the reference)."""

    step_init: float = 1e-3
    step_min: float = 1e-15
    shrink: float = 0.5
    grow: float = 1.0
    rel_tol: float = 0.01
    max_evals: int = 10_000
    energy_tol: float = 0.0
    record_every: int = 0
    max_records: int = 0


def max_iters(settings: DescentSettings) -> int:
    """Iteration budget ``max_evals // 2`` (odd budgets do not underflow)."""
    return settings.max_evals // 2


def max_rounds(settings: DescentSettings, chunk_iters: int) -> int:
    """Upper bound on host rounds (``descent.py:212-215``)."""
    assert chunk_iters >= 1, "chunk_iters must be positive"
    return max_iters(settings) // chunk_iters + 2


def adaptive_descent(energy, s0, settings: DescentSettings):
    """Relax one configuration by adaptive descent (``descent.py:218-255``).

    Runs the same device path as ``relax`` on a batch of one and returns the
    lane's ``RelaxResult`` (wrapped positions; ``n_evals`` counts 2 per
    iteration).
    """
    from xla_cco._types import require_float64
    from xla_cco.minimize import relax

    require_float64(s0, "s0")
    s0 = np.asarray(s0)
    assert s0.ndim == 2, "s0 must have shape (n, d)"
    return relax(energy, s0[None], settings).lane(0)
