"""L-BFGS with the C++ three-pass rescale schedule (settings and host helpers).

Settings mirror ``xla_cco/minimize/lbfgs.py:55-67``. The iteration runs on the
device (``csrc/cco_opt.cu``): a per-lane state machine that advances one
line-search probe per energy evaluation.

Algorithm (restated; the reference delegates the direction and the line
search to optax 0.2.8, which is not vendored, so the iterates themselves are
not pinned - the schedule, statuses and evaluation accounting are):

* pass p optimizes x = R_p s (R = 1e4, 1, 1e-2); Phi(x) = Phi(x / R),
  dPhi/dx = dPhi/ds / R (``lbfgs.py:75-97``);
* direction: L-BFGS two-loop recursion over the last ``memory`` pairs
  (x_k - x_{k-1}, g_k - g_{k-1}) with rho = 1 / (y.s) (0 when y.s = 0) and the
  initial scaling gamma = (y.s)/(y.y) of the newest pair, or min(1, 1/|g|) on
  the first iteration of a pass (optax ``scale_by_lbfgs``);
* step: zoom line search from an initial step of 1 (Nocedal & Wright
  Alg. 3.5/3.6 with the Hager-Zhang approximate-Wolfe decrease test,
  c1 = 1e-4, c2 = 0.9, eps = 1e-6), at most ``max_linesearch_steps`` probes;
  a search that finds no point with sufficient decrease fails and keeps the
  previous point (``lbfgs.py:200-225,273-276``);
* evaluations per iteration = probes (>= 1); stagnation counter reset on a
  strict decrease (``:228-232``); pass end on budget / stagnation / failure
  advances to the next rescale with the history reset, s carried and
  g rescaled by R/R_next (``:280-301``); global stops energy_tol and
  |g_s| < grad_tol (``:235-254``).
"""

from __future__ import annotations

import dataclasses
from typing import Tuple

import numpy as np

DEFAULT_CHUNK_ITERS: int = 2_000

# line-search constants (optax scale_by_zoom_linesearch defaults)
LS_C1: float = 1e-4
LS_C2: float = 0.9
LS_APPROX_EPS: float = 1e-6
LS_GROW: float = 2.0


@dataclasses.dataclass(frozen=True)
class LBFGSSettings:
    """L-BFGS settings (same names and defaults as the reference)."""

    memory: int = 100
    rescales: Tuple[float, ...] = (1e4, 1.0, 1e-2)
    max_evals_per_pass: int = 500_000
    energy_tol: float = 0.0
    grad_tol: float = 0.0
    stagnation_patience: int = 50
    max_linesearch_steps: int = 30
    record_every: int = 0
    max_records: int = 0
    # Not in the reference: "mixed" evaluates a lane of a d >= 2 problem in
    # FP32 (FP64-seeded tables, compensated FP32 density sums, FP32
    # back-projection) while its energy is above 1e-6 N, then in FP64 for
    # good; every status is judged in FP64. A mixed lane that ends above
    # energy_tol (> 0) runs again from its initial positions in plain FP64, so
    # it returns exactly the plain result; 1-D lanes run FP64 throughout.
    precision: str = "fp64"


def max_rounds(settings: LBFGSSettings, chunk_iters: int) -> int:
    """Upper bound on host rounds (``lbfgs.py:344-350``)."""
    assert chunk_iters >= 1, "chunk_iters must be positive"
    total = len(settings.rescales) * (
        settings.max_evals_per_pass + settings.max_linesearch_steps + 1
    )
    return total // chunk_iters + 2


def update_stagnation(f_new, f_old, stag):
    """Consecutive non-decrease counter: 0 on a strict decrease, else +1."""
    return np.where(np.asarray(f_new) < np.asarray(f_old), 0, np.asarray(stag) + 1)


def lbfgs(energy, s0, settings: LBFGSSettings):
    """Relax one configuration with the three-pass schedule (``lbfgs.py:353-390``)."""
    from xla_cco._types import require_float64
    from xla_cco.minimize import relax

    require_float64(s0, "s0")
    s0 = np.asarray(s0)
    assert s0.ndim == 2, "s0 must have shape (n, d)"
    return relax(energy, s0[None], settings).lane(0)
