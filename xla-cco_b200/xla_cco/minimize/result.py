"""Result containers and per-lane status codes of the minimizers.

Codes and field names follow ``xla_cco/minimize/result.py:35-75``:
0 running, 1 energy below tolerance, 2 step below floor, 3 evaluation budget
exhausted, 4 stagnated, 5 line-search failure, 6 gradient below tolerance,
7 MD energy drift. The device kernels write the same integers into an int64
status array (``include/cco.h`` defines them as ``CCO_STATUS_*``).
"""

from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

STATUS_RUNNING: int = 0
STATUS_ENERGY_TOL: int = 1
STATUS_STEP_FLOOR: int = 2
STATUS_BUDGET: int = 3
STATUS_STAGNATED: int = 4
STATUS_LINESEARCH_FAIL: int = 5
STATUS_GRAD_TOL: int = 6
STATUS_DRIFT: int = 7
STATUS_CANCELLED: int = 8  # serving pool only (no reference counterpart)


@dataclasses.dataclass
class Trajectory:
    """Recorded trajectory: ``count`` valid rows of a fixed capacity.

    ``s`` rows are wrapped into [0, 1) (``_loop.py:70-84``).
    """

    s: np.ndarray
    energy: np.ndarray
    step: np.ndarray
    iteration: np.ndarray
    count: np.ndarray


@dataclasses.dataclass
class RelaxResult:
    """Outcome of a relaxation; batched results carry a leading lane axis."""

    s: np.ndarray
    energy: np.ndarray
    grad_norm: np.ndarray
    n_evals: np.ndarray
    n_iters: np.ndarray
    status: np.ndarray
    trajectory: Optional[Trajectory]

    def lane(self, i: int) -> "RelaxResult":
        """Lane ``i`` of a batched result (the reference uses tree_map(x[i]))."""
        traj = None
        if self.trajectory is not None:
            t = self.trajectory
            traj = Trajectory(t.s[i], t.energy[i], t.step[i], t.iteration[i], t.count[i])
        return RelaxResult(
            self.s[i], self.energy[i], self.grad_norm[i], self.n_evals[i],
            self.n_iters[i], self.status[i], traj,
        )  # fmt: skip
