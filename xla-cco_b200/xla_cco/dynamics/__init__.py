"""MD integrator steps on the stealthy energy (drop-in for ``xla_cco.dynamics.integrators``)."""

from xla_cco.dynamics.integrators import (
    ANDERSEN_MODES,
    MDStepSettings,
    andersen_reset,
    baoab_step,
    make_force_fn,
    make_key,
    md_run,
    verlet_step,
)

__all__ = [
    "ANDERSEN_MODES", "MDStepSettings", "andersen_reset", "baoab_step", "make_force_fn",
    "make_key", "md_run", "verlet_step",
]  # fmt: skip
