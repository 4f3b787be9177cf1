"""MD on the stealthy energy (drop-in for ``xla_cco.dynamics``): integrator
steps, the device segment driver with tracked-wave observables, thermal
helpers and checkpoints."""

from xla_cco.dynamics.checkpoint import CheckpointError, load_state, read_meta, save_state
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
from xla_cco.dynamics.observables import (
    center_of_mass,
    com_correct,
    wave_densities,
    winding_update,
)
from xla_cco.dynamics.run import (
    begin_segment,
    init_state,
    make_waves,
    md_chunk,
    select_dt,
    simulate,
)
from xla_cco.dynamics.state import SCHEMES, MDResult, MDSettings, MDState, RhoTrace, Snapshots, Waves
from xla_cco.dynamics.thermal import (
    harmonic_sample,
    kinetic_energy,
    kinetic_temperature,
    maxwell_boltzmann,
)

__all__ = [
    "ANDERSEN_MODES", "CheckpointError", "MDResult", "MDSettings", "MDState", "MDStepSettings",
    "RhoTrace", "SCHEMES", "Snapshots", "Waves", "andersen_reset", "baoab_step", "begin_segment",
    "center_of_mass", "com_correct", "harmonic_sample", "init_state", "kinetic_energy",
    "kinetic_temperature", "load_state", "make_force_fn", "make_key", "make_waves",
    "maxwell_boltzmann", "md_chunk", "md_run", "read_meta", "save_state", "select_dt",
    "simulate", "verlet_step", "wave_densities", "winding_update",
]  # fmt: skip
