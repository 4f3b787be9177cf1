"""xla_cco (B200 build): collective-coordinate hot path on sm_100a.

Drop-in for the relaxation path of the reference package ``xla_cco``
(``src/xla_cco/__init__.py:54-100``): the same names for the k-set, box,
energy and minimizer API. Everything is float64; computation runs in the
hand-written CUDA kernels of ``libcco.so`` (no CPU fallback).
"""

from xla_cco._types import require_float64
from xla_cco.analysis.pairs import (
    g2_from_histogram,
    nearest_neighbor_distances,
    pair_distance_histogram,
)
from xla_cco.analysis.structure import isotropic_structure_factor, structure_factor
from xla_cco.box import Box, cubic_box, wrap_fractional
from xla_cco.energy import (
    AbstractEnergy,
    StealthyEnergy,
    collective_density,
    make_stealthy_energy,
)
from xla_cco.io.configpack import (
    PackedConfig,
    read_configpack,
    stack_fractional,
    write_configpack,
)
from xla_cco.io.tables import write_function_table
from xla_cco.kvectors import (
    KSet,
    chi_from_count,
    enumerate_kvectors,
    k_outer_from_ka,
    ka_from_chi,
    unit_ball_volume,
)
from xla_cco.minimize import relax, relax_mixed
from xla_cco.minimize.descent import DescentSettings, adaptive_descent
from xla_cco.minimize.lbfgs import LBFGSSettings, lbfgs
from xla_cco.minimize.result import RelaxResult, Trajectory

__all__ = [
    "AbstractEnergy",
    "Box",
    "DescentSettings",
    "KSet",
    "LBFGSSettings",
    "PackedConfig",
    "RelaxResult",
    "StealthyEnergy",
    "Trajectory",
    "adaptive_descent",
    "chi_from_count",
    "collective_density",
    "cubic_box",
    "enumerate_kvectors",
    "g2_from_histogram",
    "isotropic_structure_factor",
    "k_outer_from_ka",
    "ka_from_chi",
    "lbfgs",
    "make_stealthy_energy",
    "nearest_neighbor_distances",
    "pair_distance_histogram",
    "read_configpack",
    "relax",
    "relax_mixed",
    "require_float64",
    "stack_fractional",
    "structure_factor",
    "unit_ball_volume",
    "wrap_fractional",
    "write_configpack",
    "write_function_table",
]
