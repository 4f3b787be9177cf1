"""Analysis of relaxed ensembles: structure factor and pair statistics."""

from xla_cco.analysis.pairs import (
    g2_from_histogram,
    nearest_neighbor_distances,
    pair_distance_histogram,
)
from xla_cco.analysis.structure import isotropic_structure_factor, structure_factor

__all__ = ["g2_from_histogram", "isotropic_structure_factor", "nearest_neighbor_distances",
           "pair_distance_histogram", "structure_factor"]  # fmt: skip
