"""Seeded synthetic workloads of the mixed-size batch and the request stream.

There is no public dataset for this path; the reference draws uniform
fractional positions from ``np.random.default_rng(seed).uniform`` (its
``tests/conftest.py`` and ``bench_energy.py``), in a cubic unit-density box
with packing fraction 0.05 and the k-set of ``enumerate_kvectors(basis, 0,
k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))``. These generators keep
that convention and fix the order in which one seed drives the instance
parameters, so a run is reproducible from its seed alone:

* ``mixed_ensemble``: per instance N = round(exp(U[ln n_lo, ln n_hi])),
  d uniform over ``dims``, chi = U[chi_lo, chi_hi], then the (N, d) positions.
* ``request_stream``: the same per request, preceded by an exponential
  inter-arrival time of mean 1 / rate.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Sequence, Tuple

import numpy as np

from xla_cco.box import cubic_box
from xla_cco.energy import StealthyEnergy, make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi

PHI_PACK = 0.05

__all__ = ["Instance", "mixed_ensemble", "request_stream", "energy_for"]


@dataclass
class Instance:
    n: int
    d: int
    chi: float
    energy: StealthyEnergy
    s0: np.ndarray          # (n, d) float64
    arrival_s: float = 0.0  # request streams only: arrival time from the start

    @property
    def m(self) -> int:
        """Real k-vectors (padding rows excluded)."""
        return int(self.energy._rows.size)


def energy_for(n: int, d: int, chi: float, cache: Dict[Tuple[int, int, float], StealthyEnergy]
               | None = None) -> StealthyEnergy:  # fmt: skip
    """The stealthy energy of N particles in d dimensions at chi (cached by key)."""
    key = (int(n), int(d), float(chi))
    if cache is not None and key in cache:
        return cache[key]
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, PHI_PACK, d), PHI_PACK, d))
    en = make_stealthy_energy(box, ks)
    if cache is not None:
        cache[key] = en
    return en


def _draw(rng: np.random.Generator, n_lo: int, n_hi: int, dims: Sequence[int], chi_lo: float,
          chi_hi: float) -> Tuple[int, int, float]:  # fmt: skip
    n = int(round(float(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))))
    d = int(dims[int(rng.integers(0, len(dims)))])
    chi = float(rng.uniform(chi_lo, chi_hi))
    return n, d, chi


def mixed_ensemble(count: int = 512, seed: int = 0, n_lo: int = 200, n_hi: int = 8000,
                   dims: Sequence[int] = (1, 2, 3), chi_lo: float = 0.05,
                   chi_hi: float = 0.49) -> List[Instance]:  # fmt: skip
    """Instances of uneven N, d and chi (defaults: 512, N in [200, 8000], d in {1,2,3})."""
    rng = np.random.default_rng(seed)
    cache: Dict[Tuple[int, int, float], StealthyEnergy] = {}
    out = []
    for _ in range(count):
        n, d, chi = _draw(rng, n_lo, n_hi, dims, chi_lo, chi_hi)
        en = energy_for(n, d, chi, cache)
        out.append(Instance(n, d, chi, en, rng.uniform(size=(n, d))))
    return out


def request_stream(count: int = 20000, seed: int = 0, rate: float = 200.0, n_lo: int = 100,
                   n_hi: int = 20000, dims: Sequence[int] = (2, 3), chi_lo: float = 0.10,
                   chi_hi: float = 0.45) -> List[Instance]:  # fmt: skip
    """A Poisson arrival stream (defaults: 200 req/s, N in [100, 20000], d in {2, 3})."""
    rng = np.random.default_rng(seed)
    cache: Dict[Tuple[int, int, float], StealthyEnergy] = {}
    t = 0.0
    out = []
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate))
        n, d, chi = _draw(rng, n_lo, n_hi, dims, chi_lo, chi_hi)
        en = energy_for(n, d, chi, cache)
        out.append(Instance(n, d, chi, en, rng.uniform(size=(n, d)), arrival_s=t))
    return out
