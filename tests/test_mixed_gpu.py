"""Mixed batches: lanes of different N, d and k-set relaxed in one device run.

The reference relaxes one (energy, batch) pair per call
(``minimize/__init__.py:102-151``); its contract that a lane's result does
not depend on the rest of the batch (``tests/integration/test_relax.py``,
per-lane stopping and freezing) is what these tests hold the mixed entry
points to: every lane of a mixed run must equal, bit for bit, the same
configuration relaxed alone through ``relax``. Energies are also checked
against the oracle's direct sum.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import RTOL_KERNEL_E, energy_atol
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize import relax, relax_mixed
from xla_cco.minimize.descent import DescentSettings
from xla_cco.minimize.lbfgs import LBFGSSettings

pytestmark = pytest.mark.gpu

FIELDS = ("s", "energy", "grad_norm", "n_evals", "n_iters", "status")


def _instances(count: int, seed: int):
    """Seeded instances with N in [40, 400], d in {1, 2, 3}, chi in [0.05, 0.45]."""
    rng = np.random.default_rng(seed)
    cache = {}
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(40), np.log(400))))
        d = int(rng.integers(1, 4))
        chi = round(float(rng.uniform(0.05, 0.45)), 2)
        key = (n, d, chi)
        if key not in cache:
            box = cubic_box(n, d)
            ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
            cache[key] = (box, ks, make_stealthy_energy(box, ks))
        out.append((cache[key], rng.uniform(size=(n, d))))
    return out


def _assert_lane_equal(mixed, alone, i):
    for f in FIELDS:
        a, b = np.asarray(getattr(mixed, f)), np.asarray(getattr(alone, f))
        assert np.array_equal(a, b), f"lane {i}: field {f} differs from the lone run"


@pytest.mark.parametrize("which", ["lbfgs", "descent"])
def test_mixed_lanes_equal_lone_runs(which):
    inst = _instances(12, seed=7)
    if which == "lbfgs":
        st = LBFGSSettings(energy_tol=1e-20, max_evals_per_pass=4000)
    else:
        st = DescentSettings(max_evals=400, grow=2.0)
    res = relax_mixed([e for (_, _, e), _ in inst], [s for _, s in inst], st)
    assert len(res) == len(inst)
    for i, (((_, ks, en), s0), r) in enumerate(zip(inst, res)):
        alone = relax(en, s0[None], st)
        _assert_lane_equal(r, alone, i)
        assert r.s.shape == (1,) + s0.shape
        # energy at the returned positions agrees with the oracle's direct sum
        box = cubic_box(s0.shape[0], s0.shape[1])
        e_ref, _ = oracle.energy_grad(r.s[0], ks.n, ks.weights, box.volume)
        atol = energy_atol(s0.shape[0], ks.n.shape[0], e_ref)
        np.testing.assert_allclose(float(r.energy[0]), e_ref, rtol=RTOL_KERNEL_E, atol=atol)


def test_mixed_trajectories_match_lone_runs():
    inst = _instances(5, seed=3)
    st = DescentSettings(max_evals=60, record_every=5, max_records=8)
    res = relax_mixed([e for (_, _, e), _ in inst], [s for _, s in inst], st)
    for i, (((_, _, en), s0), r) in enumerate(zip(inst, res)):
        alone = relax(en, s0[None], st)
        for f in ("s", "energy", "step", "iteration", "count"):
            a = np.asarray(getattr(r.trajectory, f))
            b = np.asarray(getattr(alone.trajectory, f))
            assert np.array_equal(a, b), f"lane {i}: trajectory field {f} differs"


def test_mixed_device_tensors_stay_on_device():
    import torch

    inst = _instances(3, seed=11)
    s0 = [torch.from_numpy(s).cuda() for _, s in inst]
    res = relax_mixed([e for (_, _, e), _ in inst], s0, LBFGSSettings(energy_tol=1e-20))
    for r, x in zip(res, s0):
        assert isinstance(r.s, torch.Tensor) and r.s.is_cuda
        assert tuple(r.s.shape) == (1,) + tuple(x.shape)


def test_mixed_rejects_mismatched_inputs():
    inst = _instances(2, seed=5)
    with pytest.raises(ValueError):
        relax_mixed([inst[0][0][2]], [inst[0][1], inst[1][1]], LBFGSSettings())
    with pytest.raises(TypeError):
        relax_mixed([inst[0][0][2]], [inst[0][1].astype(np.float32)], LBFGSSettings())
