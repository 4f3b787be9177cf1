"""relax over any AbstractEnergy (src/xla_cco/minimize/__init__.py:102-107):
the device lanes of the fused path, with each tick's evaluation done by the
energy's own value_and_grad (cco_stepper_*).

An energy that evaluates through the kernels gives the fused path's bits
exactly (the lanes, update kernels and evaluations are the same); a plain
torch energy with the autodiff defaults relaxes to its known minimum.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from xla_cco import DescentSettings, LBFGSSettings, relax
from xla_cco.box import cubic_box
from xla_cco.energy import AbstractEnergy, make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi

pytestmark = pytest.mark.gpu


def _stealthy(n, d, chi):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return make_stealthy_energy(box, ks)


class Delegate(AbstractEnergy):
    """A user energy that happens to evaluate through the stealthy kernels."""

    def __init__(self, inner, batched=False):
        self.inner = inner
        if batched:
            self.value_and_grad_batch = lambda s: inner.evaluate(s)[:2]

    def __call__(self, s):
        return self.inner(s)

    def value_and_grad(self, s):
        phi, g, _, _ = self.inner.evaluate(s[None])
        return phi[0], g[0]


class Wells(AbstractEnergy):
    """sum_j,a (1 - cos 2 pi (s_ja - c_ja)): torch operations, autodiff defaults."""

    def __init__(self, centres):
        import torch

        self.c = torch.as_tensor(centres, dtype=torch.float64, device="cuda")

    def __call__(self, s):
        import torch

        return torch.sum(1.0 - torch.cos(2.0 * math.pi * (s - self.c)))


@pytest.mark.parametrize("batched", [False, True])
@pytest.mark.parametrize("settings", [LBFGSSettings(energy_tol=1e-20),
                                      DescentSettings(grow=2.0, max_evals=4000, energy_tol=1e-12)])
def test_user_energy_through_the_kernels_matches_the_fused_path_bitwise(settings, batched):
    en = _stealthy(200, 2, 0.3)
    s0 = np.random.default_rng(4).uniform(size=(5, 200, 2))
    fused = relax(en, s0, settings)
    user = relax(Delegate(en, batched), s0, settings)
    np.testing.assert_array_equal(user.s, fused.s)
    for k in ("energy", "grad_norm", "n_evals", "n_iters", "status"):
        np.testing.assert_array_equal(getattr(user, k), getattr(fused, k))


def test_torch_energy_with_autodiff_defaults_relaxes_to_its_minimum():
    rng = np.random.default_rng(8)
    centres = rng.uniform(size=(30, 3))
    s0 = np.stack([np.mod(centres + rng.uniform(-0.2, 0.2, size=(30, 3)), 1.0) for _ in range(3)])
    res = relax(Wells(centres), s0, LBFGSSettings(energy_tol=1e-20))
    assert (res.status == 1).all() and (res.energy < 1e-20).all()
    d = np.mod(res.s - centres[None] + 0.5, 1.0) - 0.5
    assert np.abs(d).max() < 1e-9
    # the default hessian (autograd): 4 pi^2 cos(...) on the diagonal
    h = Wells(centres).hessian(centres).cpu().numpy()
    np.testing.assert_allclose(np.diag(h), 4 * math.pi**2, rtol=1e-12)
    assert np.abs(h - np.diag(np.diag(h))).max() == 0.0


def test_external_relax_rejects_what_it_cannot_do():
    en = Delegate(_stealthy(64, 2, 0.2))
    s0 = np.random.default_rng(0).uniform(size=(2, 64, 2))
    with pytest.raises(ValueError):
        relax(en, s0, LBFGSSettings(precision="mixed"))
    with pytest.raises(ValueError):
        relax(en, s0, LBFGSSettings(record_every=1, max_records=4))
    with pytest.raises(TypeError):
        relax(object(), s0, LBFGSSettings())
