"""Closed-form Hessian kernels (``cco_hessian``) against the oracle.

The reference's ``StealthyEnergy.hessian`` (src/xla_cco/energy.py:272-299)
is restated by the oracle as NumPy direct sums; the kernels must agree with
it to 1e-11 of max|H|, be exactly symmetric, agree with central differences
of the oracle's gradient, and give a batch the same bits as single calls.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from xla_cco.box import Box, cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi

pytestmark = pytest.mark.gpu

RTOL_HESS = 1e-11   # of max|H|: M-term sums of O(|rho| n^2) terms, both sides FP64


def _system(n, d, chi):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return box, ks, make_stealthy_energy(box, ks)


@pytest.mark.parametrize("n,d,chi", [(40, 1, 0.3), (64, 2, 0.25), (150, 2, 0.45), (60, 3, 0.3),
                                     (130, 3, 0.15), (200, 1, 0.45)])  # fmt: skip
def test_hessian_vs_oracle_direct_sum(n, d, chi):
    box, ks, en = _system(n, d, chi)
    s = np.random.default_rng(n * d).uniform(size=(n, d))
    h = en.hessian(s)
    ref = oracle.hessian_direct(s, ks.n, ks.weights, box.volume)
    assert h.shape == (n * d, n * d)
    np.testing.assert_allclose(h, ref, rtol=0, atol=RTOL_HESS * np.abs(ref).max())
    np.testing.assert_array_equal(h, h.T)


def test_hessian_vs_central_differences_of_the_gradient():
    box, ks, en = _system(48, 2, 0.3)
    s = np.random.default_rng(2).uniform(size=(48, 2))
    h = en.hessian(s)
    eps = 1e-6
    cols = []
    for i in range(s.size):
        dp, dm = s.copy().ravel(), s.copy().ravel()
        dp[i] += eps
        dm[i] -= eps
        _, gp = oracle.energy_grad_accurate(dp.reshape(1, 48, 2), ks.n, ks.weights, box.volume)
        _, gm = oracle.energy_grad_accurate(dm.reshape(1, 48, 2), ks.n, ks.weights, box.volume)
        cols.append(((gp - gm) / (2 * eps)).ravel())
    fd = np.stack(cols, axis=1)
    np.testing.assert_allclose(h, fd, rtol=0, atol=1e-6 * np.abs(fd).max())


def test_hessian_batch_equals_single_calls_and_sheared_box():
    basis = np.array([[2.0, 0.0, 0.0], [0.7, 1.5, 0.0], [0.3, -0.4, 1.8]]) * 3.0
    box = Box(basis)
    ks = enumerate_kvectors(basis, 0.5, 4.0)
    en = make_stealthy_energy(box, ks)
    s = np.random.default_rng(5).uniform(-1.0, 2.0, size=(3, 70, 3))   # unwrapped positions
    hb = en.hessian(s)
    assert hb.shape == (3, 210, 210)
    for i in range(3):
        np.testing.assert_array_equal(hb[i], en.hessian(s[i]))
        ref = oracle.hessian_direct(s[i], ks.n, ks.weights, box.volume)
        np.testing.assert_allclose(hb[i], ref, rtol=0, atol=RTOL_HESS * np.abs(ref).max())


def test_hessian_row_sums_vanish():
    """Translation invariance: sum over l of H[(j,a),(l,b)] = 0 for every j, a, b."""
    _, _, en = _system(300, 2, 0.4)
    s = np.random.default_rng(9).uniform(size=(300, 2))
    h = en.hessian(s).reshape(300, 2, 300, 2)
    rows = h.sum(axis=2)
    assert np.abs(rows).max() <= 1e-10 * np.abs(h).max() * 300
