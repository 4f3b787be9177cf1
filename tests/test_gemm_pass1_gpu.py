"""Parity of the two forms of the FP64 density pass: the complex-GEMM form
(dense k-sets, d = 2 and d = 3) and the per-segment form (the same problem
built with CCO_PASS1_GEMM=0), each against the C oracle's direct sums
(energy 1e-12 relative, forces 1e-12 of max |F| against the accurate oracle), batch sizes that leave
ragged particle tiles and ragged run groups."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from conftest import RTOL_KERNEL_E, RTOL_KERNEL_F
from xla_cco import _native
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi

pytestmark = pytest.mark.gpu

# k-sets that take the (folded) GEMM form: d = 2 with window widths 16 and 32
# columns and a 108-entry prefix table, d = 3 with one and several run groups
CASES = [(2, 1000, 0.40, 5), (2, 600, 0.49, 3), (2, 333, 0.30, 3), (2, 20000, 0.45, 1),
         (3, 4000, 0.45, 2), (3, 20000, 0.45, 1)]
# sparse ones (folded cells above 8 FMAs per k-set row) and 1-D ones keep the
# per-segment kernel
SEGMENT_ONLY = [(3, 400, 0.30), (3, 120, 0.30), (1, 500, 0.40)]


def _energy(n, d, chi):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return make_stealthy_energy(box, ks), ks


def _gemm_blocks(en, n) -> int:
    out = ctypes.c_int(-1)
    _native.check(_native.load().cco_problem_pass1_form(en.problem_handle(0, n), ctypes.byref(out)),
                  "cco_problem_pass1_form")  # fmt: skip
    return out.value


@pytest.mark.parametrize("d,n,chi,b", CASES)
def test_gemm_and_segment_forms_vs_oracle(monkeypatch, d, n, chi, b):
    s = np.random.default_rng(n + d).uniform(size=(b, n, d))
    phis, grads = {}, {}
    for form in ("gemm", "segment"):
        if form == "segment":
            monkeypatch.setenv("CCO_PASS1_GEMM", "0")
        en, ks = _energy(n, d, chi)   # a fresh problem reads the switch when it is created
        blocks = _gemm_blocks(en, n)
        assert (blocks > 0) == (form == "gemm"), (form, blocks)
        phi, g, _, _ = en.evaluate(s)
        phis[form], grads[form] = phi, g
    e_ref, g_ref = oracle.energy_grad_accurate(s, ks.n.astype(np.int64), np.ones(ks.n.shape[0]), float(n))
    for form in ("gemm", "segment"):
        np.testing.assert_allclose(phis[form], e_ref, rtol=RTOL_KERNEL_E, atol=0)
        for i in range(b):
            scale = np.abs(g_ref[i]).max()
            np.testing.assert_allclose(grads[form][i], g_ref[i], rtol=0, atol=RTOL_KERNEL_F * scale)
    np.testing.assert_allclose(phis["gemm"], phis["segment"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("d,n,chi", SEGMENT_ONLY)
def test_sparse_k_sets_keep_the_segment_form(d, n, chi):
    en, _ = _energy(n, d, chi)
    assert _gemm_blocks(en, n) == 0


def test_gemm_form_on_a_sheared_box():
    from xla_cco.box import Box

    n, d = 1000, 2
    basis = np.array([[1.0, 0.0], [0.35, 1.0]]) * np.sqrt(n)   # 69% of the block cells used
    box = Box(basis)
    ks = enumerate_kvectors(basis, 0.0, k_outer_from_ka(ka_from_chi(0.40, 0.05, d), 0.05, d))
    en = make_stealthy_energy(box, ks)
    assert _gemm_blocks(en, n) > 0
    s = np.random.default_rng(31).uniform(size=(3, n, d))
    phi, g, _, _ = en.evaluate(s)
    e_ref, g_ref = oracle.energy_grad_accurate(s, ks.n.astype(np.int64), np.ones(ks.n.shape[0]), box.volume)
    np.testing.assert_allclose(phi, e_ref, rtol=RTOL_KERNEL_E, atol=0)
    for i in range(3):
        np.testing.assert_allclose(g[i], g_ref[i], rtol=0, atol=RTOL_KERNEL_F * np.abs(g_ref[i]).max())


def test_lbfgs_relaxation_through_the_gemm_form_vs_oracle():
    """The headline path (L-BFGS with the GEMM density pass) reaches the ground
    state, confirmed by the oracle's direct sums at the device's final positions
    (L-BFGS iterates themselves are not pinned to the reference)."""
    from xla_cco import LBFGSSettings, relax

    n, d, b = 600, 2, 4
    en, ks = _energy(n, d, 0.49)
    assert _gemm_blocks(en, n) > 0
    s0 = np.random.default_rng(17).uniform(size=(b, n, d))
    res = relax(en, s0, LBFGSSettings(energy_tol=1e-20))
    assert (res.energy < 1e-20).all() and (res.status == 1).all()
    # the device's final energies, re-evaluated by the oracle at the device's positions
    # (the accurate mode: at Phi ~ 1e-20 the plain FP64 oracle's own rounding exceeds 1e-24)
    e_chk, _ = oracle.energy_grad_accurate(res.s, ks.n.astype(np.int64), np.ones(ks.n.shape[0]), float(n))
    np.testing.assert_allclose(res.energy, e_chk, rtol=1e-6, atol=1e-24)
