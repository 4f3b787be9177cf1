"""Parity of the two forms of the FP64 density pass: the complex-GEMM form
(dense k-sets, d = 2 and d = 3) and the per-segment form (the same problem
built with CCO_PASS1_GEMM=0), each against the C oracle's direct sums
(energy 1e-12 relative, forces 1e-10 of max |F|), batch sizes that leave
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

# dense k-sets that take the GEMM form (d = 2 incl. a 108-entry prefix table, d = 3)
CASES = [(2, 1000, 0.40, 5), (2, 600, 0.49, 3), (2, 20000, 0.45, 1), (3, 20000, 0.45, 1)]
# sparse ones that keep the per-segment kernel
SEGMENT_ONLY = [(2, 333, 0.30), (3, 4000, 0.45), (1, 500, 0.40)]


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
    e_ref, g_ref = oracle.energy_grad_batch(s, ks.n.astype(np.int64), np.ones(ks.n.shape[0]), float(n),
                                            threads=oracle.max_threads())  # fmt: skip
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
