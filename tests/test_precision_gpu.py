"""Mixed precision: FP32 evaluations early, FP64 for the finish and the judgement.

The reference is FP64 only, so these tests hold the mixed path to the FP64
path and to the oracle: the FP32 evaluation stays within a stated error of
the oracle's direct sum, mixed-precision relaxations reach Phi < 1e-20 on
exactly the lanes where plain FP64 does (identical success masks on seeded
ensembles), every mixed result's final energy is an FP64 value that the
oracle confirms, and the lanes really ran FP32 evaluations first.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from conftest import RTOL_KERNEL_E, energy_atol
from xla_cco import _native
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize import relax, relax_device
from xla_cco.minimize.lbfgs import LBFGSSettings
from xla_cco.serve import RelaxServer

pytestmark = pytest.mark.gpu

TOL = 1e-20
# FP32 evaluation vs the FP64 oracle on uniform configurations: |rho_k| ~ sqrt(N),
# each phase carries ~1e-6 relative error, so Phi is good to ~1e-5 relative and
# the gradient to ~1e-4 of its largest component.
RTOL_FP32_E = 1e-4
RTOL_FP32_F = 1e-3


def _system(n, d, chi):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return box, ks, make_stealthy_energy(box, ks)


@pytest.mark.parametrize("n,d,chi,b", [(400, 1, 0.3, 3), (500, 2, 0.4, 3), (300, 3, 0.45, 3), (600, 2, 0.49, 3)])
def test_fp32_evaluation_against_oracle(n, d, chi, b):
    import torch

    box, ks, en = _system(n, d, chi)
    s = np.random.default_rng(n + d).uniform(size=(b, n, d))
    st = torch.from_numpy(s).cuda()
    phi = torch.empty(b, dtype=torch.float64, device="cuda")
    g = torch.empty_like(st)
    h = en.problem_handle(torch.cuda.current_device(), n)
    code = _native.load().cco_energy_grad_fp32(h, None, b, st.data_ptr(), phi.data_ptr(), g.data_ptr())
    assert code == _native.CCO_OK
    torch.cuda.synchronize()
    for i in range(b):
        pr, gr = oracle.energy_grad(s[i], ks.n, ks.weights, box.volume)
        np.testing.assert_allclose(phi[i].item(), pr, rtol=RTOL_FP32_E)
        np.testing.assert_allclose(g[i].cpu().numpy(), gr, rtol=0, atol=RTOL_FP32_F * np.abs(gr).max())


@pytest.mark.parametrize("n,d,chi,b", [(500, 2, 0.40, 24), (300, 3, 0.45, 16), (900, 2, 0.49, 16)])
def test_mixed_precision_success_masks_match_plain(n, d, chi, b):
    import torch

    box, ks, en = _system(n, d, chi)
    s0 = torch.from_numpy(np.random.default_rng(7 + n).uniform(size=(b, n, d))).cuda()
    plain = relax_device(en, s0, LBFGSSettings(energy_tol=TOL))
    mixed = relax_device(en, s0, LBFGSSettings(energy_tol=TOL, precision="mixed"))
    ok_p = (plain["energy"] < TOL).cpu().numpy()
    ok_m = (mixed["energy"] < TOL).cpu().numpy()
    np.testing.assert_array_equal(ok_m, ok_p)
    n32 = mixed["n_evals_fp32"].cpu().numpy()
    assert (n32 > 0).all(), "every mixed lane starts in FP32"
    assert (plain["n_evals_fp32"].cpu().numpy() == 0).all()
    # the final energy of a mixed result is an FP64 evaluation: the oracle agrees
    s_fin = mixed["s"].cpu().numpy()
    e_fin = mixed["energy"].cpu().numpy()
    for i in range(b):
        e_ref, _ = oracle.energy_grad(s_fin[i], ks.n, ks.weights, box.volume)
        np.testing.assert_allclose(e_fin[i], e_ref, rtol=RTOL_KERNEL_E,
                                   atol=energy_atol(n, ks.n.shape[0], e_ref))  # fmt: skip


@pytest.mark.parametrize("case", ["grad_tol", "budget", "energy_tol"])
def test_fp32_lane_never_ends_on_an_fp32_judgement(case):
    """A lane still in FP32 that meets a stopping rule (gradient tolerance,
    budget, or an energy below the tolerance) first switches to FP64; the
    status and the energy it reports are FP64 results at its final point."""
    import torch

    box, ks, en = _system(300, 2, 0.3)
    b = 4
    s0 = torch.from_numpy(np.random.default_rng(11).uniform(size=(b, 300, 2))).cuda()
    if case == "grad_tol":   # met at the first iteration, while every lane is in FP32
        st = LBFGSSettings(grad_tol=1e30, precision="mixed")
        want = 6
    elif case == "budget":   # one pass whose budget ends inside the FP32 phase
        st = LBFGSSettings(rescales=(1.0,), max_evals_per_pass=6, precision="mixed")
        want = 3
    else:                    # a tolerance the very first (FP32) evaluation meets
        st = LBFGSSettings(energy_tol=1e30, precision="mixed")
        want = 1
    out = relax_device(en, s0, st)
    status = out["status"].cpu().numpy()
    np.testing.assert_array_equal(status, np.full(b, want))
    n32 = out["n_evals_fp32"].cpu().numpy()
    ne = out["n_evals"].cpu().numpy()
    assert (n32 > 0).all() and (n32 < ne).all(), (n32, ne)
    # the reported energy is an FP64 evaluation at the reported (wrapped) positions
    phi64, _, _, _ = en.evaluate(out["s"], want_grad=False)
    np.testing.assert_allclose(out["energy"].cpu().numpy(), phi64.cpu().numpy(), rtol=1e-12, atol=0)


def test_failed_mixed_lane_returns_the_plain_fp64_result():
    """A mixed lane that ends above energy_tol runs again from s0 in FP64: its
    positions, energy, status and iterations are the plain run's bits; its
    evaluation count includes the discarded mixed run."""
    import torch

    _, _, en = _system(300, 2, 0.35)
    s0 = torch.from_numpy(np.random.default_rng(21).uniform(size=(4, 300, 2))).cuda()
    st = dict(energy_tol=TOL, max_evals_per_pass=40)    # too small a budget to reach 1e-20
    plain = relax_device(en, s0, LBFGSSettings(**st))
    mixed = relax_device(en, s0, LBFGSSettings(precision="mixed", **st))
    assert (plain["energy"] >= TOL).all()
    for k in ("s", "energy", "grad_norm", "n_iters", "status"):
        np.testing.assert_array_equal(mixed[k].cpu().numpy(), plain[k].cpu().numpy())
    ne_m, ne_p = mixed["n_evals"].cpu().numpy(), plain["n_evals"].cpu().numpy()
    n32 = mixed["n_evals_fp32"].cpu().numpy()
    assert (n32 > 0).all() and (ne_m > ne_p + n32 - 1).all(), (ne_m, ne_p, n32)


def test_one_dimensional_lanes_stay_fp64_in_mixed_mode():
    """1-D lanes of a mixed run never evaluate in FP32 and equal plain FP64
    lanes bit for bit (the FP64 lanes of a mixed run use the plain kernels)."""
    import torch

    _, _, en = _system(500, 1, 0.3)
    s0 = torch.from_numpy(np.random.default_rng(22).uniform(size=(3, 500, 1))).cuda()
    plain = relax_device(en, s0, LBFGSSettings(energy_tol=TOL))
    mixed = relax_device(en, s0, LBFGSSettings(energy_tol=TOL, precision="mixed"))
    assert (mixed["n_evals_fp32"].cpu().numpy() == 0).all()
    for k in ("s", "energy", "n_evals", "n_iters", "status"):
        np.testing.assert_array_equal(mixed[k].cpu().numpy(), plain[k].cpu().numpy())


def test_mixed_precision_served_equals_relaxed_alone():
    _, _, en = _system(400, 2, 0.35)
    rng = np.random.default_rng(3)
    s0 = [rng.uniform(size=(400, 2)) for _ in range(4)]
    st = LBFGSSettings(energy_tol=TOL, precision="mixed")
    with RelaxServer(st) as srv:
        results = [srv.result(t) for t in [srv.submit(en, s) for s in s0]]
    for s, r in zip(s0, results):
        alone = relax(en, s[None], st)
        np.testing.assert_array_equal(r.s, alone.s[0])
        assert r.energy == float(alone.energy[0]) and r.n_evals == int(alone.n_evals[0])
        assert r.n_evals_fp32 > 0


def test_precision_setting_is_validated():
    _, _, en = _system(50, 2, 0.2)
    with pytest.raises(ValueError):
        relax(en, np.zeros((1, 50, 2)), LBFGSSettings(precision="fp16"))
    assert ctypes.sizeof(_native.LBFGSSettingsC) == 17 * 8
