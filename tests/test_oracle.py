"""Pin the CPU oracle against the reference's golden data before trusting it.

* energies/forces: the reference oracle (tests/oracle.py there) on small
  systems, and the C++ engine's energies of tests/data/md_cxx_samples.npz;
* descent: the reference test's verbatim transcription of the C++ loop
  (tests/unit/test_descent.py:52-128 there): steps exact, accepts equal,
  iterates within 1e-14;
* L-BFGS: behaviour only (iterates are unpinned: optax is not vendored).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import ATOL_DESCENT_ITERATE, RTOL_KERNEL_E, RTOL_KERNEL_F, RTOL_MD_CXX_PHI
from xla_cco.box import Box, cubic_box
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize.descent import DescentSettings
from xla_cco.minimize.lbfgs import LBFGSSettings


def test_oracle_energy_forces_vs_reference_oracle(golden):
    arrays, meta = golden
    for c in meta["energy_cases"]:
        i = c["i"]
        s, n, basis = arrays[f"energy{i}_s"], arrays[f"energy{i}_n"], arrays[f"energy{i}_basis"]
        phi, g = oracle.energy_grad(s, n, np.ones(n.shape[0]), c["volume"])
        np.testing.assert_allclose(phi, c["phi"], rtol=RTOL_KERNEL_E)
        f = Box(basis).cartesian_forces(g)
        ref = arrays[f"energy{i}_forces"]
        np.testing.assert_allclose(f, ref, rtol=RTOL_KERNEL_F, atol=RTOL_KERNEL_F * np.abs(ref).max())
        phi2, g2 = oracle.energy_direct(s, n, np.ones(n.shape[0]), c["volume"])
        np.testing.assert_allclose(phi2, c["phi"], rtol=RTOL_KERNEL_E)
        np.testing.assert_allclose(g2, g, rtol=1e-10, atol=1e-10 * np.abs(g).max())
        # the accurate mode (exact phase reduction, compensated sums) against the same pins
        pa, ga = oracle.energy_grad_accurate(s[None], n, np.ones(n.shape[0]), c["volume"])
        np.testing.assert_allclose(pa[0], c["phi"], rtol=RTOL_KERNEL_E)
        fa = Box(basis).cartesian_forces(ga[0])
        np.testing.assert_allclose(fa, ref, rtol=0, atol=RTOL_KERNEL_F * np.abs(ref).max())


def test_oracle_matches_cpp_golden_energies(golden):
    arrays, meta = golden
    basis = arrays["cxx_basis"]
    ks = enumerate_kvectors(basis, 0.0, meta["cxx"]["K"])
    assert ks.n.shape[0] == meta["cxx"]["M"]
    vol = Box(basis).volume
    phi, _ = oracle.energy_grad_batch(arrays["cxx_s"], ks.n, ks.weights, vol)
    rel = np.abs(phi - arrays["cxx_phi"]) / arrays["cxx_phi"]
    assert rel.max() <= RTOL_MD_CXX_PHI
    assert rel.max() < 1e-12  # measured ~1e-13: far inside the reference's gate


@pytest.mark.parametrize("which", [0, 1])
def test_oracle_descent_matches_transcribed_cpp(golden, which):
    arrays, meta = golden
    c = meta["descent_cases"][which]
    n, d, iters = c["n"], c["d"], c["iters"]
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, c["k_outer"])
    cfg = DescentSettings(step_init=c["step0"], grow=c["grow"], max_evals=2 * iters,
                          record_every=1, max_records=iters + 1)  # fmt: skip
    res = oracle.relax_one("descent", arrays[f"descent{which}_s0"], ks.n, ks.weights, box.volume, cfg)
    tr = res["trajectory"]
    assert tr["count"] == iters + 1
    steps = tr["step"][1:]
    np.testing.assert_array_equal(steps, arrays[f"descent{which}_steps"])
    prev = np.concatenate([[c["step0"]], steps[:-1]])
    acc = steps > prev if c["grow"] > 1.0 else steps == prev
    acc = np.where(steps < prev, False, acc)
    np.testing.assert_array_equal(acc, arrays[f"descent{which}_accepts"])
    xs = arrays[f"descent{which}_xs"]
    diff = tr["s"][1:] - xs
    dev = np.max(np.abs(diff - np.round(diff)))
    assert dev <= ATOL_DESCENT_ITERATE


def test_oracle_descent_budget_and_floor():
    box = cubic_box(12, 2)
    ks = enumerate_kvectors(box.basis, 0.0, 4.0)
    s0 = np.random.default_rng(1).uniform(size=(12, 2))
    r = oracle.relax_one("descent", s0, ks.n, ks.weights, box.volume, DescentSettings(max_evals=14))
    assert (r["n_iters"], r["n_evals"], r["status"]) == (7, 14, 3)
    r = oracle.relax_one("descent", s0, ks.n, ks.weights, box.volume, DescentSettings(rel_tol=1e-30))
    assert (r["status"], r["n_iters"]) == (2, 40)


def test_oracle_lbfgs_reaches_ground_state():
    """d=2, N=64, chi=0.25 reaches Phi < 1e-20 (reference test_lbfgs.py:149-156)."""
    box = cubic_box(64, 2)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(0.25, 0.05, 2), 0.05, 2))
    s0 = np.random.default_rng(0).uniform(size=(64, 2))
    r = oracle.relax_one("lbfgs", s0, ks.n, ks.weights, box.volume, LBFGSSettings(energy_tol=1e-20))
    assert r["energy"] < 1e-20 and r["status"] == 1
    phi, _ = oracle.energy_grad(r["s"], ks.n, ks.weights, box.volume)
    assert phi < 1e-19


def test_oracle_hessian_vs_central_differences():
    """The oracle's closed-form Hessian restatement against central differences
    of its own gradient (small box)."""
    rng = np.random.default_rng(4)
    n_pts, d = 12, 2
    basis = np.sqrt(n_pts) * np.eye(2)
    nv, _ = oracle.halfspace_kvectors(basis, 0.0, 4.0)
    w = np.ones(nv.shape[0])
    s = rng.uniform(size=(n_pts, d))
    h = oracle.hessian_direct(s, nv, w, float(n_pts))
    eps = 1e-6
    fd = np.zeros_like(h)
    for i in range(s.size):
        dp, dm = s.ravel().copy(), s.ravel().copy()
        dp[i] += eps
        dm[i] -= eps
        _, gp = oracle.energy_grad(dp.reshape(n_pts, d), nv, w, float(n_pts))
        _, gm = oracle.energy_grad(dm.reshape(n_pts, d), nv, w, float(n_pts))
        fd[:, i] = ((gp - gm) / (2 * eps)).ravel()
    np.testing.assert_allclose(h, fd, rtol=0, atol=1e-6 * np.abs(h).max())
    np.testing.assert_allclose(h, h.T, rtol=0, atol=1e-12 * np.abs(h).max())
