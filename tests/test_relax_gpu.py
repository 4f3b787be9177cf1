"""Batched relaxation on the device vs the oracle and the reference's contracts.

Mirrors tests/unit/test_descent.py, tests/unit/test_lbfgs.py and
tests/integration/test_relax.py of the reference: C++ transcription parity,
budgets and statuses, per-lane stopping and bit-exact freezing, original
order, chunk_iters independence, wrapped output, pass schedule.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import ATOL_DESCENT_ITERATE, ATOL_VMAP_S, RTOL_VMAP_E
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize import relax
from xla_cco.minimize.descent import DescentSettings, adaptive_descent
from xla_cco.minimize.lbfgs import LBFGSSettings, lbfgs
from xla_cco.minimize.result import (
    STATUS_BUDGET,
    STATUS_ENERGY_TOL,
    STATUS_GRAD_TOL,
    STATUS_LINESEARCH_FAIL,
    STATUS_RUNNING,
    STATUS_STAGNATED,
    STATUS_STEP_FLOOR,
)

pytestmark = pytest.mark.gpu


def small_system(n, d, k_outer):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer)
    return box, ks, make_stealthy_energy(box, ks)


def _batch(b=5, n=16, seed=0):
    return np.random.default_rng(seed).uniform(size=(b, n, 2))


def _same(a, b):
    for f in ("s", "energy", "grad_norm", "n_evals", "n_iters", "status"):
        if not np.array_equal(np.asarray(getattr(a, f)), np.asarray(getattr(b, f))):
            return False
    return True


# ------------------------------------------------------------ descent


@pytest.mark.parametrize("which", [0, 1])
def test_descent_matches_transcribed_cpp(golden, which):
    arrays, meta = golden
    c = meta["descent_cases"][which]
    n, d, iters = c["n"], c["d"], c["iters"]
    _, _, energy = small_system(n, d, c["k_outer"])
    cfg = DescentSettings(step_init=c["step0"], grow=c["grow"], max_evals=2 * iters,
                          record_every=1, max_records=iters + 1)  # fmt: skip
    res = adaptive_descent(energy, arrays[f"descent{which}_s0"], cfg)
    tr = res.trajectory
    assert int(tr.count) == iters + 1
    steps = tr.step[1:]
    np.testing.assert_array_equal(steps, arrays[f"descent{which}_steps"])
    prev = np.concatenate([[c["step0"]], steps[:-1]])
    acc = steps > prev if c["grow"] > 1.0 else steps == prev
    acc = np.where(steps < prev, False, acc)
    np.testing.assert_array_equal(acc, arrays[f"descent{which}_accepts"])
    diff = tr.s[1:] - arrays[f"descent{which}_xs"]
    assert np.max(np.abs(diff - np.round(diff))) <= ATOL_DESCENT_ITERATE


def test_descent_budgets_and_statuses():
    _, _, energy = small_system(12, 2, 4.0)
    s0 = np.random.default_rng(1).uniform(size=(12, 2))
    r = adaptive_descent(energy, s0, DescentSettings(max_evals=14))
    assert (int(r.n_iters), int(r.n_evals), int(r.status)) == (7, 14, STATUS_BUDGET)
    r = adaptive_descent(energy, s0, DescentSettings(max_evals=11))
    assert (int(r.n_iters), int(r.n_evals), int(r.status)) == (5, 10, STATUS_BUDGET)
    r = adaptive_descent(energy, s0, DescentSettings(max_evals=1))
    assert (int(r.n_iters), int(r.status)) == (0, STATUS_BUDGET)
    r = adaptive_descent(energy, s0, DescentSettings(rel_tol=1e-30))
    assert (int(r.status), int(r.n_iters)) == (STATUS_STEP_FLOOR, 40)
    np.testing.assert_array_equal(r.s, s0)
    f0 = energy(s0)
    r = adaptive_descent(energy, s0, DescentSettings(energy_tol=0.5 * f0))
    assert int(r.status) == STATUS_ENERGY_TOL and 0 < int(r.n_iters) < 5000 and r.energy < 0.5 * f0
    r = adaptive_descent(energy, s0, DescentSettings(energy_tol=2.0 * f0))
    assert int(r.status) == STATUS_ENERGY_TOL and int(r.n_iters) == 0


@pytest.mark.parametrize("grow", [1.0, 2.0])
def test_descent_zero_gradient_stops(grow):
    en = make_stealthy_energy(cubic_box(1, 2), enumerate_kvectors(np.eye(2), 0.0, 7.0))
    s0 = np.zeros((1, 2))
    r = adaptive_descent(en, s0, DescentSettings(grow=grow, max_evals=2200))
    assert int(r.status) == STATUS_GRAD_TOL and int(r.n_iters) == 0
    np.testing.assert_array_equal(r.s, s0)


def test_descent_trajectory_recording():
    _, _, energy = small_system(12, 2, 4.0)
    s0 = np.random.default_rng(1).uniform(size=(12, 2))
    r = adaptive_descent(energy, s0, DescentSettings(max_evals=40, record_every=3, max_records=4))
    assert int(r.trajectory.count) == 4
    assert list(r.trajectory.iteration) == [0, 3, 6, 9]
    for t in range(4):
        assert energy(r.trajectory.s[t]) == pytest.approx(float(r.trajectory.energy[t]), rel=1e-9)
    r2 = adaptive_descent(energy, s0, DescentSettings(max_evals=40, record_every=3, max_records=50))
    assert int(r2.trajectory.count) == 7
    assert adaptive_descent(energy, s0, DescentSettings(max_evals=20)).trajectory is None


def test_descent_matches_oracle_lane_by_lane():
    _, ks, energy = small_system(16, 2, 4.0)
    box = cubic_box(16, 2)
    s0 = _batch(b=6, seed=4)
    cfg = DescentSettings(max_evals=300, step_init=3e-2)
    out = relax(energy, s0, cfg, chunk_iters=11)
    ref = oracle.relax_batch("descent", s0, ks.n, ks.weights, box.volume, cfg)
    np.testing.assert_array_equal(out.n_iters, ref["n_iters"])
    np.testing.assert_array_equal(out.n_evals, ref["n_evals"])
    np.testing.assert_array_equal(out.status, ref["status"])
    np.testing.assert_allclose(out.energy, ref["energy"], rtol=RTOL_VMAP_E)
    d = out.s - ref["s"]
    assert np.max(np.abs(d - np.round(d))) <= ATOL_VMAP_S


# ------------------------------------------------------------ relax semantics

_METHODS = [
    lambda: DescentSettings(max_evals=300, step_init=3e-2, record_every=10, max_records=8),
    lambda: LBFGSSettings(max_evals_per_pass=20),
]


@pytest.mark.parametrize("make", _METHODS, ids=["descent", "lbfgs"])
def test_relax_batched_equals_single(make):
    settings = make()
    _, _, energy = small_system(16, 2, 4.0)
    s0 = _batch()
    out = relax(energy, s0, settings, chunk_iters=11)
    single = adaptive_descent if isinstance(settings, DescentSettings) else lbfgs
    for i in range(5):
        one = single(energy, s0[i], settings)
        assert _same(out.lane(i), one)  # lanes are computed identically: bitwise


@pytest.mark.parametrize("make", _METHODS, ids=["descent", "lbfgs"])
def test_relax_per_config_stopping_and_freeze(make):
    base = make()
    settings = type(base)(**{**base.__dict__, "energy_tol": 1e-12})
    _, _, energy = small_system(16, 2, 5.0)
    g = np.arange(4) / 4
    lattice = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    s0 = np.concatenate([lattice[None], np.random.default_rng(2).uniform(size=(3, 16, 2))])
    assert energy(s0[0]) < 1e-12 < energy(s0[1])
    short = relax(energy, s0, settings, chunk_iters=3)
    long = relax(energy, s0, settings, chunk_iters=10_000)
    assert int(short.status[0]) == STATUS_ENERGY_TOL and int(short.n_iters[0]) == 0
    np.testing.assert_array_equal(short.s[0], s0[0] % 1.0)
    assert np.all(short.status[1:] != STATUS_RUNNING)
    assert _same(short, long)


@pytest.mark.parametrize("make", _METHODS, ids=["descent", "lbfgs"])
def test_relax_compaction_preserves_results(make):
    base = make()
    _, _, energy = small_system(16, 2, 4.0)
    s0 = _batch(b=6, seed=4)
    pre = relax(energy, s0, base, chunk_iters=10_000)
    tol = float(np.median(pre.energy))
    settings = type(base)(**{**base.__dict__, "energy_tol": tol})
    fine = relax(energy, s0, settings, chunk_iters=7)
    coarse = relax(energy, s0, settings, chunk_iters=10_000)
    assert _same(fine, coarse)
    assert fine.n_iters.min() != fine.n_iters.max()


def test_relax_returns_original_order():
    _, _, energy = small_system(16, 2, 4.0)
    s0 = _batch(b=4, seed=7)
    cfg = DescentSettings(max_evals=200, step_init=3e-2, energy_tol=0.5)
    perm = np.array([2, 0, 3, 1])
    a = relax(energy, s0, cfg, chunk_iters=5)
    b = relax(energy, s0[perm], cfg, chunk_iters=5)
    for f in ("s", "energy", "n_iters", "status"):
        np.testing.assert_array_equal(np.asarray(getattr(a, f))[perm], getattr(b, f))


def test_relax_odd_batch_and_budget():
    _, _, energy = small_system(16, 2, 4.0)
    out = relax(energy, _batch(b=7, seed=3), DescentSettings(max_evals=400, step_init=3e-2,
                energy_tol=2.0), chunk_iters=2)  # fmt: skip
    assert out.s.shape[0] == 7 and np.all(out.status != STATUS_RUNNING)
    out = relax(energy, _batch(b=3), DescentSettings(max_evals=21), chunk_iters=4)
    assert np.all(out.status == STATUS_BUDGET) and np.all(out.n_iters == 10) and np.all(out.n_evals == 20)


def test_relax_rejects_bad_input():
    _, _, energy = small_system(8, 2, 4.0)
    with pytest.raises(TypeError):
        relax(energy, np.zeros((2, 8, 2), np.float32), DescentSettings())
    with pytest.raises(TypeError):
        relax(energy, np.zeros((2, 8, 2)), object())


def test_output_wrapped_into_unit_cube():
    _, _, energy = small_system(16, 2, 4.0)
    s = np.random.default_rng(5).uniform(size=(16, 2))
    s[:8, 0] = 1e-4
    s[8:, 0] = 1.0 - 1e-4
    for cfg in (DescentSettings(step_init=0.3, max_evals=24), LBFGSSettings(max_evals_per_pass=20)):
        r = relax(energy, s[None], cfg)
        assert r.s.min() >= 0.0 and r.s.max() < 1.0


# ------------------------------------------------------------ L-BFGS


def _poisson(n, d, chi, seed=0):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return box, ks, make_stealthy_energy(box, ks), np.random.default_rng(seed).uniform(size=(n, d))


def test_lbfgs_reaches_ground_state():
    box, ks, energy, s0 = _poisson(64, 2, 0.25)
    res = lbfgs(energy, s0, LBFGSSettings())
    assert float(res.energy) < 1e-20
    assert energy(res.s) < 1e-19
    pr, _ = oracle.energy_grad(res.s, ks.n, ks.weights, box.volume)
    assert pr < 1e-19


def test_lbfgs_energy_and_grad_tol():
    _, _, energy, s0 = _poisson(16, 2, 0.25)
    r = lbfgs(energy, s0, LBFGSSettings(energy_tol=1e-6))
    assert int(r.status) == STATUS_ENERGY_TOL and r.energy < 1e-6
    r = lbfgs(energy, s0, LBFGSSettings(grad_tol=1e-3))
    assert int(r.status) == STATUS_GRAD_TOL and r.grad_norm < 1e-3


def test_lbfgs_rescale_passes_equal_chained_single_passes():
    _, _, energy, s0 = _poisson(16, 2, 0.25)
    cfg = LBFGSSettings(max_evals_per_pass=12)
    full = lbfgs(energy, s0, cfg)
    cur, n_evals, n_iters = s0, 1, 0
    for r in cfg.rescales:
        one = lbfgs(energy, cur, LBFGSSettings(rescales=(r,), max_evals_per_pass=12))
        cur = one.s
        n_evals += int(one.n_evals) - 1
        n_iters += int(one.n_iters)
    assert int(full.n_iters) == n_iters and int(full.n_evals) == n_evals
    assert np.max(np.abs(full.s - cur)) < 1e-8
    assert int(full.n_evals) <= 1 + 3 * (12 + 30) and int(full.n_evals) > 1 + 3 * 12
    assert float(full.energy) > 1e-6


def test_lbfgs_stagnation_at_exact_minimum():
    en = make_stealthy_energy(cubic_box(1, 2), enumerate_kvectors(np.eye(2), 0.0, 7.0))
    r = lbfgs(en, np.zeros((1, 2)), LBFGSSettings(rescales=(1.0,), stagnation_patience=1))
    assert int(r.status) == STATUS_STAGNATED


def test_lbfgs_budget_status():
    _, _, energy, s0 = _poisson(16, 2, 0.25)
    r = lbfgs(energy, s0, LBFGSSettings(rescales=(1.0,), max_evals_per_pass=3))
    assert int(r.status) == STATUS_BUDGET


def test_lbfgs_trajectory():
    _, _, energy, s0 = _poisson(16, 2, 0.25)
    cfg = LBFGSSettings(max_evals_per_pass=60, record_every=5, max_records=6)
    tr = lbfgs(energy, s0, cfg).trajectory
    assert int(tr.count) == 6 and list(tr.iteration) == [0, 5, 10, 15, 20, 25]
    assert tr.step[0] == 0.0 and np.all(tr.step[1:] > 0.0)
    assert np.all(np.diff(tr.energy) <= 0.0)
    tr2 = lbfgs(energy, s0 + 3.0, cfg).trajectory
    rec = tr2.s[: int(tr2.count)]
    assert rec.min() >= 0.0 and rec.max() < 1.0


def test_lbfgs_ground_state_lane_returned_bit_exactly():
    _, _, energy, _ = _poisson(16, 2, 0.25)
    box, ks, en4 = small_system(16, 2, 4.0)
    s0 = np.random.default_rng(11).uniform(size=(1, 16, 2))
    res = relax(en4, s0, LBFGSSettings(max_evals_per_pass=300))
    assert float(res.energy[0]) < 1e-20
    s = res.s[0]
    for cfg in (DescentSettings(energy_tol=1e-20), LBFGSSettings(energy_tol=1e-20)):
        out = relax(en4, np.stack([s, s, s]), cfg, chunk_iters=3)
        np.testing.assert_array_equal(out.s, np.stack([s] * 3))
        assert np.all(out.status == STATUS_ENERGY_TOL) and np.all(out.n_iters == 0)


@pytest.mark.parametrize("chi", [0.05, 0.25])
def test_lbfgs_success_mask_matches_oracle(chi):
    """Seeded ensembles: the device and the oracle agree on Phi < 1e-20 per lane."""
    box, ks, energy, _ = _poisson(64, 2, chi)
    s0 = np.random.default_rng(42).uniform(size=(8, 64, 2))
    cfg = LBFGSSettings(energy_tol=1e-20)
    dev = relax(energy, s0, cfg)
    ref = oracle.relax_batch("lbfgs", s0, ks.n, ks.weights, box.volume, cfg)
    np.testing.assert_array_equal(dev.energy < 1e-20, ref["energy"] < 1e-20)
    assert np.all(dev.status != STATUS_LINESEARCH_FAIL) or np.all(dev.energy < 1e-20)


def test_small_descent_lanes_run_in_one_persistent_launch():
    """Lanes of a problem small enough for one CTA (here d=3 N=100 chi=0.05,
    M=13) run their whole descent in one launch: no graph ticks, a handful of
    launches, and the same bits alone and in a batch."""
    import torch

    from xla_cco.minimize import relax_device

    box = cubic_box(100, 3)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(0.05, 0.05, 3), 0.05, 3))
    en = make_stealthy_energy(box, ks)
    s0 = torch.from_numpy(np.random.default_rng(1).uniform(size=(4, 100, 3))).cuda()
    st = DescentSettings(grow=2.0, max_evals=20_000, energy_tol=1e-20)
    out = relax_device(en, s0, st)
    assert out["ticks"] == 0 and out["launches"] <= 5, (out["ticks"], out["launches"])
    assert (out["energy"] < 1e-20).all()
    for i in range(4):
        one = relax_device(en, s0[i:i + 1].contiguous(), st)
        for k in ("s", "energy", "n_evals", "n_iters", "status"):
            assert torch.equal(one[k][0], out[k][i]), (i, k)


@pytest.mark.parametrize("branches,overlap", [(1, 0), (2, 0), (2, 1), (3, 1), (6, 0)])
def test_tick_schedules_give_the_same_bits(monkeypatch, branches, overlap):
    """Every tick schedule the tuner may pick - one graph branch, several, and
    the overlap form (branches half a tick apart, update kernels at high stream
    priority) - advances every lane through the same kernels: the results are
    bit-identical to the default schedule's."""
    import torch

    from xla_cco.minimize import relax_device

    box = cubic_box(300, 2)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(0.4, 0.05, 2), 0.05, 2))
    en = make_stealthy_energy(box, ks)
    s0 = torch.from_numpy(np.random.default_rng(3).uniform(size=(48, 300, 2))).cuda()
    st = LBFGSSettings(energy_tol=1e-20)
    monkeypatch.setenv("CCO_AUTOTUNE", "0")
    base = relax_device(en, s0, st)
    monkeypatch.setenv("CCO_BRANCHES", str(branches))
    monkeypatch.setenv("CCO_OVERLAP", str(overlap))
    out = relax_device(en, s0, st)
    assert out["schedule"][0] == branches and out["overlap"] == bool(overlap)
    for k in ("s", "energy", "grad_norm", "n_evals", "n_iters", "status"):
        assert torch.equal(base[k], out[k]), k
    assert (out["energy"] < 1e-20).all()
