"""Gradient flow (Dormand-Prince 5(4)) on the device vs the oracle and the
reference's flow tests (``tests/unit/test_flow.py``): the oracle restates
the same stage machine on the C direct sum, so step counts, statuses and
clocks agree and positions agree to accumulated rounding; then the
reference's properties - monotone energy along the recorded flow, the
stealthy ground state, a vanishing gradient, batch = loop, the arclength
parametrization, resume from ``dt``, ``dt0`` below the floor, recording.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors
from xla_cco.minimize.flow import FlowSettings, gradient_flow
from xla_cco.minimize.result import (
    STATUS_BUDGET,
    STATUS_ENERGY_TOL,
    STATUS_GRAD_TOL,
    STATUS_STEP_FLOOR,
)

pytestmark = pytest.mark.gpu


def _stealthy(n, d, shells):
    """Stealthy energy constraining the first ``shells`` shells of a cubic box."""
    box = cubic_box(n, d)
    side = float(np.asarray(box.basis)[0, 0])
    ks = enumerate_kvectors(np.asarray(box.basis), 0.0, 2.0 * np.pi / side * (shells + 0.5))
    return make_stealthy_energy(box, ks), np.asarray(box.basis), ks, box


@pytest.mark.parametrize("param", ["time", "arclength"])
def test_flow_matches_oracle_restatement(param):
    en, basis, ks, box = _stealthy(24, 2, 2)
    s0 = np.random.default_rng(1).uniform(size=(24, 2))
    st = FlowSettings(max_steps=40, parametrization=param)
    dev = gradient_flow(en, s0, basis, st)
    ref = oracle.gradient_flow_dopri5(s0, ks.n, ks.weights, box.volume, basis, st)
    assert int(dev.status) == ref["status"] == STATUS_BUDGET
    assert int(dev.n_steps) == ref["n_steps"] and int(dev.n_evals) == ref["n_evals"]
    np.testing.assert_allclose(dev.s, ref["s"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(float(dev.t), ref["t"], rtol=1e-9)
    np.testing.assert_allclose(float(dev.length), ref["length"], rtol=1e-9)
    np.testing.assert_allclose(float(dev.dt), ref["dt"], rtol=1e-6)
    np.testing.assert_allclose(float(dev.energy), ref["energy"], rtol=1e-9)


def test_energy_monotone_along_recorded_flow():
    en, basis, _, _ = _stealthy(16, 2, 2)
    s0 = np.random.default_rng(2).uniform(size=(16, 2))
    res = gradient_flow(en, s0, basis, FlowSettings(energy_tol=1e-20, record_every=1,
                                                    max_records=50_000))  # fmt: skip
    n = int(res.trajectory.count)
    t = res.trajectory.t[:n]
    e = res.trajectory.energy[:n]
    assert n > 10 and np.all(np.diff(t) > 0.0)
    assert np.all(np.diff(e) <= 1e-12 * e[:-1] + 1e-30)


def test_flow_reaches_stealthy_ground_state():
    en, basis, _, _ = _stealthy(20, 2, 2)
    s0 = np.random.default_rng(3).uniform(size=(20, 2))
    res = gradient_flow(en, s0, basis, FlowSettings(energy_tol=1e-20))
    assert int(res.status) == STATUS_ENERGY_TOL and float(res.energy) < 1e-20


def test_zero_gradient_stops_immediately():
    # one particle: Im(rho) cos - Re(rho) sin vanishes for every k. The device
    # forms rho and the back-projection phases along different table paths,
    # so the gradient is zero to rounding (|g| ~ 1e-16), not bit-exactly as in
    # the reference's trig path; a gradient tolerance far above rounding
    # checks the same stop.
    en, basis, _, _ = _stealthy(1, 2, 1)
    s0 = np.array([[0.3, 0.7]])
    res = gradient_flow(en, s0, basis, FlowSettings(grad_tol=1e-9))
    assert int(res.status) == STATUS_GRAD_TOL and int(res.n_steps) == 0
    np.testing.assert_array_equal(res.s, s0)


def test_recording_first_last_and_capacity():
    en, basis, _, _ = _stealthy(16, 2, 2)
    s0 = np.random.default_rng(4).uniform(size=(16, 2))
    res = gradient_flow(en, s0, basis, FlowSettings(energy_tol=1e-20, record_every=3,
                                                    max_records=4000))  # fmt: skip
    tr = res.trajectory
    n = int(tr.count)
    assert 2 <= n <= 4000
    np.testing.assert_array_equal(tr.s[0], s0)
    np.testing.assert_array_equal(tr.s[n - 1], res.s)
    assert float(tr.t[n - 1]) == float(res.t) and float(tr.t[0]) == 0.0
    small = gradient_flow(en, s0, basis, FlowSettings(energy_tol=1e-20, record_every=1,
                                                      max_records=5))  # fmt: skip
    assert int(small.trajectory.count) == 5
    np.testing.assert_array_equal(small.trajectory.s[4], small.s)


def test_batch_matches_loop():
    en, basis, _, _ = _stealthy(16, 2, 2)
    s0 = np.random.default_rng(5).uniform(size=(3, 16, 2))
    st = FlowSettings(energy_tol=1e-20)
    batched = gradient_flow(en, s0, basis, st)
    for i in range(3):
        one = gradient_flow(en, s0[i], basis, st)
        np.testing.assert_array_equal(batched.s[i], one.s)
        assert int(batched.n_steps[i]) == int(one.n_steps)
        assert float(batched.t[i]) == float(one.t)


def test_arclength_traces_the_same_streamline():
    en, basis, _, _ = _stealthy(16, 2, 2)
    s0 = np.random.default_rng(6).uniform(size=(16, 2))
    common = dict(energy_tol=1e-16, rtol=1e-9)
    a = gradient_flow(en, s0, basis, FlowSettings(**common))
    b = gradient_flow(en, s0, basis, FlowSettings(parametrization="arclength", **common))
    assert int(a.status) == int(b.status) == STATUS_ENERGY_TOL
    assert float(b.length) == pytest.approx(float(a.length), rel=1e-6)


def test_resume_continues_the_same_flow():
    en, basis, _, _ = _stealthy(16, 2, 2)
    s0 = np.random.default_rng(7).uniform(size=(16, 2))
    whole = gradient_flow(en, s0, basis, FlowSettings(energy_tol=1e-14))
    first = gradient_flow(en, s0, basis, FlowSettings(max_steps=60))
    second = gradient_flow(en, first.s, basis, FlowSettings(energy_tol=1e-14, dt_init=float(first.dt)))
    assert int(second.status) == STATUS_ENERGY_TOL
    np.testing.assert_allclose(second.s, whole.s, atol=1e-6)
    assert float(first.t) + float(second.t) == pytest.approx(float(whole.t), rel=1e-3)


def test_dt0_below_floor_stops_immediately():
    en, basis, _, _ = _stealthy(16, 2, 2)
    s0 = np.random.default_rng(8).uniform(size=(16, 2))
    res = gradient_flow(en, s0, basis, FlowSettings(), dt0=0.0)
    assert int(res.status) == STATUS_STEP_FLOOR and int(res.n_steps) == 0
    np.testing.assert_array_equal(res.s, s0)


def test_rosenbrock_agrees_with_dopri():
    en, basis, _, _ = _stealthy(8, 2, 1)
    s0 = np.random.default_rng(9).uniform(size=(8, 2))
    t_stop = 0.05
    ref = gradient_flow(en, s0, basis, FlowSettings(rtol=1e-10, t_max=t_stop))
    ros = gradient_flow(en, s0, basis, FlowSettings(method="rosenbrock", rtol=1e-3, atol=1e-10,
                                                    t_max=t_stop))  # fmt: skip
    np.testing.assert_allclose(ros.s, ref.s, atol=1e-5)
    assert float(ros.t) == pytest.approx(t_stop, rel=1e-12)
