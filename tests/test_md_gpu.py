"""MD steps on the device vs the host step functions chained on their keys.

``md_run`` advances lanes by many steps with the step arithmetic fused into
the device tick; the host steps (``verlet_step``, ``andersen_reset``,
``baoab_step`` with the force from the same stealthy kernels) are the
reference's functions (``dynamics/integrators.py:83-176``) and share the
Philox draws, so both must agree to accumulated rounding and the keys
bit-exactly. Plus the physics: energy conservation of Verlet, the Andersen
count schedule, the drift stop.
"""

from __future__ import annotations

import numpy as np
import pytest

from xla_cco.box import cubic_box
from xla_cco.dynamics import (
    MDStepSettings,
    andersen_reset,
    baoab_step,
    make_force_fn,
    make_key,
    md_run,
    verlet_step,
)
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize.result import STATUS_BUDGET, STATUS_DRIFT

pytestmark = pytest.mark.gpu


def _system(n=48, d=2, chi=0.3):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return make_stealthy_energy(box, ks), np.asarray(box.basis)


def _start(b, n, d, seed, basis):
    rng = np.random.default_rng(seed)
    r = rng.uniform(size=(b, n, d)) @ basis
    v = rng.normal(scale=0.5, size=(b, n, d))
    return r, v


def _host_chain(en, basis, r, v, key, st: MDStepSettings, acc=0.0):
    force = make_force_fn(en, basis)
    out = force(r)
    f = np.asarray(out[1])
    resets = 0
    for _ in range(st.n_steps):
        if st.scheme == "verlet":
            r, v, out = verlet_step(r, v, f, force, st.dt)
            if st.andersen != "off":
                key, v, acc, n = andersen_reset(key, v, acc, st.temperature, st.andersen_p,
                                                st.andersen)  # fmt: skip
                resets += n
        else:
            key, r, v, out = baoab_step(key, r, v, f, force, st.dt, st.gamma, st.temperature)
        f = np.asarray(out[1])
    return r, v, key, resets, float(np.asarray(out[0]))


@pytest.mark.parametrize("scheme,andersen", [("verlet", "off"), ("verlet", "count"),
                                             ("verlet", "bernoulli"), ("baoab", "off")])
def test_device_run_matches_host_steps(scheme, andersen):
    en, basis = _system()
    b, n, d = 3, 48, 2
    r0, v0 = _start(b, n, d, 1, basis)
    st = MDStepSettings(dt=0.02, n_steps=25, scheme=scheme, andersen=andersen, andersen_p=0.25,
                        gamma=1.5, temperature=0.4)  # fmt: skip
    keys = np.stack([make_key(100 + i) for i in range(b)])
    dev = md_run(en, r0, v0, basis, st, keys)
    assert (dev["status"] == STATUS_BUDGET).all()
    for i in range(b):
        r, v, key, resets, phi = _host_chain(en, basis, r0[i], v0[i], keys[i], st)
        np.testing.assert_allclose(dev["r"][i], r, rtol=0, atol=1e-10)
        np.testing.assert_allclose(dev["v"][i], v, rtol=0, atol=1e-9)
        np.testing.assert_array_equal(dev["keys"][i], key)
        assert int(dev["n_resets"][i]) == resets
        np.testing.assert_allclose(dev["energy"][i], phi, rtol=1e-9, atol=1e-12)
    if andersen == "count":
        assert (dev["n_resets"] == 6).all()     # 25 steps at p = 1/4


def test_verlet_conserves_energy():
    en, basis = _system(64, 2, 0.3)
    r0, v0 = _start(2, 64, 2, 5, basis)
    res = md_run(en, r0, 0.1 * v0, basis, MDStepSettings(dt=0.005, n_steps=400), make_key(1))
    e = res["energy"] + res["kinetic"]
    assert (res["max_drift"] < 1e-4 * np.abs(e)).all()


def test_drift_stop_and_zero_steps():
    en, basis = _system()
    r0, v0 = _start(2, 48, 2, 6, basis)
    res = md_run(en, r0, v0, basis, MDStepSettings(dt=0.5, n_steps=200, drift_tol=1e-12),
                 make_key(2))  # fmt: skip
    assert (res["status"] == STATUS_DRIFT).all()
    res0 = md_run(en, r0, v0, basis, MDStepSettings(dt=0.01, n_steps=0), make_key(2))
    np.testing.assert_array_equal(res0["r"], r0)
    assert (res0["status"] == STATUS_BUDGET).all()
