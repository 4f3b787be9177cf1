"""MD step functions on the host: Philox known answers, step arithmetic and
the Andersen schedules (``dynamics/integrators.py`` of the reference), with
force functions that need no GPU."""

from __future__ import annotations

import math

import numpy as np
import pytest

from xla_cco.dynamics.integrators import (
    andersen_reset,
    baoab_step,
    make_key,
    philox4x32_10,
    verlet_step,
)


def test_philox_known_answers():
    # Random123 known-answer vectors of philox4x32_10 (Salmon et al., SC11)
    cases = [
        ((0, 0), (0, 0, 0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 2, (0xFFFFFFFF,) * 4, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0xA4093822, 0x299F31D0), (0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]  # fmt: skip
    for key, ctr, want in cases:
        got = philox4x32_10(np.array(key, np.uint32), np.array([ctr], np.uint32))[0]
        assert tuple(int(x) for x in got) == want


def _harmonic(k=2.0):
    def force_fn(r):
        return 0.5 * k * float(np.sum(r * r)), -k * r, np.zeros(1), np.zeros(1)
    return force_fn


def test_verlet_step_arithmetic_and_harmonic_energy():
    f_fn = _harmonic()
    r = np.array([[1.0, 0.0], [0.0, -0.5]])
    v = np.array([[0.0, 1.0], [0.3, 0.0]])
    f = f_fn(r)[1]
    dt = 0.01
    r1, v1, out = verlet_step(r, v, f, f_fn, dt)
    np.testing.assert_array_equal(r1, r + dt * (v + 0.5 * dt * f))
    np.testing.assert_array_equal(v1, (v + 0.5 * dt * f) + 0.5 * dt * out[1])
    e0 = f_fn(r)[0] + 0.5 * np.sum(v * v)
    for _ in range(2000):
        r, v, out = verlet_step(r, v, out[1], f_fn, dt)
    assert abs(out[0] + 0.5 * np.sum(v * v) - e0) < 1e-4 * e0


def test_andersen_count_mode_fires_on_schedule():
    key = make_key(7)
    v = np.zeros((10, 3))
    acc, fired = 0.0, 0
    for _ in range(20):   # p = 1/4 is exact: the accumulator reaches 1 every 4th step
        key, v, acc, n = andersen_reset(key, v, acc, 2.0, 0.25, "count")
        fired += n
    assert fired == 5 and acc == 0.0
    assert np.count_nonzero(np.any(v != 0.0, axis=1)) <= 5


def test_andersen_bernoulli_rate_and_validation():
    key = make_key(11)
    v = np.zeros((5, 2))
    fired = 0
    for _ in range(4000):
        key, v, _, n = andersen_reset(key, v, 0.0, 1.0, 0.25, "bernoulli")
        fired += n
    assert abs(fired / 4000 - 0.25) < 0.03
    with pytest.raises(ValueError):
        andersen_reset(key, v, 0.0, 1.0, 1.5, "count")
    with pytest.raises(ValueError):
        andersen_reset(key, v, 0.0, 1.0, 0.5, "sometimes")


def test_baoab_noise_statistics_and_zero_friction():
    f_fn = _harmonic(0.0)          # free particles: only the thermostat acts
    key = make_key(3)
    r = np.zeros((200, 3))
    v = np.zeros((200, 3))
    out = f_fn(r)
    ke = []
    for i in range(400):
        key, r, v, out = baoab_step(key, r, v, out[1], f_fn, 0.1, 1.0, 0.7)
        if i > 100:
            ke.append(np.mean(v * v))
    assert abs(np.mean(ke) - 0.7) < 0.05          # equipartition: <v^2> = T
    # gamma = 0: c = 1, no noise - BAOAB is a symplectic step with split drift
    f_fn = _harmonic()
    r0 = np.array([[1.0, 0.0]])
    v0 = np.array([[0.0, 1.0]])
    _, r1, v1, _ = baoab_step(make_key(0), r0, v0, f_fn(r0)[1], f_fn, 0.01, 0.0, 1.0)
    r2, v2, _ = verlet_step(r0, v0, f_fn(r0)[1], f_fn, 0.01)
    np.testing.assert_allclose(r1, r2, rtol=0, atol=1e-15)
    np.testing.assert_allclose(v1, v2, rtol=0, atol=1e-15)
    with pytest.raises(ValueError):
        baoab_step(key, r0, v0, v0, f_fn, 0.01, -1.0, 1.0)
    assert math.isfinite(float(np.sum(v)))
