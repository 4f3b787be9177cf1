"""Host-side API contracts that need no GPU: settings, box, validation order."""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from xla_cco import Box, DescentSettings, LBFGSSettings, cubic_box, make_stealthy_energy, wrap_fractional
from xla_cco.energy import StealthyEnergy
from xla_cco.kvectors import enumerate_kvectors
from xla_cco.minimize import relax
from xla_cco.minimize import descent as descent_mod
from xla_cco.minimize import lbfgs as lbfgs_mod


def test_settings_defaults_match_reference():
    assert dataclasses.asdict(DescentSettings()) == dict(
        step_init=1e-3, step_min=1e-15, shrink=0.5, grow=1.0, rel_tol=0.01, max_evals=10_000,
        energy_tol=0.0, record_every=0, max_records=0,
    )  # fmt: skip
    fields = dataclasses.asdict(LBFGSSettings())
    # the one field the reference does not have: opt-in mixed precision, off by default
    assert fields.pop("precision") == "fp64"
    assert fields == dict(
        memory=100, rescales=(1e4, 1.0, 1e-2), max_evals_per_pass=500_000, energy_tol=0.0,
        grad_tol=0.0, stagnation_patience=50, max_linesearch_steps=30, record_every=0,
        max_records=0,
    )  # fmt: skip
    assert descent_mod.max_rounds(DescentSettings(), 2000) == 5000 // 2000 + 2
    assert lbfgs_mod.max_rounds(LBFGSSettings(), 2000) == 3 * (500_000 + 31) // 2000 + 2


def test_update_stagnation_counts_consecutive_non_decreases():
    fs = [3.0, 2.0, 2.0, 1.0, 1.0, 1.0, 0.0]
    stag, expected = 0, 0
    for old, new in zip(fs[:-1], fs[1:]):
        stag = int(lbfgs_mod.update_stagnation(new, old, stag))
        expected = 0 if new < old else expected + 1
        assert stag == expected


def test_box_and_wrap():
    box = cubic_box(100, 3)
    assert box.dim == 3 and box.volume == pytest.approx(100.0, rel=1e-14)
    rec = box.reciprocal()
    np.testing.assert_allclose(rec @ box.basis.T, 2 * np.pi * np.eye(3), atol=1e-12)
    s = np.array([[-1e-20, 0.5, 1.0], [2.25, -0.75, 0.999999999999]])
    w = wrap_fractional(s)
    assert w.min() >= 0.0 and w.max() < 1.0
    np.testing.assert_array_equal(w[1], [0.25, 0.25, 0.999999999999])
    with pytest.raises(TypeError):
        Box(np.eye(2, dtype=np.float32))
    with pytest.raises(TypeError):
        wrap_fractional(np.zeros(3, np.float32))
    g = np.random.default_rng(0).normal(size=(5, 3))
    np.testing.assert_allclose(box.cartesian_forces(g), -g @ np.linalg.inv(box.basis).T)


def test_factory_pads_and_validates():
    box = cubic_box(12, 2)
    ks = enumerate_kvectors(box.basis, 0.0, 4.0)
    en = make_stealthy_energy(box, ks, chunk_size=7, pad_to=64)
    m = ks.n.shape[0]
    assert en.n_vectors.shape == (-(-m // 64) * 64, 2) and en.n_vectors.dtype == np.float64
    assert en.weights[m:].sum() == 0.0 and en.chunk_size == 7
    with pytest.raises(ValueError, match="empty"):
        make_stealthy_energy(box, enumerate_kvectors(box.basis, 0.0, 1e-3))
    with pytest.raises(ValueError):
        StealthyEnergy(en.n_vectors, en.weights, en.volume, n_max=0)
    with pytest.raises(ValueError):
        StealthyEnergy(en.n_vectors, en.weights, en.volume, n_max=-1)
    with pytest.raises(TypeError):
        en(np.zeros((12, 2), np.float32))  # dtype is checked before any device work


def test_relax_validates_before_device_work():
    box = cubic_box(8, 2)
    en = make_stealthy_energy(box, enumerate_kvectors(box.basis, 0.0, 4.0))
    with pytest.raises(TypeError):
        relax(en, np.zeros((2, 8, 2), np.float32), DescentSettings())
    with pytest.raises(TypeError):
        relax(en, np.zeros((2, 8, 2)), object())


def test_flow_settings_defaults_and_validation():
    import math

    import numpy as np

    from xla_cco.minimize.flow import FlowSettings, gradient_flow

    assert dataclasses.asdict(FlowSettings()) == dict(
        rtol=1e-6, atol=1e-14, parametrization="time", method="dopri5", dt_init=1e-3,
        dt_min=1e-14, dt_max=math.inf, t_max=math.inf, max_steps=200_000, energy_tol=0.0,
        grad_tol=0.0, record_every=0, max_records=0,
    )  # fmt: skip
    s0, basis = np.zeros((4, 2)), np.eye(2)
    bad = [FlowSettings(atol=0.0), FlowSettings(parametrization="x"), FlowSettings(method="x"),
           FlowSettings(method="rosenbrock", parametrization="arclength"),
           FlowSettings(parametrization="arclength", t_max=1.0),
           FlowSettings(record_every=1, max_records=1)]  # fmt: skip
    for st in bad:
        with pytest.raises(ValueError):
            gradient_flow(None, s0, basis, st)
    with pytest.raises(TypeError):
        gradient_flow(None, np.zeros((4, 2), np.float32), basis, FlowSettings())
    with pytest.raises(ValueError):
        gradient_flow(None, s0, np.eye(3), FlowSettings())


def test_top_level_exports_cover_the_reference_package():
    """Every name the reference's package __init__ exports (src/xla_cco/__init__.py:54-100)."""
    import xla_cco

    ref_names = {
        "AbstractEnergy", "Box", "DescentSettings", "KSet", "LBFGSSettings", "PackedConfig",
        "RelaxResult", "StealthyEnergy", "Trajectory", "adaptive_descent", "chi_from_count",
        "collective_density", "cubic_box", "enumerate_kvectors", "g2_from_histogram",
        "isotropic_structure_factor", "k_outer_from_ka", "ka_from_chi", "lbfgs",
        "make_stealthy_energy", "nearest_neighbor_distances", "pair_distance_histogram",
        "read_configpack", "relax", "require_float64", "stack_fractional", "structure_factor",
        "unit_ball_volume", "wrap_fractional", "write_configpack", "write_function_table",
    }  # fmt: skip
    assert ref_names <= set(xla_cco.__all__)
    for name in ref_names:
        assert getattr(xla_cco, name) is not None


def test_auto_chunk_size_as_the_reference():
    from xla_cco.energy import auto_chunk_size

    assert auto_chunk_size(1000, 802) is None                     # 1000 x 802 x 96 B < 1 GiB
    assert auto_chunk_size(20000, 27085) == (1 << 30) // (20000 * 96)
    assert auto_chunk_size(10, 5, budget_bytes=100, bytes_per_pair=96) == 1


def test_device_guard_names_the_cause():
    from xla_cco._device import classify_failure, require_gpu

    assert classify_failure(1, {}, None) is None
    assert "CUDA_VISIBLE_DEVICES" in classify_failure(0, {"CUDA_VISIBLE_DEVICES": ""}, None)
    assert "no CPU path" in classify_failure(0, {}, None)
    assert "cannot be loaded" in classify_failure(0, {}, "libcco.so not found")
    from xla_cco import _native

    if _native.device_count() == 0:
        with pytest.raises(RuntimeError, match="CUDA|GPU"):
            require_gpu()
    else:
        require_gpu()   # a visible device passes the guard
