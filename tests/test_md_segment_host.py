"""Host logic of the MD segment driver: settings validation, tracked waves,
begin_segment, checkpoints, thermal helpers (``src/xla_cco/dynamics/*``)."""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import pytest

from xla_cco.dynamics import (
    CheckpointError,
    MDSettings,
    MDState,
    RhoTrace,
    Snapshots,
    begin_segment,
    kinetic_energy,
    kinetic_temperature,
    load_state,
    make_key,
    make_waves,
    maxwell_boltzmann,
    read_meta,
    save_state,
)
from xla_cco.dynamics.run import _check_settings
from xla_cco.kvectors import enumerate_kvectors
from xla_cco.minimize.result import STATUS_DRIFT, STATUS_RUNNING


def _state(b=2, n=5, d=2, w=3, R=2, Q=3, seed=0) -> MDState:
    rng = np.random.default_rng(seed)
    f = lambda *s: rng.normal(size=s)  # noqa: E731
    return MDState(
        r=f(b, n, d), v=f(b, n, d), f=f(b, n, d), phi=f(b), temperature=np.abs(f(b)),
        key=rng.integers(0, 2**32, size=(b, 2), dtype=np.uint32), step=np.arange(b, dtype=np.int64),
        time=f(b), reset_acc=f(b), rho_prev=f(b, w, 2), wind_abs=f(b, w), wind_net=f(b, w),
        n_valid=np.ones((b, w), np.int64), e0=f(b), max_drift=f(b), sum_kinetic=f(b), sum_phi=f(b),
        sum_phi2=f(b), sum_s=f(b, w), n_sum=np.full(b, 3, np.int64),
        status=np.array([STATUS_RUNNING, STATUS_DRIFT][:b], np.int64),
        snap=Snapshots(step=np.full((b, R), -1, np.int64), time=f(b, R), wind_abs=f(b, R, w),
                       wind_net=f(b, R, w), rho=f(b, R, w, 2), r=f(b, R, n, d), phi=f(b, R),
                       kinetic=f(b, R), count=np.zeros(b, np.int64)),
        trace=RhoTrace(rho=f(b, Q, w, 2), time=f(b, Q), count=np.zeros(b, np.int64)),
    )  # fmt: skip


@pytest.mark.parametrize("bad", [
    dict(scheme="leapfrog"), dict(andersen_mode="always"), dict(dt=0.0), dict(dt=math.inf),
    dict(andersen_p=1.5), dict(gamma=-1.0), dict(chunk_steps=0), dict(wind_every=0),
    dict(record_steps=(3, 2)), dict(record_steps=(0,)), dict(record_steps=tuple(range(1, 258))),
    dict(record_rho_every=2, max_rho_records=0), dict(phase_floor=-1.0), dict(drift_tol=0.0),
])  # fmt: skip
def test_settings_rejected(bad):
    with pytest.raises(ValueError):
        _check_settings(MDSettings(**bad))
    _check_settings(MDSettings(drift_tol=math.inf, record_steps=(1, 5)))


def test_make_waves_constrained_first():
    basis = np.eye(2) * 6.0
    w = make_waves(basis, 2.0, 3.5)
    inner = enumerate_kvectors(basis, 0.0, 2.0)
    outer = enumerate_kvectors(basis, 2.0, 3.5)
    assert w.n_constrained == inner.n.shape[0]
    np.testing.assert_array_equal(w.n_vectors, np.concatenate([inner.n, outer.n]).astype(float))
    np.testing.assert_allclose(w.kvec, w.n_vectors @ (2 * math.pi * np.linalg.inv(basis).T))
    assert w.constrained.sum() == w.n_constrained and w.constrained[:w.n_constrained].all()
    same = make_waves(basis, 2.0, 2.0)
    assert same.n_vectors.shape[0] == same.n_constrained
    for args in ((0.0, 1.0), (2.0, 1.0), (1.0, math.inf), (0.1, 0.2)):
        with pytest.raises(ValueError):
            make_waves(basis, *args)


@pytest.mark.parametrize("reset_sums,reset_winding", [(False, False), (True, False), (True, True)])
def test_begin_segment(reset_sums, reset_winding):
    st = _state()
    out = begin_segment(st, MDSettings(remove_com=True), reset_sums, reset_winding)
    # lane 0 runs: COM momentum removed, e0 = phi + KE, drift reset
    np.testing.assert_allclose(out.v[0].mean(0), 0.0, atol=1e-15)
    assert out.e0[0] == st.phi[0] + kinetic_energy(out.v[0])
    assert out.max_drift[0] == 0.0
    assert (out.sum_phi[0] == 0.0) == reset_sums and (out.n_sum[0] == 0) == reset_sums
    assert np.isnan(out.rho_prev[0]).all() == reset_winding
    assert (out.wind_abs[0] == 0.0).all() == reset_winding
    # lane 1 (stopped) is untouched
    for f in dataclasses.fields(MDState):
        if f.name not in ("snap", "trace"):
            np.testing.assert_array_equal(getattr(out, f.name)[1], getattr(st, f.name)[1])
    np.testing.assert_array_equal(out.r, st.r)
    keep = begin_segment(st, MDSettings(remove_com=False), False, False)
    np.testing.assert_array_equal(keep.v, st.v)


def test_checkpoint_round_trip(tmp_path):
    st = _state()
    save_state(tmp_path / "c.npz", st, {"steps_done": 3})
    assert read_meta(tmp_path / "c.npz") == {"steps_done": 3}
    got, meta = load_state(tmp_path / "c.npz", st)
    assert meta["steps_done"] == 3
    for f in dataclasses.fields(MDState):
        a, b = getattr(got, f.name), getattr(st, f.name)
        if f.name in ("snap", "trace"):
            for g in dataclasses.fields(a):
                np.testing.assert_array_equal(getattr(a, g.name), getattr(b, g.name))
        else:
            np.testing.assert_array_equal(a, b)
    with pytest.raises(CheckpointError):
        load_state(tmp_path / "c.npz", _state(w=4))
    (tmp_path / "bad.npz").write_bytes(b"not a zip")
    with pytest.raises(CheckpointError):
        read_meta(tmp_path / "bad.npz")
    with pytest.raises(TypeError):
        save_state(tmp_path / "x.npz", st, {"x": object()})
    assert not (tmp_path / "x.npz").exists() and not (tmp_path / "x.npz.tmp").exists()


# The reference's leaf order (jax.tree_util flattening of its MDState,
# src/xla_cco/dynamics/state.py:129-164): fields in declaration order, the
# Snapshots and RhoTrace buffers flattened in place.
_REFERENCE_LEAVES = (
    "r", "v", "f", "phi", "temperature", "key", "step", "time", "reset_acc", "rho_prev",
    "wind_abs", "wind_net", "n_valid", "e0", "max_drift", "sum_kinetic", "sum_phi", "sum_phi2",
    "sum_s", "n_sum", "status", "snap.step", "snap.time", "snap.wind_abs", "snap.wind_net",
    "snap.rho", "snap.r", "snap.phi", "snap.kinetic", "snap.count", "trace.rho", "trace.time",
    "trace.count",
)  # fmt: skip


def _field(state, dotted):
    obj = state
    for name in dotted.split("."):
        obj = getattr(obj, name)
    return np.asarray(obj)


def test_checkpoint_reads_and_writes_the_reference_layout(tmp_path):
    """A file in the reference's layout (leaf_NNN, __n_leaves__, __meta__),
    written here by hand, loads into the right fields; our own files have
    exactly that layout, key as uint32[2]."""
    st = _state()
    arrays = {f"leaf_{i:03d}": _field(st, name) for i, name in enumerate(_REFERENCE_LEAVES)}
    arrays["__n_leaves__"] = np.int64(len(_REFERENCE_LEAVES))
    arrays["__meta__"] = np.asarray('{"chunk": 7}')
    np.savez(tmp_path / "ref.npz", **arrays)
    got, meta = load_state(tmp_path / "ref.npz", st)
    assert meta == {"chunk": 7}
    for name in _REFERENCE_LEAVES:
        np.testing.assert_array_equal(_field(got, name), _field(st, name))
    save_state(tmp_path / "ours.npz", st, {"chunk": 7})
    with np.load(tmp_path / "ours.npz") as z:
        assert sorted(z.files) == sorted(arrays)
        assert int(z["__n_leaves__"]) == len(_REFERENCE_LEAVES)
        for i, name in enumerate(_REFERENCE_LEAVES):
            np.testing.assert_array_equal(z[f"leaf_{i:03d}"], _field(st, name))
        assert z["leaf_005"].dtype == np.uint32 and z["leaf_005"].shape[-1] == 2
    # a wrong leaf count is a CheckpointError naming both counts
    arrays["__n_leaves__"] = np.int64(32)
    np.savez(tmp_path / "short.npz", **arrays)
    with pytest.raises(CheckpointError, match="32 leaves"):
        load_state(tmp_path / "short.npz", st)


def test_thermal_helpers():
    key = make_key(3)
    v = maxwell_boltzmann(key, 4000, 3, 2.0, remove_com=True)
    assert v.shape == (4000, 3)
    np.testing.assert_allclose(v.mean(0), 0.0, atol=1e-12)
    assert abs(kinetic_temperature(v, 3 * 3999) - 2.0) < 0.1
    np.testing.assert_array_equal(maxwell_boltzmann(key, 5, 2, 1.0, False),
                                  maxwell_boltzmann(key, 5, 2, 1.0, False))  # fmt: skip
    with pytest.raises(TypeError):
        maxwell_boltzmann(np.array([1, 2], dtype=np.int64), 2, 2, 1.0, False)
    with pytest.raises(ValueError):
        maxwell_boltzmann(key, 0, 2, 1.0, False)
    with pytest.raises(ValueError):
        kinetic_temperature(v, 0)


def test_observable_helpers_match_the_oracle():
    """com_correct and winding_update (the reference's observables API) against
    the oracle's restatement used for the device parity tests."""
    import oracle
    from xla_cco.dynamics import center_of_mass, com_correct, winding_update

    rng = np.random.default_rng(4)
    w, n = 9, 30
    rho_old, rho_new = rng.normal(size=(w, 2)) * 3, rng.normal(size=(w, 2)) * 3
    rho_new[0] = 0.0                      # below the phase floor: no winding
    kvec = rng.normal(size=(w, 2))
    r = rng.uniform(size=(n, 2)) * 5
    rcm = center_of_mass(r)
    np.testing.assert_allclose(rcm, r.mean(0))
    got = com_correct(rho_new, kvec, rcm)
    ph = kvec @ rcm
    want = np.stack([rho_new[:, 0] * np.cos(ph) + rho_new[:, 1] * np.sin(ph),
                     rho_new[:, 1] * np.cos(ph) - rho_new[:, 0] * np.sin(ph)], -1)  # fmt: skip
    np.testing.assert_allclose(got, want, rtol=1e-15, atol=1e-15)
    np.testing.assert_allclose(np.hypot(*got.T), np.hypot(*rho_new.T), rtol=1e-14)  # a pure phase
    active = np.array([True] * 6 + [False] * 3)
    args = (rho_old, rho_new, np.ones(w), np.full(w, 0.5), np.arange(w, dtype=np.int64), active, n, 1e-16)
    mine = winding_update(*args)
    ref = oracle.md_winding(*args)
    for a, b in zip(mine, ref):
        np.testing.assert_array_equal(a, b)
    assert mine[3][0] == 0 and mine[3][1] == 2   # zero density: not counted; active: +1
    np.testing.assert_array_equal(mine[0][6:], rho_old[6:])   # inactive rows keep rho_prev
