"""The device MD segment driver (``simulate``) against a host chain: the
integrator step functions (the reference's step API) with forces and
densities from the oracle's direct sums, and the oracle's restatement of the
per-step observables (``src/xla_cco/dynamics/run.py:247-496``): tracked-wave
densities on the wind cadence, centre-of-mass correction, winding, running
sums, the drift guard, snapshots and the rho trace, across chunk boundaries.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import pytest

import oracle
from xla_cco.box import cubic_box
from xla_cco.dynamics import (
    MDSettings,
    andersen_reset,
    baoab_step,
    begin_segment,
    init_state,
    kinetic_energy,
    load_state,
    make_key,
    make_waves,
    md_chunk,
    read_meta,
    select_dt,
    simulate,
    verlet_step,
)
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize.result import STATUS_DRIFT, STATUS_RUNNING

pytestmark = pytest.mark.gpu


def _system(n=48, d=2, chi=0.3):
    box = cubic_box(n, d)
    basis = np.asarray(box.basis)
    k2 = k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d)
    ks = enumerate_kvectors(basis, 0.0, k2)
    en = make_stealthy_energy(box, ks)
    waves = make_waves(basis, k2, 1.4 * k2)
    return en, waves, basis, ks


def _force_fn(ks, basis):
    inv = np.linalg.inv(basis)
    nv = ks.n.astype(np.float64)
    vol = abs(np.linalg.det(basis))

    def force(r):
        s = r @ inv
        phi, g = oracle.energy_direct(s, nv, np.ones(nv.shape[0]), vol)
        re, im = oracle.density_direct(s, nv)
        return phi, -(g @ inv.T), re, im

    return force


def _host_chain(ks, waves, basis, st: MDSettings, r, v, key, temp, n_steps):
    """One lane through n_steps steps; returns a dict of the lane's final state."""
    force = _force_fn(ks, basis)
    n, d = r.shape
    nc, w = waves.n_constrained, waves.n_vectors.shape[0]
    corrected = st.scheme != "verlet"
    phi, f, _, _ = force(r)
    rho, _ = oracle.md_observe(r, basis, waves.n_vectors, waves.kvec, nc, np.zeros((w, 2)), True,
                               corrected)  # fmt: skip
    L = dict(r=r, v=v, f=f, phi=phi, key=key.copy(), acc=0.0, rho=rho, wa=np.zeros(w),
             wn=np.zeros(w), nv=np.zeros(w, np.int64), e0=phi + kinetic_energy(v), md=0.0,
             sk=0.0, sp=0.0, sp2=0.0, ss=np.zeros(w), ns=0, step=0, time=0.0,
             status=STATUS_RUNNING, snaps={}, trace=[])  # fmt: skip
    for _ in range(n_steps):
        if L["status"] != STATUS_RUNNING:
            break
        if st.scheme == "baoab":
            L["key"], r2, v2, out = baoab_step(L["key"], L["r"], L["v"], L["f"], force, st.dt, st.gamma, temp)
        else:
            r2, v2, out = verlet_step(L["r"], L["v"], L["f"], force, st.dt)
            if st.scheme == "andersen":
                L["key"], v2, L["acc"], _ = andersen_reset(L["key"], v2, L["acc"], temp, st.andersen_p,
                                                           st.andersen_mode)  # fmt: skip
        step = L["step"] + 1
        wind = step % st.wind_every == 0
        rho_new, active = oracle.md_observe(r2, basis, waves.n_vectors, waves.kvec, nc, L["rho"], wind,
                                            corrected)  # fmt: skip
        L["rho"], L["wa"], L["wn"], L["nv"] = oracle.md_winding(L["rho"], rho_new, L["wa"], L["wn"], L["nv"],
                                                                active, n, st.phase_floor)  # fmt: skip
        phi, ke = out[0], kinetic_energy(v2)
        drift = abs(phi + ke - L["e0"])
        if st.scheme == "verlet" and math.isfinite(st.drift_tol):
            if not drift <= st.drift_tol * 0.5 * d * (n - 1) * temp:
                L["status"] = STATUS_DRIFT
        L.update(r=r2, v=v2, f=out[1], phi=phi, step=step, time=L["time"] + st.dt, md=max(L["md"], drift),
                 sk=L["sk"] + ke, sp=L["sp"] + phi, sp2=L["sp2"] + phi * phi,
                 ss=L["ss"] + (L["rho"] ** 2).sum(1) / n, ns=L["ns"] + 1)  # fmt: skip
        if step in st.record_steps:
            L["snaps"][step] = (L["time"], L["wa"].copy(), L["wn"].copy(), L["rho"].copy(), r2.copy(), phi, ke)
        if st.record_rho_every > 0 and step % st.record_rho_every == 0 and len(L["trace"]) < st.max_rho_records:
            L["trace"].append((L["rho"].copy(), L["time"]))
    return L


def _start(b, n, d, basis, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(size=(b, n, d)) @ basis, rng.normal(scale=0.5, size=(b, n, d))


@pytest.mark.parametrize("scheme", ["verlet", "andersen", "baoab"])
def test_segment_matches_host_chain(scheme):
    en, waves, basis, ks = _system()
    b, n, d = 2, 48, 2
    r0, v0 = _start(b, n, d, basis, 11)
    st = MDSettings(dt=0.02, scheme=scheme, andersen_p=0.3, andersen_mode="count", gamma=1.5,
                    chunk_steps=5, wind_every=3, record_steps=(2, 5, 9, 40), record_rho_every=2,
                    max_rho_records=4, drift_tol=math.inf)  # fmt: skip
    keys = np.stack([make_key(50 + i) for i in range(b)])
    temps = np.array([0.4, 0.7])
    lanes = init_state(en, waves, basis, r0, v0, temps, keys, st)
    assert np.isfinite(lanes.rho_prev).all() and np.isfinite(lanes.e0).all()
    res = simulate(en, waves, basis, st, lanes, 12)
    S = res.state
    assert (S.step == 12).all() and (S.status == STATUS_RUNNING).all()
    for i in range(b):
        L = _host_chain(ks, waves, basis, st, r0[i], v0[i], keys[i], temps[i], 12)
        np.testing.assert_allclose(S.r[i], L["r"], rtol=0, atol=1e-10)
        np.testing.assert_allclose(S.v[i], L["v"], rtol=0, atol=1e-9)
        np.testing.assert_array_equal(S.key[i], L["key"])
        np.testing.assert_allclose(S.phi[i], L["phi"], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(S.rho_prev[i], L["rho"], rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(S.wind_abs[i], L["wa"], rtol=0, atol=1e-8)
        np.testing.assert_allclose(S.wind_net[i], L["wn"], rtol=0, atol=1e-8)
        np.testing.assert_array_equal(S.n_valid[i], L["nv"])
        np.testing.assert_allclose([S.sum_kinetic[i], S.sum_phi[i], S.sum_phi2[i], S.time[i]],
                                   [L["sk"], L["sp"], L["sp2"], L["time"]], rtol=1e-9)  # fmt: skip
        np.testing.assert_allclose(S.sum_s[i], L["ss"], rtol=1e-9, atol=1e-9)
        assert S.n_sum[i] == L["ns"] == 12
        np.testing.assert_allclose(S.e0[i], L["e0"], rtol=1e-11)
        # snapshots at steps 2, 5, 9 (40 not reached), trace every 2 steps, 4 rows
        assert res.snapshots.count[i] == 3
        assert res.snapshots.step[i].tolist() == [2, 5, 9, -1]
        for j, s in enumerate((2, 5, 9)):
            t, wa, wn, rho, r, phi, ke = L["snaps"][s]
            np.testing.assert_allclose(res.snapshots.time[i, j], t, rtol=1e-12)
            np.testing.assert_allclose(res.snapshots.rho[i, j], rho, rtol=1e-9, atol=1e-9)
            np.testing.assert_allclose(res.snapshots.r[i, j], r, rtol=0, atol=1e-10)
            np.testing.assert_allclose(res.snapshots.wind_abs[i, j], wa, rtol=0, atol=1e-8)
            np.testing.assert_allclose([res.snapshots.phi[i, j], res.snapshots.kinetic[i, j]], [phi, ke],
                                       rtol=1e-9, atol=1e-12)  # fmt: skip
        assert res.trace.count[i] == 4
        for q, (rho, t) in enumerate(L["trace"]):
            np.testing.assert_allclose(res.trace.rho[i, q], rho, rtol=1e-9, atol=1e-9)
            assert res.trace.time[i, q] == pytest.approx(t, rel=1e-12)


def test_reset_winding_repairs_and_continues():
    en, waves, basis, ks = _system()
    r0, v0 = _start(1, 48, 2, basis, 3)
    st = MDSettings(dt=0.02, scheme="baoab", gamma=1.0, chunk_steps=4, drift_tol=math.inf)
    lanes = init_state(en, waves, basis, r0, v0, np.array([0.5]), make_key(9)[None], st)
    lanes = simulate(en, waves, basis, st, lanes, 6).state
    seg = begin_segment(lanes, st, reset_sums=True, reset_winding=True)
    assert np.isnan(seg.rho_prev).all() and seg.n_sum[0] == 0
    # as the reference: simulate(n_steps=0) runs no chunk, the rows stay pending
    assert np.isnan(simulate(en, waves, basis, st, seg, 0).state.rho_prev).all()
    zero = md_chunk(en, waves, basis, st, seg, 0)   # a chunk repairs them before its steps
    want, _ = oracle.md_observe(seg.r[0], basis, waves.n_vectors, waves.kvec, waves.n_constrained,
                                np.zeros_like(seg.rho_prev[0]), True, True)  # fmt: skip
    np.testing.assert_allclose(zero.rho_prev[0], want, rtol=1e-9, atol=1e-9)
    np.testing.assert_array_equal(zero.r, seg.r)
    assert zero.step[0] == 6 and (zero.wind_abs == 0).all()
    one = md_chunk(en, waves, basis, st, seg, 3)   # pending rows are repaired first here too
    assert one.step[0] == 9 and one.n_sum[0] == 3 and np.isfinite(one.rho_prev).all()


def test_drift_guard_stops_and_freezes():
    en, waves, basis, ks = _system()
    r0, v0 = _start(2, 48, 2, basis, 5)
    st = MDSettings(dt=0.05, scheme="verlet", chunk_steps=7, drift_tol=1e-9)
    lanes = init_state(en, waves, basis, r0, v0, np.array([0.3, 0.3]), np.stack([make_key(1)] * 2), st)
    out = simulate(en, waves, basis, st, lanes, 30).state
    assert (out.status == STATUS_DRIFT).all() and (out.step < 30).all()
    again = simulate(en, waves, basis, st, out, 10).state
    for f in ("r", "v", "step", "rho_prev", "sum_phi"):
        np.testing.assert_array_equal(getattr(again, f), getattr(out, f))


def test_single_lane_chunk_and_checkpoint(tmp_path):
    en, waves, basis, ks = _system()
    r0, v0 = _start(2, 48, 2, basis, 8)
    st = MDSettings(dt=0.02, scheme="andersen", andersen_p=0.5, chunk_steps=4, drift_tol=math.inf)
    one = init_state(en, waves, basis, r0[0], v0[0], 0.4, make_key(4), st)
    assert one.r.shape == (48, 2) and np.ndim(one.step) == 0
    c1 = md_chunk(en, waves, basis, st, one, 10)
    assert c1.step == 4
    batch = init_state(en, waves, basis, r0, v0, np.array([0.4, 0.4]), np.stack([make_key(4)] * 2), st)
    res = simulate(en, waves, basis, st, batch, 9, checkpoint=tmp_path / "ck.npz", checkpoint_every_s=1e-9)
    assert read_meta(tmp_path / "ck.npz") == {"source": "xla_cco.dynamics.run.simulate",
                                               "steps_done": 9, "n_steps": 9}  # fmt: skip
    got, _ = load_state(tmp_path / "ck.npz", res.state)
    np.testing.assert_array_equal(got.r, res.state.r)
    np.testing.assert_array_equal(got.trace.rho, res.state.trace.rho)
    with pytest.raises(ValueError):
        simulate(en, waves, basis, st, one, 3)       # unbatched
    with pytest.raises(ValueError):
        simulate(en, waves, basis, st, batch, -1)


def test_waves_must_be_the_energy_rows():
    en, waves, basis, ks = _system()
    r0, v0 = _start(1, 48, 2, basis, 1)
    bad = dataclasses.replace(waves, n_vectors=waves.n_vectors[::-1].copy(), kvec=waves.kvec[::-1].copy())
    with pytest.raises(ValueError, match="constrained"):
        init_state(en, bad, basis, r0, v0, np.array([0.1]), make_key(1)[None], MDSettings())


def test_select_dt():
    en, waves, basis, ks = _system()
    r0, v0 = _start(2, 48, 2, basis, 2)
    st = MDSettings(drift_tol=math.inf)
    lanes = init_state(en, waves, basis, r0, 0.2 * v0, np.array([0.1, 0.1]), np.stack([make_key(2)] * 2), st)
    dt = select_dt(en, waves, basis, lanes, [0.2, 0.05, 0.005], 40, 5e-3)
    assert dt in (0.05, 0.005)
    with pytest.raises(ValueError):
        select_dt(en, waves, basis, lanes, [0.5], 40, 1e-14)


def test_device_resident_state_matches_host_state():
    """CUDA-tensor states stay on the device and give the same results bit for bit."""
    import torch

    en, waves, basis, ks = _system()
    r0, v0 = _start(2, 48, 2, basis, 21)
    st = MDSettings(dt=0.02, scheme="baoab", gamma=1.0, chunk_steps=3, wind_every=2,
                    record_steps=(2, 4), record_rho_every=1, max_rho_records=5, drift_tol=math.inf)  # fmt: skip
    keys = np.stack([make_key(7), make_key(8)])
    host = init_state(en, waves, basis, r0, v0, np.array([0.2, 0.3]), keys, st)
    dev = init_state(en, waves, basis, torch.from_numpy(r0).cuda(), torch.from_numpy(v0).cuda(),
                     np.array([0.2, 0.3]), keys, st)  # fmt: skip
    assert dev.r.is_cuda and dev.snap.rho.is_cuda
    a = simulate(en, waves, basis, st, host, 7).state
    b = simulate(en, waves, basis, st, dev, 7).state
    assert b.r.is_cuda
    for f in ("r", "v", "f", "phi", "rho_prev", "wind_abs", "sum_s", "step", "status"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f).cpu().numpy())
    np.testing.assert_array_equal(a.key, b.key.cpu().numpy().view(np.uint32))
    np.testing.assert_array_equal(a.trace.rho, b.trace.rho.cpu().numpy())
    seg = begin_segment(b, st, True, True)
    assert seg.r.is_cuda and torch.isnan(seg.rho_prev).all()
