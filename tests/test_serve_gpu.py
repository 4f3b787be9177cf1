"""Serving pool: continuous batching, admission, cancellation, isolation.

The reference has no serving loop, so the contract held here is the one its
relax tests hold per lane (``tests/integration/test_relax.py``: a lane's
result does not depend on the rest of the batch): every request served in a
changing mix of other requests must be bit-identical to the same
configuration relaxed alone through ``relax``. Failures are injected on the
host only (a NaN in an input, a request over the budget, a cancel).
"""

from __future__ import annotations

import time

import numpy as np
import pytest

from xla_cco import _native
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize import relax
from xla_cco.minimize.lbfgs import LBFGSSettings
from xla_cco.minimize.result import STATUS_CANCELLED, STATUS_RUNNING
from xla_cco.serve import RelaxServer

pytestmark = pytest.mark.gpu

SETTINGS = LBFGSSettings(energy_tol=1e-20, max_evals_per_pass=3000)
_CACHE: dict = {}


def _energy(n, d, chi):
    key = (n, d, chi)
    if key not in _CACHE:
        box = cubic_box(n, d)
        ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
        _CACHE[key] = make_stealthy_energy(box, ks)
    return _CACHE[key]


def _requests(count, seed):
    """Seeded requests: N log-uniform in [40, 300], d in {2, 3}, chi in [0.10, 0.45]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(40), np.log(300))))
        d = int(rng.integers(2, 4))
        chi = round(float(rng.uniform(0.10, 0.45)), 2)
        out.append((_energy(n, d, chi), rng.uniform(size=(n, d))))
    return out


def _assert_same_as_alone(res, energy, s0, settings=SETTINGS):
    alone = relax(energy, s0[None], settings)
    np.testing.assert_array_equal(res.s, alone.s[0])
    assert res.energy == float(alone.energy[0])
    assert res.grad_norm == float(alone.grad_norm[0])
    assert res.n_evals == int(alone.n_evals[0])
    assert res.n_iters == int(alone.n_iters[0])
    assert res.status == int(alone.status[0])


def test_same_alone_and_in_the_mix():
    reqs = _requests(16, seed=1)
    with RelaxServer(SETTINGS) as srv:
        first = [srv.submit(e, s) for e, s in reqs[:8]]
        # the second wave arrives while the first runs
        time.sleep(0.002)
        second = [srv.submit(e, s) for e, s in reqs[8:]]
        results = [srv.result(t) for t in first + second]
        st = srv.stats()
    assert st.completed == 16 and st.cancelled == 0
    assert st.rebuilds >= 2, "the running set never changed"
    for (e, s), r in zip(reqs, results):
        assert r.error == _native.CCO_OK
        assert r.status != STATUS_RUNNING
        assert r.done_ns >= r.admit_ns >= r.submit_ns
        _assert_same_as_alone(r, e, s)


def test_admission_budget_bounds_resident_lanes():
    e, s = _requests(1, seed=2)[0]
    with RelaxServer(SETTINGS) as srv:
        srv.result(srv.submit(e, s))
        rec_bytes = srv.stats().peak_bytes
    assert rec_bytes > 0
    with RelaxServer(SETTINGS, hbm_budget_bytes=int(2.5 * rec_bytes)) as srv:
        tickets = [srv.submit(e, s) for _ in range(6)]
        results = [srv.result(t) for t in tickets]
        st = srv.stats()
        # a request larger than the whole budget is refused at submission
        big = _energy(600, 3, 0.45)
        with pytest.raises(_native.CcoError) as err:
            srv.submit(big, np.random.default_rng(0).uniform(size=(600, 3)))
        assert err.value.code == _native.CCO_ERR_ADMISSION
    assert st.peak_bytes <= st.budget_bytes
    assert 1 <= st.peak_lanes <= 2
    for r in results:
        _assert_same_as_alone(r, e, s)


def test_cancel_queued_and_running():
    reqs = _requests(6, seed=3)
    with RelaxServer(SETTINGS, max_lanes=2) as srv:
        tickets = [srv.submit(e, s) for e, s in reqs]
        srv.cancel(tickets[0])    # admitted (or about to be): ends at a graph boundary
        srv.cancel(tickets[5])    # queued behind max_lanes
        results = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert results[5].status == STATUS_CANCELLED
    assert results[0].status != STATUS_RUNNING   # cancelled, unless it finished first
    assert st.cancelled >= 1
    for (e, s), r in zip(reqs[1:5], results[1:5]):
        _assert_same_as_alone(r, e, s)


def test_nan_input_stays_in_its_lane():
    reqs = _requests(4, seed=4)
    e_bad, s_bad = reqs[1]
    s_bad = s_bad.copy()
    s_bad[0, 0] = np.nan
    with RelaxServer(SETTINGS) as srv:
        tickets = [srv.submit(reqs[0][0], reqs[0][1]), srv.submit(e_bad, s_bad)]
        tickets += [srv.submit(e, s) for e, s in reqs[2:]]
        results = [srv.result(t) for t in tickets]
    bad = results[1]
    assert bad.status != STATUS_RUNNING and bad.error == _native.CCO_OK
    for i in (0, 2, 3):
        _assert_same_as_alone(results[i], *reqs[i])


def test_poll_does_not_block_and_releases_the_ticket():
    e, s = _requests(1, seed=5)[0]
    with RelaxServer(SETTINGS) as srv:
        t = srv.submit(e, s)
        early = srv.poll(t, 0.0)
        res = early if early is not None else srv.result(t)
        assert res.status != STATUS_RUNNING
        with pytest.raises(ValueError):
            srv.poll(t, 0.0)


def test_close_cancels_outstanding_requests():
    reqs = _requests(8, seed=6)
    srv = RelaxServer(SETTINGS, max_lanes=1)
    for e, s in reqs:
        srv.submit(e, s)
    srv.close()
    with pytest.raises(RuntimeError):
        srv.stats()
