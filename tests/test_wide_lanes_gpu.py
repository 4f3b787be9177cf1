"""Wide lanes: configurations whose L-BFGS history rows exceed 1024 double2
words (N d > 2048) take the finer-split history passes (element chunks in
pass A, pair groups in pass B), and wide 1-D k-sets split their pass-1
segments over several CTAs when a launch has few tiles.

Both splits follow from the lane's own size (the pass-1 chunk count is a
launch-level choice whose segment sums are unchanged), so the reference's
per-lane contract still holds bit for bit: a lane relaxed in a mixed batch
equals the same configuration relaxed alone (``minimize/__init__.py:102-151``,
``tests/integration/test_relax.py`` per-lane stopping). The split passes are
an L-BFGS direction like any other: a wide lane relaxed to 1e-20 must end as
the oracle's run of the same seeds does (``minimize/lbfgs.py:200-350``).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import RTOL_KERNEL_E, energy_atol
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize import relax, relax_mixed
from xla_cco.minimize.lbfgs import LBFGSSettings

pytestmark = pytest.mark.gpu

FIELDS = ("s", "energy", "grad_norm", "n_evals", "n_iters", "status")


def _problem(n, d, chi):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return box, ks, make_stealthy_energy(box, ks)


def test_wide_lanes_in_a_mixed_batch_equal_lone_runs():
    # d=1 N=5000 chi=0.45: 2500-word history rows and 282 pass-1 segments, split
    # over two CTAs per tile when the lane runs alone but not in this batch (six
    # of them fill the launch); d=2 N=1300, d=3 N=800: wide history rows; and
    # narrow lanes.
    shapes = [(5000, 1, 0.45)] * 6 + [(1300, 2, 0.30), (800, 3, 0.20), (300, 2, 0.40),
                                      (120, 3, 0.30), (900, 1, 0.35)]
    rng = np.random.default_rng(11)
    cache = {}
    probs = [cache.setdefault(sh, _problem(*sh)) for sh in shapes]
    s0s = [rng.uniform(size=(n, d)) for n, d, _ in shapes]
    st = LBFGSSettings(energy_tol=1e-20, max_evals_per_pass=150)
    res = relax_mixed([en for _, _, en in probs], s0s, st)
    for i, ((box, ks, en), s0, r) in enumerate(zip(probs, s0s, res)):
        alone = relax(en, s0[None], st)
        for f in FIELDS:
            a, b = np.asarray(getattr(r, f)), np.asarray(getattr(alone, f))
            assert np.array_equal(a, b), f"lane {i} {shapes[i]}: {f} differs from the lone run"
        e_ref, _ = oracle.energy_grad_accurate(r.s, ks.n, ks.weights, box.volume)
        atol = energy_atol(s0.shape[0], ks.n.shape[0], float(e_ref[0]))
        np.testing.assert_allclose(float(r.energy[0]), float(e_ref[0]), rtol=RTOL_KERNEL_E, atol=atol)


def test_wide_lbfgs_lanes_end_as_the_oracle_does():
    n, d, chi = 1100, 2, 0.40   # 1100 double2 words per history row: two pass-A chunks
    box, ks, en = _problem(n, d, chi)
    s0 = np.random.default_rng(5).uniform(size=(3, n, d))
    st = LBFGSSettings(energy_tol=1e-20)
    res = relax(en, s0, st)
    ref = oracle.relax_lanes("lbfgs", s0, ks.n, ks.weights, box.volume, oracle.lbfgs_settings(energy_tol=1e-20))
    np.testing.assert_array_equal(res.status, ref["status"])
    np.testing.assert_array_equal(res.energy < 1e-20, ref["energy"] < 1e-20)
    assert (res.energy < 1e-20).all()
    # the iterates are not pinned (the reference takes them from optax), but a
    # direction that lost a pair group or a chunk would cost far more evaluations
    np.testing.assert_allclose(res.n_evals, ref["n_evals"], rtol=0.3)
    e_chk, _ = oracle.energy_grad_accurate(res.s, ks.n, ks.weights, box.volume)
    for i in range(s0.shape[0]):
        atol = energy_atol(n, ks.n.shape[0], float(e_chk[i]))
        np.testing.assert_allclose(res.energy[i], e_chk[i], rtol=RTOL_KERNEL_E, atol=atol)
