"""k-set construction and chi/cutoff conversions: bit-exact with the reference.

Golden values come from the reference's own ``enumerate_kvectors`` and
conversion functions (tests/golden/make_golden.py). Mirrors the reference's
tests/unit/test_kvectors.py:39-142 plus the benchmark problem sizes (d1-d3, N 100-20000).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from xla_cco.box import cubic_box
from xla_cco.kvectors import (
    chi_from_count,
    enumerate_kvectors,
    k_outer_from_ka,
    ka_from_chi,
    unit_ball_volume,
)


def test_kset_bit_exact_vs_reference(golden):
    arrays, meta = golden
    assert len(meta["kset_cases"]) >= 50
    for case in meta["kset_cases"]:
        i = case["i"]
        basis = arrays[f"kset{i}_basis"]
        ks = enumerate_kvectors(basis, float.fromhex(case["k_inner"]), float.fromhex(case["k_outer"]))
        assert ks.n.shape[0] == case["M"], case["name"]
        np.testing.assert_array_equal(ks.n, arrays[f"kset{i}_n"], err_msg=case["name"])
        np.testing.assert_array_equal(ks.k, arrays[f"kset{i}_k"], err_msg=case["name"])
        np.testing.assert_array_equal(ks.k_sq, arrays[f"kset{i}_ksq"], err_msg=case["name"])
        assert ks.n.dtype == np.int64 and ks.k.dtype == np.float64
        np.testing.assert_array_equal(ks.weights, np.ones(ks.n.shape[0]))


def test_baseline_kset_sizes(golden):
    _, meta = golden
    sizes = {c["name"]: c["M"] for c in meta["kset_cases"]}
    assert sizes["cubic_n100_d3_chi0.05"] == 13
    assert sizes["cubic_n1000_d2_chi0.4"] == 802
    assert sizes["cubic_n4000_d3_chi0.45"] == 5413
    assert sizes["cubic_n20000_d3_chi0.45"] == 27085
    assert sizes["cubic_n8000_d1_chi0.49"] == 3919


def test_conversions_bit_exact(golden):
    _, meta = golden
    sc = meta["scalars"]
    for d in (1, 2, 3, 4, 5):
        assert float.hex(unit_ball_volume(d)) == sc[f"unit_ball_volume_{d}"]
    for chi, d in [(0.05, 3), (0.40, 2), (0.45, 3), (0.49, 1), (0.10, 2), (0.25, 2), (0.35, 3)]:
        ka = ka_from_chi(chi, 0.05, d)
        assert float.hex(ka) == sc[f"ka_{chi}_{d}"]
        assert float.hex(k_outer_from_ka(ka, 0.05, d)) == sc[f"k2_{chi}_{d}"]
    assert float.hex(chi_from_count(13, 100, 3)) == sc["chi_13_100_3"]


def test_known_answers_engine_log():
    """C++ engine.log numbers (reference test_kvectors.py:46-73)."""
    assert ka_from_chi(0.05, 0.05, 3) == pytest.approx(0.5963271031078479, rel=1e-14)
    a = (0.05 / unit_ball_volume(3)) ** (1.0 / 3.0)
    assert a == pytest.approx(0.228539, rel=1e-6)
    assert k_outer_from_ka(ka_from_chi(0.05, 0.05, 3), 0.05, 3) == pytest.approx(2.6093, rel=1e-4)
    box = cubic_box(100, 3)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(0.05, 0.05, 3), 0.05, 3))
    assert ks.n.shape == (13, 3)
    assert chi_from_count(13, 100, 3) == pytest.approx(13.0 / 297.0, rel=1e-15)


@pytest.mark.parametrize("side", [1.0, 2.0, 3.7])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_shell_boundary_ulp(side, dim):
    basis = side * np.eye(dim)
    unit = float(oracle.reciprocal_basis(basis)[0, 0])
    assert enumerate_kvectors(basis, 0.0, unit).n.shape[0] == 0
    assert enumerate_kvectors(basis, 0.0, float(np.nextafter(unit, np.inf))).n.shape[0] == dim
    assert enumerate_kvectors(basis, unit, 1.2 * unit).n.shape[0] == 0
    assert enumerate_kvectors(basis, float(np.nextafter(unit, 0.0)), 1.2 * unit).n.shape[0] == dim


def test_rejects_invalid_input():
    eye = np.eye(2)
    for args in [(np.ones((2, 3)), 0.0, 5.0), (np.ones((2, 2)), 0.0, 5.0), (eye, 5.0, 5.0),
                 (eye, -1.0, 5.0), (eye, 0.0, float("inf")),
                 (np.array([[1.0, np.nan], [0.0, 1.0]]), 0.0, 5.0)]:  # fmt: skip
        with pytest.raises(ValueError):
            enumerate_kvectors(*args)


@pytest.mark.parametrize(
    "basis,k2",
    [
        (np.array([[1.0, 0, 0], [8.0, 1, 0], [-6.0, 7, 1]]), 9.0),
        (4.0 * np.array([[1.0, 0, 0], [0.9, 1, 0], [0.7, 0.8, 1]]), 5.0),
        (cubic_box(100, 2).basis, 2.6093),
        (cubic_box(100, 3).basis, 2.6093),
    ],
)
def test_matches_bruteforce_scan(basis, k2):
    ks = enumerate_kvectors(basis, 0.0, k2)
    n_ref, _ = oracle.halfspace_kvectors(basis, 0.0, k2)
    assert {tuple(r) for r in ks.n.tolist()} == {tuple(r) for r in n_ref.tolist()}
    assert ks.n.shape[0] == n_ref.shape[0] > 0


def test_order_and_half_space():
    ks = enumerate_kvectors(cubic_box(1000, 2).basis, 0.0, 4.0)
    first = np.array([r[np.flatnonzero(r)[0]] for r in ks.n])
    assert np.all(first > 0)
    keys = [(q, *r) for q, r in zip(ks.k_sq.tolist(), ks.n.tolist())]
    assert keys == sorted(keys)
    assert math.isclose(chi_from_count(ks.n.shape[0], 1000, 2), ks.n.shape[0] / 1998.0)
