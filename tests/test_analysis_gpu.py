"""Device parity of the analysis callers: minimum-image pair statistics
(``cco_pair_histogram``, ``cco_nearest_neighbor``) and S(k) from the
evaluation kernels' densities, against the oracle (pinned to the reference's
oracle and its ``_isotropic_kset`` / ``_bin_moments`` by io_golden).

Cases follow ``tests/unit/test_analysis.py`` of the reference: sheared and
cubic cells, the |k| = k_max equality, wide bins, error contracts,
translation invariance, the ideal-gas g2.
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from xla_cco.analysis import (
    g2_from_histogram,
    isotropic_structure_factor,
    nearest_neighbor_distances,
    pair_distance_histogram,
    structure_factor,
)
from xla_cco.box import Box, cubic_box

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
SHEARED_2D = np.array([[1.3, 0.0], [0.4, 0.9]])


@pytest.fixture(scope="module")
def io_golden():
    with np.load(GOLD / "io_golden.npz") as z:
        arrays = {k: z[k] for k in z.files}
    return arrays, json.loads((GOLD / "io_golden.json").read_text())


def _hist_oracle(s: np.ndarray, basis: np.ndarray, edges: np.ndarray) -> np.ndarray:
    tot = np.zeros(edges.size - 1, dtype=np.int64)
    for c in s:
        _, dist = oracle.min_image_distances(c, basis)
        tot += np.histogram(dist, bins=edges)[0]
    return tot


def test_pairs_match_reference_oracle(io_golden):
    z, meta = io_golden
    for c in meta["pairs"]:
        s, basis = z[f"pairs_{c['name']}_s"], z[f"pairs_{c['name']}_basis"]
        box = Box(basis)
        nn = nearest_neighbor_distances(s, box)
        np.testing.assert_allclose(nn, z[f"pairs_{c['name']}_nn"], rtol=1e-12, atol=0)
        dist = z[f"pairs_{c['name']}_dist"]
        edges = np.linspace(0.0, dist.max() * 0.9137, 7)   # clips some pairs
        want = np.histogram(dist, bins=edges)[0]
        np.testing.assert_array_equal(pair_distance_histogram(s[None], box, edges), want)


@pytest.mark.parametrize("n,d,b", [(300, 2, 3), (129, 3, 2), (700, 1, 2), (1000, 2, 1)])
def test_pair_histogram_vs_oracle(n, d, b):
    rng = np.random.default_rng(n + d)
    s = rng.uniform(size=(b, n, d))
    basis = cubic_box(n, d).basis if d != 2 else np.array([[1.0, 0.0], [0.3, 1.1]]) * math.sqrt(n)
    box = Box(np.asarray(basis, dtype=np.float64))
    side = float(np.abs(np.linalg.det(box.basis))) ** (1.0 / d)
    edges = np.linspace(0.0, 0.45 * side, 41)
    np.testing.assert_array_equal(pair_distance_histogram(s, box, edges),
                                  _hist_oracle(s, np.asarray(box.basis), edges))  # fmt: skip
    for i in range(b):
        want, _ = oracle.min_image_distances(s[i], np.asarray(box.basis))
        np.testing.assert_allclose(nearest_neighbor_distances(s[i], box), want, rtol=1e-13, atol=0)


def test_histogram_counts_and_edges():
    s = np.random.default_rng(8).uniform(size=(2, 37, 2))
    box = cubic_box(37, 2)
    big = np.array([0.0, 1e9])
    assert pair_distance_histogram(s, box, big).tolist() == [2 * 37 * 36 // 2]
    # a distance equal to an inner edge goes right, to the last edge stays in
    pts = np.array([[[0.0, 0.0], [0.5, 0.0]]])
    box2 = Box(np.eye(2) * 4.0)   # distance 2 exactly
    assert pair_distance_histogram(pts, box2, np.array([0.0, 2.0, 3.0])).tolist() == [0, 1]
    assert pair_distance_histogram(pts, box2, np.array([0.0, 1.0, 2.0])).tolist() == [0, 1]
    assert pair_distance_histogram(pts, box2, np.array([2.5, 3.0])).tolist() == [0]
    # more bins than the shared-memory histogram holds
    edges = np.linspace(0.0, 3.0, 20001)
    np.testing.assert_array_equal(pair_distance_histogram(s, box, edges),
                                  _hist_oracle(s, np.asarray(box.basis), edges))  # fmt: skip


def test_pair_errors_and_single_particle():
    box = cubic_box(3, 2)
    with pytest.raises(TypeError):
        pair_distance_histogram(np.zeros((1, 3, 2), dtype=np.float32), box, np.array([0.0, 1.0]))
    with pytest.raises(TypeError):
        nearest_neighbor_distances(np.zeros((3, 2), dtype=np.float32), box)
    for bad in (np.array([0.0]), np.array([1.0, 0.5]), np.array([-1.0, 1.0]), np.array([0.0, np.inf])):
        with pytest.raises(ValueError):
            pair_distance_histogram(np.zeros((1, 3, 2)), box, bad)
    got = nearest_neighbor_distances(np.array([[0.3, 0.3]]), Box(np.eye(2) * 2.0))
    assert math.isclose(float(got[0]), 2.0, rel_tol=1e-14)


def test_nn_translation_invariant():
    s = np.random.default_rng(6).uniform(size=(40, 3))
    box = cubic_box(40, 3)
    a = nearest_neighbor_distances(s, box)
    b = nearest_neighbor_distances((s + np.array([0.3, 0.71, 0.05])) % 1.0, box)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


def test_g2_ideal_gas_unity():
    """Poisson gas: E[g2] = (N - 1) / N for fixed-N pairs; within 5 SEM."""
    b, n, d = 200, 50, 2
    s = np.random.default_rng(2024).uniform(size=(b, n, d))
    box = cubic_box(n, d)
    edges = np.linspace(0.0, float(np.asarray(box.basis)[0, 0]) / 2.0, 13)
    per = np.array([g2_from_histogram(pair_distance_histogram(s[i:i + 1], box, edges), edges, n, 1,
                                      float(n), d) for i in range(b)])  # fmt: skip
    mean, sem = per.mean(0), per.std(0, ddof=1) / math.sqrt(b)
    assert np.all(np.abs(mean[1:] - (n - 1) / n) < 5 * sem[1:] + 1e-12)
    tot = g2_from_histogram(pair_distance_histogram(s, box, edges), edges, n, b, float(n), d)
    np.testing.assert_allclose(tot, mean, rtol=1e-12)


def test_structure_factor_vs_reference_oracle(io_golden):
    z, meta = io_golden
    for c in meta["sk"]:
        got = structure_factor(z[f"sk_{c['name']}_s"], z[f"sk_{c['name']}_n"])
        np.testing.assert_allclose(got, z[f"sk_{c['name']}_out"], rtol=1e-11, atol=1e-13)
    s = np.zeros((5, 2))
    np.testing.assert_allclose(structure_factor(s, np.array([[1.0, 2.0], [3.0, -1.0]])), [5.0, 5.0],
                               rtol=1e-14)  # fmt: skip


def _iso_oracle(s, basis, k_dir, k_max, width):
    nv, ksq = oracle.isotropic_kset(basis, k_dir, k_max)
    sk = np.array([oracle.structure_factor_direct(c, nv) for c in s])
    tot, tot2 = np.zeros(nv.shape[0]), np.zeros(nv.shape[0])
    for row in sk:
        tot, tot2 = tot + row, tot2 + row * row
    return oracle.bin_moments(np.sqrt(ksq), tot / s.shape[0], tot2 / s.shape[0], s.shape[0], width)


@pytest.mark.parametrize("basis,k_dir,k_max,width", [
    (np.array([[2.7]]), 5.0, 30.0, 0.01), (SHEARED_2D, 6.0, 14.0, 0.01),
    (np.eye(3) * 1.9, 4.0, 9.0, 0.01), (np.array([[20.0]]), 5.0, 8.0, 0.5),
    (SHEARED_2D * 3.0, 3.0, 10.0, 1.0), (np.eye(3) * 6.0, 2.5, 6.0, 0.5),
])  # fmt: skip
def test_isotropic_sk_vs_oracle(basis, k_dir, k_max, width):
    dim = basis.shape[0]
    s = np.random.default_rng(3 + dim).uniform(size=(3, 7, dim))
    got = isotropic_structure_factor(s, Box(basis), k_dir, k_max, width)
    want = _iso_oracle(s, basis, k_dir, k_max, width)
    assert got[0].shape == want[0].shape
    np.testing.assert_array_equal(got[0], want[0])          # |k| columns: host, bit-exact
    np.testing.assert_array_equal(got[2], want[2])
    np.testing.assert_allclose(got[1], want[1], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(got[3], want[3], rtol=1e-7, atol=1e-9, equal_nan=True)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_isotropic_sk_cutoff_equality_included(dim):
    basis = np.eye(dim) * (2.0 * math.pi)
    s = np.random.default_rng(20 + dim).uniform(size=(2, 4, dim))
    got = isotropic_structure_factor(s, Box(basis), 3.0, 5.0, 0.01)
    want = _iso_oracle(s, basis, 3.0, 5.0, 0.01)
    assert got[0].max() == 5.0 and got[0].shape == want[0].shape
    np.testing.assert_allclose(got[1], want[1], rtol=1e-10, atol=1e-12)


def test_isotropic_sk_cli_sized_and_invariance():
    """The driver's k-set (5, 400) at N = 64, d = 2 (6202 vectors) and
    translation invariance of S(k)."""
    s = np.random.default_rng(4).uniform(size=(4, 64, 2))
    box = cubic_box(64, 2)
    a = isotropic_structure_factor(s, box, 5.0, 400.0)
    b = isotropic_structure_factor((s + np.array([0.37, 0.81])) % 1.0, box, 5.0, 400.0)
    np.testing.assert_allclose(a[1], b[1], rtol=1e-9, atol=1e-9)
    assert a[0].size > 100 and np.all(np.isfinite(a[1]))


def test_isotropic_sk_error_contracts():
    box = cubic_box(7, 2)
    with pytest.raises(TypeError):
        isotropic_structure_factor(np.zeros((2, 7, 2), dtype=np.float32), box)
    with pytest.raises(ValueError):
        isotropic_structure_factor(np.zeros((7, 2)), box)
    with pytest.raises(ValueError):
        isotropic_structure_factor(np.zeros((2, 7, 2)), box, k_dir_max=9.0, k_max=3.0)
