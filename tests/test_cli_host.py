"""Host logic of the ground-state driver (``src/xla_cco/cli/relax.py``):
input cell conventions, physics set-up, settings and the summary - the parts
that run before and after the device relaxation, checked on the CPU."""

from __future__ import annotations

import math

import numpy as np
import pytest

from xla_cco.cli import relax as cli
from xla_cco.io import PackedConfig, write_configpack
from xla_cco.kvectors import chi_from_count, enumerate_kvectors, k_outer_from_ka, ka_from_chi
from xla_cco.minimize.descent import DescentSettings
from xla_cco.minimize.lbfgs import LBFGSSettings

PHI = 0.05


def _pack(path, n, d, count, basis=None, lo=0.0, hi=1.0):
    rng = np.random.default_rng(5)
    b = np.eye(d) if basis is None else basis
    cfgs = [PackedConfig(b, rng.uniform(lo, hi, size=(n, d)), 1.0, (b"a\x00\x00\x00",) * n)
            for _ in range(count)]  # fmt: skip
    write_configpack(path, cfgs)
    return cfgs


def _args(tmp_path, *extra, dim=2, ka=None):
    ka = ka_from_chi(0.25, PHI, dim) if ka is None else ka
    return cli.build_parser().parse_args([
        "--dim", str(dim), "--ka", repr(ka), "--phi", str(PHI), "--load", str(tmp_path / "in"),
        "--save", str(tmp_path / "out"), *extra])  # fmt: skip


@pytest.mark.parametrize("scale,mode,ok", [(1.0, "auto", True), (1.0, "unit", True), (1.0, "scaled", False),
                                           (4.0, "auto", True), (4.0, "scaled", True), (4.0, "unit", False),
                                           (3.0, "auto", False)])  # fmt: skip
def test_load_input_cell_conventions(tmp_path, scale, mode, ok):
    """N = 16, d = 2: |det| = 1 is the unit convention, 16 (basis x 4) the scaled one."""
    cfgs = _pack(tmp_path / "in", 16, 2, 3, basis=np.eye(2) * scale, lo=-1.5, hi=2.5)
    if not ok:
        with pytest.raises(ValueError, match="N\\^\\(1/d\\)"):
            cli.load_input(tmp_path / "in", 2, mode)
        return
    unit_cfgs, s0, unit = cli.load_input(tmp_path / "in", 2, mode)
    np.testing.assert_allclose(unit, np.eye(2), rtol=0, atol=1e-15)
    assert all(np.allclose(c.basis, np.eye(2)) for c in unit_cfgs)
    assert s0.shape == (3, 16, 2) and s0.min() >= 0.0 and s0.max() < 1.0
    np.testing.assert_array_equal(s0[1], cfgs[1].relative - np.floor(cfgs[1].relative))


def test_load_input_rejects_dimension_mismatch_and_empty(tmp_path):
    _pack(tmp_path / "in", 8, 3, 1)
    with pytest.raises(ValueError, match="--dim 2"):
        cli.load_input(tmp_path / "in", 2)
    with pytest.raises(FileNotFoundError):
        cli.load_input(tmp_path / "missing", 2)


@pytest.mark.parametrize("dim,n,k1a", [(2, 64, 0.0), (3, 125, 0.0), (2, 100, 0.3), (1, 50, 0.0)])
def test_build_physics(tmp_path, dim, n, k1a):
    args = _args(tmp_path, "--k1a", repr(k1a), dim=dim)
    box, energy, info = cli.build_physics(np.eye(dim), n, args)
    k2 = k_outer_from_ka(args.ka, PHI, dim)
    k1 = k_outer_from_ka(k1a, PHI, dim) if k1a > 0 else 0.0
    ks = enumerate_kvectors(np.asarray(box.basis), k1, k2)
    assert info["M"] == ks.n.shape[0] and info["K2"] == k2 and info["K1"] == k1
    assert info["chi"] == chi_from_count(info["M"], n, dim)
    assert math.isclose(info["a"], args.ka / k2, rel_tol=1e-15)
    np.testing.assert_allclose(np.asarray(box.basis), np.eye(dim) * n ** (1.0 / dim), rtol=1e-15)
    assert energy.n_vectors.shape[0] % 64 == 0
    with pytest.raises(ValueError, match="at least 2"):
        cli.build_physics(np.eye(dim), 1, args)


def test_build_physics_sheared_basis(tmp_path):
    unit = np.array([[1.0, 0.0], [0.3, 1.0]])
    box, _, info = cli.build_physics(unit, 64, _args(tmp_path))
    np.testing.assert_allclose(np.asarray(box.basis), unit * 8.0, rtol=1e-15)
    assert info["M"] > 0


def test_make_settings(tmp_path):
    st = cli.make_settings(_args(tmp_path, "--max-steps", "77", "--stop-tol", "1e-25",
                                 "--record-every", "3", "--max-records", "9"))  # fmt: skip
    assert isinstance(st, LBFGSSettings)
    assert st.max_evals_per_pass == 77 and st.energy_tol == 1e-25
    assert st.record_every == 3 and st.max_records == 9
    st = cli.make_settings(_args(tmp_path, "--method", "descent", "--grow", "2.0", "--max-steps", "50"))
    assert isinstance(st, DescentSettings) and st.grow == 2.0 and st.max_evals == 50
    assert cli.make_settings(_args(tmp_path)) == LBFGSSettings()


def test_summarize_counts_and_strict_success():
    out = {"status": np.array([1, 5, 5, 3]), "n_evals": np.array([10, 20, 30, 40]),
           "energy": np.array([1e-21, 1e-20, 5e-21, 1e-3])}  # fmt: skip
    s = cli.summarize(out, 1e-20)
    assert s["n_success"] == 2   # strictly below tol
    assert s["status_counts"] == {"STATUS_ENERGY_TOL": 1, "STATUS_LINESEARCH_FAIL": 2, "STATUS_BUDGET": 1}
    assert s["n_evals"] == {"min": 10, "mean": 25.0, "median": 25.0, "max": 40}


def test_pack_configs_scales_headers():
    tmpl = [PackedConfig(np.eye(2), np.zeros((3, 2)), 1.0, (b"abcd",) * 3)]
    s = np.full((1, 3, 2), 0.25)
    out = cli.pack_configs(tmpl, s, 4.0)
    assert out[0].cell_size == 4.0 and np.array_equal(out[0].basis, np.eye(2) * 4.0)
    assert out[0].names == (b"abcd",) * 3 and np.array_equal(out[0].relative, s[0])
