"""The ground-state driver end to end on the GPU (``xla_cco.cli.relax``).

Follows ``tests/integration/test_cli.py`` of the reference: output files and
headers, the strict Success selection, the wrapped InitConfig, K1 sharing a,
trajectories independent of the batch size, reading its own output, the
input-basis conventions, and S(k) of exactly the Success set.
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from xla_cco.analysis.structure import isotropic_structure_factor
from xla_cco.box import cubic_box
from xla_cco.cli import relax as cli
from xla_cco.io import PackedConfig, read_configpack, write_configpack
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi

pytestmark = pytest.mark.gpu
PHI = 0.05
LOG_KEYS = {"args", "N", "d", "M", "chi", "a", "K1", "K2", "tol", "method", "settings",
            "status_counts", "n_success", "n_evals", "wall_seconds", "jax_version", "device"}


def _pack(path: Path, n: int, d: int, count: int, basis=None):
    rng = np.random.default_rng(7)
    b = np.eye(d) if basis is None else basis
    cfgs = [PackedConfig(b, rng.uniform(size=(n, d)), 1.0, (b"a\x00\x00\x00",) * n)
            for _ in range(count)]  # fmt: skip
    write_configpack(path, cfgs)
    return cfgs


def _args(tmp_path: Path, *extra: str, ka: float, dim: int = 2):
    return cli.build_parser().parse_args([
        "--dim", str(dim), "--ka", repr(ka), "--phi", str(PHI), "--load", str(tmp_path / "in"),
        "--save", str(tmp_path / "out"), *extra])  # fmt: skip


def _ka() -> float:
    return ka_from_chi(0.25, PHI, 2)


def _table(path: Path) -> np.ndarray:
    rows = [r.split("\t")[:4] for r in path.read_text().splitlines()]
    return np.array([[float(x) for x in r] for r in rows])


@pytest.mark.parametrize("method", ["lbfgs", "descent"])
def test_end_to_end_small(tmp_path, method):
    cfgs = _pack(tmp_path / "in", 64, 2, 4)
    extra = ["--method", method, "--batch-size", "3"]
    if method == "descent":
        extra += ["--max-steps", "50000", "--grow", "2.0"]
    summary = cli.run(_args(tmp_path, *extra, ka=_ka()))
    assert summary["n_success"] >= 1 and abs(summary["chi"] - 0.25) < 0.03
    for suffix in (".ConfigPack", ".ConfigPackIndex", "_Success.ConfigPack", "_InitConfig.ConfigPack",
                   "_Sk.txt", "_g2.txt", "_Hp.txt", "_energies.npy", "_log.json"):  # fmt: skip
        assert Path(str(tmp_path / "out") + suffix).is_file(), suffix
    energies = np.load(tmp_path / "out_energies.npy")
    succ = read_configpack(tmp_path / "out_Success")
    assert len(succ) == int((energies < summary["tol"]).sum()) == summary["n_success"]
    for name in ("out", "out_InitConfig"):
        for c in read_configpack(tmp_path / name):
            assert c.cell_size == 8.0 and np.array_equal(c.basis, np.eye(2) * 8.0)
            assert c.names == cfgs[0].names
            assert c.relative.min() >= 0.0 and c.relative.max() < 1.0
    log = json.loads((tmp_path / "out_log.json").read_text())
    assert set(log) >= LOG_KEYS
    # the written energies are the oracle's energies of the written positions
    en = cli.build_physics(np.eye(2), 64, _args(tmp_path, ka=_ka()))[1]
    relaxed = read_configpack(tmp_path / "out")
    nv = np.asarray(en.n_vectors)[np.asarray(en.weights) != 0]
    for c, e in zip(relaxed, energies):
        phi, _ = oracle.energy_direct(c.relative, nv, np.ones(nv.shape[0]), 64.0)
        assert abs(phi - e) <= 1e-12 * phi + 1e-18


def test_mixed_success_selects_exact_configs(tmp_path):
    cfgs = _pack(tmp_path / "in", 64, 2, 4)
    base = ["--dim", "2", "--ka", repr(_ka()), "--phi", str(PHI), "--load", str(tmp_path / "in")]
    cli.run(cli.build_parser().parse_args([*base, "--save", str(tmp_path / "probe"),
                                           "--max-steps", "60"]))  # fmt: skip
    e = np.sort(np.load(tmp_path / "probe_energies.npy"))
    tol = float(np.sqrt(e[1] * e[2]))
    assert e[1] < tol < e[2]
    summary = cli.run(cli.build_parser().parse_args([*base, "--save", str(tmp_path / "out"),
                                                     "--max-steps", "60", "--tol", repr(tol)]))  # fmt: skip
    energies = np.load(tmp_path / "out_energies.npy")
    ok = energies < summary["tol"]
    assert ok.sum() == 2 == summary["n_success"]
    relaxed = read_configpack(tmp_path / "out")
    succ = read_configpack(tmp_path / "out_Success")
    for got, want in zip(succ, [c for c, f in zip(relaxed, ok) if f]):
        assert np.array_equal(got.relative, want.relative)
    for got, inp in zip(read_configpack(tmp_path / "out_InitConfig"), cfgs):
        assert np.array_equal(got.relative, inp.relative - np.floor(inp.relative))
    s_succ = np.stack([c.relative for c in succ])
    want_sk = isotropic_structure_factor(s_succ, cubic_box(64, 2), 5.0, 400.0)
    sk = _table(tmp_path / "out_Sk.txt")
    for j in range(4):
        np.testing.assert_allclose(sk[:, j], want_sk[j], rtol=1e-9, atol=0.0, equal_nan=True)
    g2 = _table(tmp_path / "out_g2.txt")
    assert g2.shape == (200, 4)
    assert math.isclose(g2[-1, 0] + g2[-1, 2], 0.2 * 8.0, rel_tol=1e-12)
    hp = _table(tmp_path / "out_Hp.txt")
    assert hp.shape == (200, 4) and math.isclose((hp[:, 1] * 2 * hp[:, 2]).sum(), 1.0, rel_tol=1e-9)


def test_records_trajectory_and_batch_independence(tmp_path):
    _pack(tmp_path / "in", 64, 2, 3)
    rec = ["--record-every", "5", "--max-records", "4", "--max-steps", "60"]
    cli.run(_args(tmp_path, *rec, "--batch-size", "2", ka=_ka()))
    multi = dict(np.load(tmp_path / "out_traj.npz"))
    cli.run(_args(tmp_path, *rec, "--batch-size", "8", ka=_ka()))
    single = dict(np.load(tmp_path / "out_traj.npz"))
    assert multi["s"].shape == (3, 4, 64, 2) and multi["energy"].shape == (3, 4)
    assert multi["iteration"].shape == (3, 4) and multi["count"].shape == (3,)
    np.testing.assert_array_equal(multi["count"], single["count"])
    # the reference's batch-independence tolerances (ATOL_VMAP_S, RTOL_VMAP_E)
    np.testing.assert_allclose(multi["s"], single["s"], rtol=0.0, atol=1e-12)
    np.testing.assert_allclose(multi["energy"], single["energy"], rtol=1e-9, atol=0.0)


def test_no_success_skips_analysis(tmp_path):
    _pack(tmp_path / "in", 64, 2, 2)
    summary = cli.run(_args(tmp_path, "--max-steps", "2", ka=_ka()))
    assert summary["n_success"] == 0 and "skipped" in summary["analysis"]
    for suffix in ("_Success.ConfigPack", "_Sk.txt", "_g2.txt", "_Hp.txt"):
        assert not Path(str(tmp_path / "out") + suffix).exists()
    assert (tmp_path / "out_InitConfig.ConfigPack").is_file()


def test_init_config_is_wrapped_input(tmp_path):
    rel = np.random.default_rng(3).uniform(-2.0, 3.0, size=(64, 2))
    write_configpack(tmp_path / "in", [PackedConfig(np.eye(2), rel, 1.0, (b"a\x00\x00\x00",) * 64)])
    cli.run(_args(tmp_path, "--max-steps", "2", ka=_ka()))
    got = read_configpack(tmp_path / "out_InitConfig")[0].relative
    assert np.array_equal(got, rel - np.floor(rel)) and got.max() < 1.0


def test_k1_uses_shared_a(tmp_path):
    _pack(tmp_path / "in", 64, 2, 1)
    summary = cli.run(_args(tmp_path, "--k1a", "0.2", "--max-steps", "2", ka=_ka()))
    k1, k2 = k_outer_from_ka(0.2, PHI, 2), k_outer_from_ka(_ka(), PHI, 2)
    log = json.loads((tmp_path / "out_log.json").read_text())
    assert log["K1"] == k1 and log["K2"] == k2 == summary["K2"]
    m = enumerate_kvectors(np.eye(2) * 8.0, k1, k2).n.shape[0]
    assert log["M"] == m < enumerate_kvectors(np.eye(2) * 8.0, 0.0, k2).n.shape[0]


def test_reads_its_own_output_and_basis_modes(tmp_path):
    _pack(tmp_path / "in", 16, 2, 3)
    first = cli.run(_args(tmp_path, ka=_ka()))
    again = tmp_path / "again"
    again.mkdir()
    argv = _args(tmp_path, ka=_ka())
    argv.load, argv.save = tmp_path / "out", again / "out"
    second = cli.run(argv)
    assert second["n_configs"] == first["n_configs"] == 3
    for a, b in zip(read_configpack(tmp_path / "out"), read_configpack(again / "out")):
        np.testing.assert_allclose(a.basis, b.basis)
    _pack(tmp_path / "in", 16, 2, 2, basis=np.eye(2) * 3.0)
    with pytest.raises(ValueError, match=r"N\^\(1/d\)"):
        cli.run(_args(tmp_path, ka=_ka()))
    for scale, mode in ((1.0, "scaled"), (4.0, "unit")):
        _pack(tmp_path / "in", 16, 2, 2, basis=np.eye(2) * scale)
        with pytest.raises(ValueError, match=f"--input-basis {mode}"):
            cli.run(_args(tmp_path, "--input-basis", mode, ka=_ka()))
    _pack(tmp_path / "in", 16, 2, 2)
    with pytest.raises(ValueError, match="--dim"):
        cli.run(_args(tmp_path, ka=_ka(), dim=3))


@pytest.mark.parametrize("dim,n", [(1, 50), (3, 100)])
def test_other_dimensions(tmp_path, dim, n):
    _pack(tmp_path / "in", n, dim, 2)
    ka = ka_from_chi(0.2, PHI, dim)
    summary = cli.run(_args(tmp_path, "--tol", "9.99999968e-21", ka=ka, dim=dim))
    assert summary["N"] == n and summary["d"] == dim
    assert len(read_configpack(tmp_path / "out")) == 2
