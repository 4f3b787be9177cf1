"""Host-side parity of the callers around the path: ConfigPack, function
tables, the isotropic S(k) k-set and binning, g2 normalisation, the pair
oracle, and the ground-state driver's argument handling and tables.

Golden data: tests/golden/io_golden.* (``make_io_golden.py``), written by the
reference's own ConfigPack and table writers, its ``_isotropic_kset`` and
``_bin_moments`` (``src/xla_cco/analysis/structure.py:113-201``) and its test
oracle. Example values follow the reference's tests
(``tests/unit/test_configpack.py``, ``test_tables.py``, ``test_analysis.py``,
``tests/integration/test_cli.py``).
"""

from __future__ import annotations

import hashlib
import json
import math
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from xla_cco.analysis.pairs import g2_from_histogram
from xla_cco.analysis.structure import _bin_moments, _isotropic_kset
from xla_cco.cli import relax as cli
from xla_cco.io import PackedConfig, read_configpack, stack_fractional, write_configpack
from xla_cco.io.tables import write_function_table

GOLD = Path(__file__).resolve().parent / "golden"
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def io_golden():
    with np.load(GOLD / "io_golden.npz") as z:
        arrays = {k: z[k] for k in z.files}
    return arrays, json.loads((GOLD / "io_golden.json").read_text())


def _cfg(n, d, seed=0, scale=1.0, cell=1.5):
    rng = np.random.default_rng(seed)
    return PackedConfig(np.eye(d) * scale, rng.uniform(size=(n, d)), cell,
                        tuple(bytes([97 + i % 26, 0, 0, 0]) for i in range(n)))  # fmt: skip


def _names(raw: np.ndarray) -> tuple:
    b = raw.tobytes()
    return tuple(b[i:i + 4] for i in range(0, len(b), 4))


# ------------------------------------------------------------------ ConfigPack


def test_reader_decodes_reference_bytes(tmp_path, io_golden):
    z, meta = io_golden
    for g in meta["packs"]:
        prefix = tmp_path / f"g{g['group']}"
        Path(f"{prefix}.ConfigPack").write_bytes(z[f"pack{g['group']}_bytes"].tobytes())
        Path(f"{prefix}.ConfigPackIndex").write_bytes(z[f"pack{g['group']}_index"].tobytes())
        got = read_configpack(prefix)
        assert len(got) == g["count"]
        for i, c in enumerate(got):
            np.testing.assert_array_equal(c.basis, z[f"pack{g['group']}_{i}_basis"])
            np.testing.assert_array_equal(c.relative, z[f"pack{g['group']}_{i}_rel"])
            assert c.names == _names(z[f"pack{g['group']}_{i}_names"])
            assert c.cell_size == g["cells"][i]


def test_writer_reproduces_reference_bytes(tmp_path, io_golden):
    z, meta = io_golden
    for g in meta["packs"]:
        k = g["group"]
        cfgs = [PackedConfig(z[f"pack{k}_{i}_basis"], z[f"pack{k}_{i}_rel"], g["cells"][i],
                             _names(z[f"pack{k}_{i}_names"])) for i in range(g["count"])]  # fmt: skip
        write_configpack(tmp_path / f"w{k}", cfgs)
        assert Path(f"{tmp_path}/w{k}.ConfigPack").read_bytes() == z[f"pack{k}_bytes"].tobytes()
        assert Path(f"{tmp_path}/w{k}.ConfigPackIndex").read_bytes() == z[f"pack{k}_index"].tobytes()


def test_bundled_inputs_reencode_to_the_same_files(tmp_path, io_golden):
    """The reference's bundled input packs, decoded by its reader, re-encode to
    files with the original SHA-256 and stack to the same fractional array."""
    z, meta = io_golden
    assert len(meta["inputs"]) == 6
    for inp in meta["inputs"]:
        key = inp["name"]
        names = _names(z[f"in_{key}_names"])
        s, bases = z[f"in_{key}_s"], z[f"in_{key}_bases"]
        n = s.shape[1]
        cfgs = [PackedConfig(bases[i], s[i], inp["cells"][i], names[i * n:(i + 1) * n])
                for i in range(inp["count"])]  # fmt: skip
        write_configpack(tmp_path / key, cfgs)
        pack = Path(f"{tmp_path}/{key}.ConfigPack").read_bytes()
        index = Path(f"{tmp_path}/{key}.ConfigPackIndex").read_bytes()
        assert hashlib.sha256(pack).hexdigest() == inp["pack_sha256"]
        assert hashlib.sha256(index).hexdigest() == inp["index_sha256"]
        s2, unit = stack_fractional(read_configpack(tmp_path / key))
        np.testing.assert_array_equal(s2, s)
        np.testing.assert_array_equal(unit, z[f"in_{key}_unit"])


def test_round_trip_and_layout(tmp_path):
    cfgs = [_cfg(10, 3, 1), _cfg(4, 2, 2), _cfg(1, 1, 3)]
    write_configpack(tmp_path / "p", cfgs)
    idx = np.fromfile(f"{tmp_path}/p.ConfigPackIndex", dtype="<i8")
    sizes = [14 + 8 * d * d + n * (8 * d + 4) for n, d in ((10, 3), (4, 2), (1, 1))]
    assert idx.tolist() == [3, 0, sizes[0], sizes[0] + sizes[1]]
    assert Path(f"{tmp_path}/p.ConfigPack").stat().st_size == sum(sizes)
    got = read_configpack(tmp_path / "p", [2, 0, 0])
    assert [g.relative.shape for g in got] == [(1, 1), (10, 3), (10, 3)]
    np.testing.assert_array_equal(got[1].relative, cfgs[0].relative)
    assert got[1].names[0] == b"a\x00\x00\x00"
    assert read_configpack(tmp_path / "p", []) == []


def test_reader_errors(tmp_path):
    write_configpack(tmp_path / "p", [_cfg(2, 2)] * 3)
    for bad in ([3], [-1]):
        with pytest.raises(ValueError):
            read_configpack(tmp_path / "p", bad)
    with pytest.raises(FileNotFoundError, match="ConfigPackIndex"):
        read_configpack(tmp_path / "missing")
    write_configpack(tmp_path / "t", [_cfg(10, 3), _cfg(10, 3)])
    pack = Path(f"{tmp_path}/t.ConfigPack")
    data = pack.read_bytes()
    for cut in (1, 5, 40, 200):
        pack.write_bytes(data[:len(data) - cut])
        with pytest.raises(ValueError):
            read_configpack(tmp_path / "t")
    for keep in (0, 1, 9):
        pack.write_bytes(data[:keep])
        with pytest.raises(ValueError):
            read_configpack(tmp_path / "t")
    pack.write_bytes(data)
    idx = Path(f"{tmp_path}/t.ConfigPackIndex")
    raw = idx.read_bytes()
    idx.write_bytes(raw[:-8])
    with pytest.raises(ValueError):
        read_configpack(tmp_path / "t")
    idx.write_bytes(b"")
    with pytest.raises(ValueError):
        read_configpack(tmp_path / "t")
    bad_dim = bytearray(data)
    bad_dim[0:2] = (7).to_bytes(2, "little")
    pack.write_bytes(bytes(bad_dim))
    idx.write_bytes(raw)
    with pytest.raises(ValueError, match="dimension"):
        read_configpack(tmp_path / "t")


def test_writer_errors(tmp_path):
    with pytest.raises(ValueError):
        write_configpack(tmp_path / "e", [])
    with pytest.raises(FileNotFoundError):
        write_configpack(tmp_path / "no" / "p", [_cfg(2, 2)])
    c = _cfg(3, 2)
    with pytest.raises(TypeError):
        write_configpack(tmp_path / "x", [PackedConfig(c.basis, c.relative.astype(np.float32), 1.0, c.names)])
    with pytest.raises(ValueError):
        write_configpack(tmp_path / "x", [PackedConfig(np.eye(3), c.relative, 1.0, c.names)])
    with pytest.raises(ValueError):
        write_configpack(tmp_path / "x", [PackedConfig(c.basis, c.relative, 1.0, c.names[:2])])
    with pytest.raises(ValueError):
        write_configpack(tmp_path / "x", [PackedConfig(c.basis, c.relative, 1.0, (b"ab",) * 3)])
    with pytest.raises(ValueError):
        write_configpack(tmp_path / "x", [PackedConfig(np.eye(5), np.zeros((2, 5)), 1.0, (b"abcd",) * 2)])


def test_stack_fractional_rules():
    a, b = _cfg(4, 2, 1, scale=2.0), _cfg(4, 2, 2, scale=3.0)
    s, unit = stack_fractional([a, b])
    assert s.shape == (2, 4, 2)
    np.testing.assert_allclose(unit, np.eye(2), rtol=0, atol=1e-15)
    with pytest.raises(ValueError):
        stack_fractional([])
    with pytest.raises(ValueError, match="mixed"):
        stack_fractional([a, _cfg(5, 2)])
    with pytest.raises(ValueError, match="bases differ"):
        stack_fractional([a, PackedConfig(np.array([[1.0, 0.5], [0.0, 1.0]]), a.relative, 1.0, a.names)])
    with pytest.raises(ValueError, match="determinant"):
        stack_fractional([PackedConfig(np.diag([-1.0, 1.0]), a.relative, 1.0, a.names)])
    with pytest.raises(TypeError):
        stack_fractional([PackedConfig(a.basis, a.relative.astype(np.float32), 1.0, a.names)])


# ------------------------------------------------------------------ tables


def test_tables_match_reference_text(tmp_path, io_golden):
    z, meta = io_golden
    for t in meta["tables"]:
        cols = [z[f"table{t['case']}_col{j}"] for j in range(t["n_cols"])]
        path = tmp_path / f"t{t['case']}.txt"
        write_function_table(path, cols)
        assert path.read_text() == t["text"]


def test_tables_reject_bad_input(tmp_path):
    out = tmp_path / "f.txt"
    for cols in ([np.zeros(2), np.zeros(3)], [np.zeros(2)] * 5, [], [np.array([np.inf])],
                 [np.array([-np.inf])], [np.zeros((2, 2))]):  # fmt: skip
        with pytest.raises(ValueError):
            write_function_table(out, cols)


# ------------------------------------------------------------------ S(k) host parts


def test_isotropic_kset_bit_exact(io_golden):
    z, meta = io_golden
    for c in meta["iso"]:
        n, q = _isotropic_kset(z[f"iso_{c['name']}_basis"], c["k_dir"], c["k_max"])
        np.testing.assert_array_equal(n, z[f"iso_{c['name']}_n"])
        np.testing.assert_array_equal(q, z[f"iso_{c['name']}_ksq"])


def test_oracle_isotropic_kset_pinned(io_golden):
    z, meta = io_golden
    for c in meta["iso"]:
        if c["k_max"] > 100.0:
            continue   # brute force only on the small cases
        n, q = oracle.isotropic_kset(z[f"iso_{c['name']}_basis"], c["k_dir"], c["k_max"])
        np.testing.assert_array_equal(n, z[f"iso_{c['name']}_n"])
        np.testing.assert_array_equal(q, z[f"iso_{c['name']}_ksq"])


def test_bin_moments_bit_exact(io_golden):
    z, meta = io_golden
    for c in meta["bins"]:
        b = c["case"]
        args = (z[f"bins{b}_in_k"], z[f"bins{b}_in_s"], z[f"bins{b}_in_s2"], c["n_cfg"], c["width"])
        for impl in (_bin_moments, oracle.bin_moments):
            out = impl(*args)
            for j in range(4):
                np.testing.assert_array_equal(out[j], z[f"bins{b}_out{j}"])
    out = _bin_moments(np.full(3, 0.1), np.ones(3), np.full(3, 0.5), 1, 0.01)
    want = meta["bins_negative_variance"]
    assert float.hex(float(out[0][0])) == want[0] and out[2][0] == 0.0 and np.isnan(out[3][0])


def test_g2_normalisation():
    edges = np.array([1.0, 2.0])
    got = g2_from_histogram(np.array([30.0]), edges, 10, 2, 20.0, 2)
    assert math.isclose(got[0], 30.0 / (math.pi * 3.0 * 0.5 * 0.5 * 10 * 2), rel_tol=1e-14)
    with pytest.raises(ValueError):
        g2_from_histogram(np.zeros(3), np.array([0.0, 1.0, 2.0]), 5, 1, 5.0, 2)
    for bad in (np.array([0.0]), np.array([1.0, 1.0]), np.array([-1.0, 1.0]), np.array([0.0, np.nan])):
        with pytest.raises(ValueError):
            g2_from_histogram(np.zeros(max(bad.size - 1, 1)), bad, 5, 1, 5.0, 2)


def test_pair_oracle_pinned(io_golden):
    z, meta = io_golden
    for c in meta["pairs"]:
        nn, dist = oracle.min_image_distances(z[f"pairs_{c['name']}_s"], z[f"pairs_{c['name']}_basis"])
        np.testing.assert_allclose(nn, z[f"pairs_{c['name']}_nn"], rtol=1e-14, atol=0)
        np.testing.assert_allclose(dist, z[f"pairs_{c['name']}_dist"], rtol=1e-14, atol=0)
    for c in meta["sk"]:
        out = oracle.structure_factor_direct(z[f"sk_{c['name']}_s"], z[f"sk_{c['name']}_n"])
        np.testing.assert_allclose(out, z[f"sk_{c['name']}_out"], rtol=1e-12, atol=1e-13)


# ------------------------------------------------------------------ driver host logic


def _argv(tmp_path, *extra, dim=2):
    return ["--dim", str(dim), "--ka", "1.5", "--phi", "0.05", "--load", str(tmp_path / "in"),
            "--save", str(tmp_path / "out"), *extra]  # fmt: skip


@pytest.mark.parametrize("extra", [["--tol", "0"], ["--grow", "2.0"], ["--k1a", "10"],
                                   ["--record-every", "3"], ["--max-steps", "0"],
                                   ["--batch-size", "0"], ["--hp-bins", "0"],
                                   ["--stop-tol", "-1"], ["--chunk-size", "0"]])  # fmt: skip
def test_driver_rejects_bad_arguments(tmp_path, extra):
    with pytest.raises(ValueError, match="--"):
        cli.run(cli.build_parser().parse_args(_argv(tmp_path, *extra)))


def test_driver_refuses_cpu_device(tmp_path):
    with pytest.raises(RuntimeError, match="--device cpu"):
        cli.select_device("cpu")


def test_driver_help_and_guard(tmp_path):
    env_path = str(ROOT / "xla-cco_b200")
    proc = subprocess.run([sys.executable, "-m", "xla_cco.cli.relax", "--help"], capture_output=True,
                          text=True, cwd=env_path, check=False)  # fmt: skip
    assert proc.returncode == 0
    assert "adaptive bins" in proc.stdout and "9.99999968e-21" in proc.stdout


def test_success_mask_is_strict():
    tol = 1e-20
    assert cli.success_mask(np.array([tol, np.nextafter(tol, 0.0), 2 * tol]), tol).tolist() == [
        False, True, False]


def test_hp_g2_tables():
    edges = np.array([0.0, 1.0, 3.0])
    counts = np.array([1, 3])
    h = np.stack(cli.table_columns(edges, cli.hp_density(counts, edges), counts), axis=1)
    np.testing.assert_allclose(h[:, 0], [0.5, 2.0])
    np.testing.assert_allclose(h[:, 2], [0.5, 1.0])
    np.testing.assert_allclose(h[:, 1], [0.25, 0.375])
    np.testing.assert_allclose(h[:, 3], [0.25, 0.375 / np.sqrt(3)])
    assert math.isclose((h[:, 1] * 2.0 * h[:, 2]).sum(), 1.0)
    g = np.stack(cli.table_columns(edges, np.array([2.0, 4.0]), np.array([4, 0])), axis=1)
    np.testing.assert_allclose(g[:, 3], [1.0, 0.0])
    np.testing.assert_allclose(g[:, 1], [2.0, 4.0])
