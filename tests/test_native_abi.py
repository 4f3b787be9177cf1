"""The C-ABI library loads and exports every symbol include/cco.h declares.

Runs without a GPU: only argument validation and device queries are called
(no compute). The Python binding's signature table must match the header.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from xla_cco import _native

HEADER = Path(__file__).resolve().parents[1] / "include" / "cco.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cco_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("cco_problem_create", "cco_energy_grad", "cco_relax_descent", "cco_relax_lbfgs",
                 "cco_device_count", "cco_last_error"):  # fmt: skip
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    for name in declared_functions():
        assert hasattr(lib, name), f"libcco.so does not export {name}"
        assert name in _native.SIGNATURES, f"binding lacks {name}"


def test_struct_layouts_match_header():
    assert ctypes.sizeof(_native.DescentSettingsC) == 9 * 8
    assert ctypes.sizeof(_native.LBFGSSettingsC) == 8 + 8 + 8 * 8 + 7 * 8
    assert ctypes.sizeof(_native.RelaxOutC) == 17 * 8


def test_abi_version_and_errors():
    lib = _native.load()
    assert lib.cco_abi_version() == 1
    assert lib.cco_error_string(_native.CCO_ERR_ROUNDS).decode().startswith("relax did not finish")
    assert lib.cco_energy_grad(None, None, 1, None, None, None, None, None) == _native.CCO_ERR_ARG
    assert b"null" in lib.cco_last_error()


def test_problem_create_validates_before_touching_a_device():
    lib = _native.load()
    out = ctypes.c_void_p()
    n = (ctypes.c_int32 * 2)(1, 0)
    w = (ctypes.c_double * 1)(1.0)
    assert lib.cco_problem_create(0, 4, 10, 1, n, w, 10.0, ctypes.byref(out)) == _native.CCO_ERR_ARG
    assert lib.cco_problem_create(0, 2, 10, 0, n, w, 10.0, ctypes.byref(out)) == _native.CCO_ERR_ARG
    assert b"empty" in lib.cco_last_error()
    assert lib.cco_problem_create(0, 2, 10, 1, n, w, -1.0, ctypes.byref(out)) == _native.CCO_ERR_ARG


def test_no_device_is_reported_not_hidden():
    if _native.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError, match="needs a CUDA device"):
        _native.require_gpu()


def test_server_without_device_is_refused():
    if _native.device_count() > 0:
        pytest.skip("a GPU is visible")
    from xla_cco.minimize import _lbfgs_c
    from xla_cco.minimize.lbfgs import LBFGSSettings

    lib = _native.load()
    cset = _lbfgs_c(LBFGSSettings())
    cfg = _native.ServerConfigC(0, 0, 0, 0)
    h = ctypes.c_void_p()
    code = lib.cco_server_create(0, ctypes.byref(cset), ctypes.byref(cfg), ctypes.byref(h))
    assert code == _native.CCO_ERR_NODEVICE and not h.value
    assert lib.cco_server_destroy(None) == _native.CCO_OK


def test_serving_structs_match_header():
    assert ctypes.sizeof(_native.ServerConfigC) == 3 * 8
    assert ctypes.sizeof(_native.RequestResultC) == 12 * 8
    assert ctypes.sizeof(_native.ServerStatsC) == 13 * 8


PAIRS = [
    ("cco_descent_settings", "DescentSettingsC"), ("cco_lbfgs_settings", "LBFGSSettingsC"),
    ("cco_relax_out", "RelaxOutC"), ("cco_flow_settings", "FlowSettingsC"),
    ("cco_flow_out", "FlowOutC"), ("cco_md_settings", "MdSettingsC"), ("cco_md_out", "MdOutC"),
    ("cco_md_segment_settings", "MdSegmentSettingsC"), ("cco_md_waves", "MdWavesC"),
    ("cco_md_state", "MdStateC"), ("cco_server_config", "ServerConfigC"),
    ("cco_request_result", "RequestResultC"), ("cco_server_stats", "ServerStatsC"),
]  # fmt: skip


def test_every_ctypes_struct_matches_the_c_layout(tmp_path):
    """Compile a probe against include/cco.h with the host C compiler and compare
    every field offset and struct size with the ctypes mirrors."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "cco.h"', "int main(void) {"]
    for cname, pyname in PAIRS:
        st = getattr(_native, pyname)
        lines.append(f'  printf("{pyname} size %zu\\n", sizeof({cname}));')
        for fname, _ in st._fields_:
            lines.append(f'  printf("{pyname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run([cc, "-std=c11", "-I", str(HEADER.parent), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = 0
    for line in filter(None, out):
        pyname, field, value = line.split()
        st = getattr(_native, pyname)
        got = ctypes.sizeof(st) if field == "size" else getattr(st, field).offset
        assert got == int(value), f"{pyname}.{field}: ctypes {got} != C {value}"
        seen += 1
    assert seen == sum(1 + len(getattr(_native, p)._fields_) for _, p in PAIRS)
