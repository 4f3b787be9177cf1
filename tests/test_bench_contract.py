"""bench.py's reference arm (the CPU arm the driver runs beside the device
arm): one JSON line with the contract's keys, measured by relaxing one lane
of the headline batch to completion on the host, and never touching the
product library."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    # run the arm in a wrapper that reports, at the very end (after a garbage
    # collection, when finalizers have run), which shared objects the process mapped
    wrapper = (
        "import gc, runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "gc.collect()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('MAPPED_LIBCCO' if 'libcco' in maps else 'NO_LIBCCO')\n"
    )
    proc = subprocess.run([sys.executable, "-c", wrapper],
                          cwd=ROOT, capture_output=True, text=True, timeout=600, check=False)  # fmt: skip
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):  # fmt: skip
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0.0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["config"]["workload"].startswith("lbfgs_relax_d2_n1000_chi0.4_m802")
    # a measured relaxation, not an extrapolation: the one timed lane reached 1e-20
    assert "1/1 relaxed" in d["cpu_baseline"]["sample"]
    assert proc.stdout.strip().splitlines()[-1] == "NO_LIBCCO", "the reference arm mapped libcco.so"
    assert "xla_cco" not in d["cpu_baseline"]["sample"]
