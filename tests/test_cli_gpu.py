"""The nse2d executable on a B200 against the reference's own verification runs.

Every case of the reference's test suite (its tests/run_tests.py command lines, kept with the
reference's diagnostics rows in tests/golden/reference_cases.json) runs through the CLI,
stopped half an output interval after the last kept row; every kept row must match the
reference's printed row to its 9 digits (relative 2e-7, with the noise rules of
test_oracle_golden). These cover the
eigenmode decay in time and space, the manufactured solution, the laminar Poiseuille flow,
the inviscid free-slip conservation runs and the forced channel's early rows.

A resumed run (--init load --resume from a snapshot) must continue the original run: its
rows after the restart equal the uninterrupted run's to 1e-12 relative.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG
from test_oracle_golden import case_args, compare_rows

pytestmark = pytest.mark.gpu

CLI = os.path.join(PKG, "nse2d")


def run_cli(args, outdir, timeout=600):
    p = subprocess.run([CLI] + list(args) + ["--outdir", outdir], capture_output=True, text=True, timeout=timeout)
    assert p.returncode == 0, p.stderr[-2000:]
    a = np.genfromtxt(os.path.join(outdir, "diagnostics.csv"), delimiter=",", names=True)
    return np.atleast_1d(a)


def test_cli_built(cuda):
    assert os.path.isfile(CLI), "build the executable with make -C nse2d-channel-gpu_b200"


def cases():
    import json
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_cases.json")))
    return sorted(g["cases"])


@pytest.mark.parametrize("case", cases())
def test_reference_case(golden, cuda, tmp_path, case):
    c = golden["cases"][case]
    rows = c["rows"]
    a = case_args(c)
    i = a.index("--tend")
    t_last = rows[-1][1]
    if c["n_rows_total"] > len(rows):
        # end half an output interval after the last kept row: the loop test t < t_end - dt/2
        # must not stop the run before the step that lands on that row
        dsave = float(a[a.index("--diag_save") + 1])
        a[i + 1] = repr(min(float(a[i + 1]), t_last + 0.5 * dsave))
    mine = run_cli(a, str(tmp_path / case))
    assert len(mine) >= len(rows), (len(mine), len(rows))
    compare_rows(case, mine, rows, c["header"], len(rows))


def test_resume_continues_the_run(cuda, tmp_path):
    base = ["--Nx", "128", "--Ny", "65", "--Ub", "1", "--Reb", "2000", "--init", "mix", "--amp", "0.05",
            "--F0", "0.05", "--nforce", "4", "--drag", "0.001", "--stretch", "tanh", "--beta", "2",
            "--diag_save", "0.05", "--snap_fields", "omega_psi"]
    full = run_cli(base + ["--tend", "0.3", "--snap_save", "0.15"], str(tmp_path / "full"))
    snap = tmp_path / "full" / "snaps" / "snap_t0.150000.bin"
    assert snap.is_file()
    res = run_cli(base + ["--tend", "0.3", "--snap_save", "0", "--init", "load", "--resume", "--load_path",
                          str(snap)], str(tmp_path / "resumed"))
    later = full[full["t"] > 0.15 + 1e-9]
    assert len(res) == len(later) and len(res) >= 2
    for name in ("t", "umax", "vmax", "K", "Omega", "epsilon", "tauw_bot", "tauw_top"):
        np.testing.assert_allclose(res[name], later[name], rtol=1e-12, atol=1e-14 * np.max(np.abs(later[name])))
