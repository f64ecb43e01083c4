"""The oracle against the reference's own test data (CPU only).

Golden vectors: tests/golden/reference_cases.json, extracted by tests/golden/make_golden.py
from the reference's tests/reference/output/<case>/diagnostics.csv (A100, CUDA 13.2). The
t = 0 row of every case is a deterministic function of the initial condition, the grid, the
Poisson solve, the Thom closure and every diagnostic reduction; the early rows add the time
stepping. The oracle must reproduce them to the 9 printed digits (relative 2e-7), except for
quantities that are round-off noise in the reference itself (|tau_w| < 1e-13, where u_tau,
C_f and Re_tau are square roots of noise) and columns that are small differences of O(1)
sums (absolute floor 1e-9 times the column scale).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ORACLE

NOISE_IF_TAU_SMALL = ("utau_avg", "Cf", "Re_tau")


def run_oracle(args, outdir, extra=()):
    exe = os.path.join(ORACLE, "_build", "nse2d_oracle")
    subprocess.run([exe] + list(args) + ["--outdir", outdir] + list(extra), check=True, capture_output=True)
    a = np.genfromtxt(os.path.join(outdir, "diagnostics.csv"), delimiter=",", names=True)
    return np.atleast_1d(a)


def compare_rows(case, mine, ref_rows, header, nrows):
    scale = {}
    for ci, name in enumerate(header):
        col = np.array([r[ci] for r in ref_rows], dtype=float)
        col = col[np.isfinite(col)]
        scale[name] = max(1.0, float(np.max(np.abs(col)))) if col.size else 1.0
    bad = []
    for k in range(nrows):
        tau = max(abs(ref_rows[k][header.index("tauw_bot")]), abs(ref_rows[k][header.index("tauw_top")]))
        for ci, name in enumerate(header):
            r = ref_rows[k][ci]
            x = float(mine[name][k])
            if np.isnan(r):
                if not np.isnan(x):
                    bad.append((k, name, x, r))
                continue
            if name in NOISE_IF_TAU_SMALL and tau < 1e-13:
                continue
            tol = 2e-7 * abs(r) + 1e-9 * scale[name]
            if abs(x - r) > tol:
                bad.append((k, name, x, r))
    assert not bad, f"{case}: {bad[:6]}"


def case_args(c):
    a = list(c["args"])
    if c["exe"] == "nse2d_freeslip":
        a.append("--free_slip")
    return a


def test_t0_rows_all_cases(oracle, golden, tmp_path):
    """The deterministic t = 0 row of all 21 reference cases."""
    for case, c in golden["cases"].items():
        out = str(tmp_path / case)
        mine = run_oracle(case_args(c), out, ["--max_steps", "0"])
        compare_rows(case, mine, c["rows"], c["header"], 1)


FAST_EARLY = ["channel", "cons_dt0.004", "cons_dt0.002", "eig_time_dt0.64", "eig_time_dt0.16",
              "eig_space_Ny33_b0", "eig_space_Ny33_b2"]


@pytest.mark.parametrize("case", FAST_EARLY)
def test_early_rows(oracle, golden, tmp_path, case):
    """The first output rows after t = 0 (time stepping, adaptive dt and output scheduling)."""
    c = golden["cases"][case]
    nrows = min(3, len(c["rows"]))
    t_stop = c["rows"][nrows - 1][1]
    a = case_args(c)
    i = a.index("--tend")
    a[i + 1] = repr(min(float(a[i + 1]), t_stop + 1e-9))
    mine = run_oracle(a, str(tmp_path / case))
    n = min(nrows, len(mine))
    assert n >= 2
    compare_rows(case, mine, c["rows"], c["header"], n)
