"""The nse2d executable on a B200 against the reference's own verification runs.

Every case of the reference's test suite (its tests/run_tests.py command lines, kept with the
reference's diagnostics rows in tests/golden/reference_cases.json) runs through the CLI,
stopped half an output interval after the last kept row; every kept row must match the
reference's printed row to its 9 digits (relative 2e-7, with the noise rules of
test_oracle_golden). These cover the
eigenmode decay in time and space, the manufactured solution, the laminar Poiseuille flow,
the inviscid free-slip conservation runs and the forced channel's early rows.

A resumed run (--init load --resume from a snapshot, HDF5 or bin) must continue the original run:
its rows after the restart equal the uninterrupted run's to 1e-12 relative. The HDF5 snapshots the
executable writes (src/io.cu:203-259 layout) are opened with the independent test reader
(tests/h5read.py); --init load --load_use_psi rebuilds omega from psi as src/init.cu:243-264 does
(uniform differences, first-order Thom walls: checked against numpy to 1e-14); --stretch table
takes y from the HDF5 file of --ytable (src/grid.cu:46-78: metrics checked against numpy's
restatement, exactly).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG
from h5read import H5File
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


@pytest.mark.parametrize("fmt", ["h5", "bin"])
def test_resume_continues_the_run(cuda, tmp_path, fmt):
    base = ["--Nx", "128", "--Ny", "65", "--Ub", "1", "--Reb", "2000", "--init", "mix", "--amp", "0.05",
            "--F0", "0.05", "--nforce", "4", "--drag", "0.001", "--stretch", "tanh", "--beta", "2",
            "--diag_save", "0.05", "--snap_fields", "omega_psi", "--snap_fmt", fmt]
    full = run_cli(base + ["--tend", "0.3", "--snap_save", "0.15"], str(tmp_path / "full"))
    snap = tmp_path / "full" / "snaps" / f"snap_t0.150000.{fmt}"
    assert snap.is_file()
    other = "bin" if fmt == "h5" else "h5"
    assert not (tmp_path / "full" / "snaps" / f"snap_t0.150000.{other}").exists()
    res = run_cli(base + ["--tend", "0.3", "--snap_save", "0", "--init", "load", "--resume", "--load_path",
                          str(snap)], str(tmp_path / "resumed"))
    later = full[full["t"] > 0.15 + 1e-9]
    assert len(res) == len(later) and len(res) >= 2
    for name in ("t", "umax", "vmax", "K", "Omega", "epsilon", "tauw_bot", "tauw_top"):
        np.testing.assert_allclose(res[name], later[name], rtol=1e-12, atol=1e-14 * np.max(np.abs(later[name])))


def test_hdf5_snapshots_of_a_run(cuda, tmp_path):
    """Every snapshot of a run opens in the independent reader with the reference's layout: omega,
    psi, u, v [Ny, Nx], y [1, Ny] with beta and stretch_code, and the root attributes."""
    a = ["--Nx", "64", "--Ny", "33", "--Ub", "1", "--Reb", "1000", "--init", "mix", "--amp", "0.05",
         "--stretch", "tanh", "--beta", "2", "--Lx", "6.283185307179586", "--tend", "0.1", "--snap_save", "0.05",
         "--diag_save", "0.05"]
    d = run_cli(a, str(tmp_path))
    files = sorted((tmp_path / "snaps").glob("snap_t*.h5"))
    assert [f.name for f in files] == ["snap_t0.000000.h5", "snap_t0.050000.h5", "snap_t0.100000.h5"]
    for f, t in zip(files, (0.0, 0.05, 0.1)):
        h = H5File(str(f))
        assert sorted(h.links) == ["omega", "psi", "u", "v", "y"]
        assert abs(h.attrs["t"] - t) < 1e-12 and (h.attrs["Nx"], h.attrs["Ny"]) == (64, 33)
        assert h.attrs["nu"] == 2.0 / 1000 and h.attrs["beta"] == 2.0 and h.attrs["stretch_code"] == 1.0
        w, psi = h.read("omega"), h.read("psi")
        assert w.shape == (33, 64) and np.all(np.isfinite(w)) and np.all(np.isfinite(psi))
        y = h.read("y").ravel()
        assert np.allclose(y, np.tanh(2.0 * np.linspace(-1, 1, 33)) / np.tanh(2.0), rtol=0, atol=1e-15)
        assert abs(psi[0].max()) < 1e-14 and np.allclose(psi[-1], 2.0)        # the Dirichlet walls
    assert len(d) == 3


def test_load_use_psi_rebuilds_omega(nse, cuda, tmp_path):
    """--init load --load_use_psi: omega from psi by uniform second differences and first-order
    Thom walls with the current Ub (src/init.cu:243-264); the run's t = 0 snapshot holds that
    omega on the interior rows (the initial solve and Thom closure change only the wall rows)."""
    Nx, Ny, Lx, h = 64, 33, 2 * np.pi, 1.0
    rng = np.random.default_rng(12)
    y = np.linspace(-h, h, Ny)
    x = np.arange(Nx) * Lx / Nx
    psi = (1.5 * (y + h) - 0.5 * (y + h) ** 3 / 4)[:, None] + 1e-2 * np.outer(np.sin(np.pi * (y + h) / 2) ** 2,
                                                                             np.cos(2 * x) + rng.random(Nx))
    src = tmp_path / "psi_only.h5"
    nse.write_snapshot(src, {"psi": psi}, t=0.0, Lx=Lx, h=h, nu=1e-3)
    run_cli(["--Nx", str(Nx), "--Ny", str(Ny), "--Lx", repr(Lx), "--Ub", "1", "--Reb", "1000", "--init", "load",
             "--load_use_psi", "--load_path", str(src), "--tend", "0.001", "--snap_save", "1", "--diag_save", "1",
             "--snap_fields", "omega"], str(tmp_path / "run"))
    w = H5File(str(tmp_path / "run" / "snaps" / "snap_t0.000000.h5")).read("omega")
    dx, dy = Lx / Nx, 2 * h / (Ny - 1)
    exp = -((np.roll(psi, -1, 1) - 2 * psi + np.roll(psi, 1, 1)) / dx ** 2)[1:-1] \
        - ((psi[2:] - 2 * psi[1:-1] + psi[:-2]) / dy ** 2)
    assert np.max(np.abs(w[1:-1] - exp)) <= 1e-14 * np.max(np.abs(exp))


def test_stretch_table(nse, cuda, tmp_path):
    """--stretch table: y from the HDF5 dataset /y ([1, Ny] or [Ny, 1]), a_node = 1 / y_eta by
    one-sided and central differences in eta (src/grid.cu:46-78), then the common edges and
    trapezoid weights (src/grid.cu:80-93)."""
    Nx, Ny = 64, 41
    y = np.sinh(1.7 * np.linspace(-1, 1, Ny)) / np.sinh(1.7)
    tab = tmp_path / "ytab.h5"
    nse.write_snapshot(tab, {"omega": np.zeros((Ny, Nx))}, t=0.0, Lx=2 * np.pi, h=1.0, nu=0.0, beta=1.0, y=y)
    g = nse.Solver(Nx=Nx, Ny=Ny, Lx=2 * np.pi, stretch="table", y_table=y, Ub=1.0, Reb=1000.0)
    deta = 2.0 / (Ny - 1)
    yeta = np.empty(Ny)
    yeta[0] = (y[1] - y[0]) / deta
    yeta[-1] = (y[-1] - y[-2]) / deta
    yeta[1:-1] = (y[2:] - y[:-2]) / (2.0 * deta)
    a = 1.0 / yeta
    de = np.diff(y)
    wn = np.empty(Ny)
    wn[0], wn[-1] = 0.5 * de[0], 0.5 * de[-1]
    wn[1:-1] = 0.5 * (de[:-1] + de[1:])
    for k, exp in enumerate((y, a, 0.5 * (a[:-1] + a[1:]), de, wn)):
        assert np.array_equal(g.metric(k), exp), k
    g.close()
    # the profiles file takes y from the grid only when beta > 0 (src/io.cu:276), as the reference does
    d = run_cli(["--Nx", str(Nx), "--Ny", str(Ny), "--Lx", repr(2 * np.pi), "--Ub", "1", "--Reb", "1000",
                 "--init", "mix", "--amp", "0.05", "--stretch", "table", "--beta", "1", "--ytable", str(tab),
                 "--tend", "0.05", "--diag_save", "0.05", "--snap_save", "0"], str(tmp_path / "run"))
    assert len(d) == 2 and np.all(np.isfinite(d["K"]))
    prof = np.genfromtxt(tmp_path / "run" / "profiles_timeavg.csv", delimiter=",", names=True)
    assert np.allclose(prof["y"], y, rtol=1e-8, atol=1e-9)           # the CSV prints 9 digits
    p = subprocess.run([CLI, "--Nx", "64", "--Ny", "41", "--stretch", "table", "--outdir", str(tmp_path / "x")],
                       capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "--ytable required" in p.stderr
