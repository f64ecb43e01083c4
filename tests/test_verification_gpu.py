"""The reference's own verification suite, run to full length on this build (B200).

The reference ships six tests (tests/run_tests.py:213-330 of the reference) over 21 runs of its
executable (tests/run_tests.py:72-111); their command lines are kept in
tests/golden/reference_cases.json. Here every run goes through this project's nse2d executable to
its full --tend, its HDF5 snapshots are read with the independent test reader (tests/h5read.py),
and each test's checks are evaluated as the reference's runner evaluates them:
  eigenmode_space  observed order in space of the viscous shear eigenmode, last pair in [1.7, 2.3],
                   uniform and tanh beta=2 grids (run_tests.py:213-231);
  eigenmode_time   mean of the first two observed orders in time in [2.5, 3.5] (:233-246);
  poiseuille       wall stresses, dp/dx, dissipation and energy within 5e-3 of the exact laminar
                   values, and the energy balance -Ub dp/dx = epsilon (:248-262);
  mms              observed order of the manufactured solution in [1.7, 2.3] (:264-283);
  conservation     free-slip inviscid run: relative drift of the discrete energy and enstrophy
                   below 1e-6 over t in [0, 2], smaller at the smaller dt (:285-305);
  channel          the scheme-consistent enstrophy identity below 1e-6 of mean eta_h at every one
                   of the 400 output times, finite diagnostics to the end (:307-330).
Then every metric is compared with the reference's published values (tests/reference/
reference.json) at the runner's relative tolerances REF_TOL (:342-345), skipping the same keys
(REF_SKIP) and values below the round-off floor 1e-13. The observed orders and drifts are printed.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG
from h5read import H5File
from test_oracle_golden import case_args

pytestmark = pytest.mark.gpu

H = 1.0
LX = 4.0 * math.pi                      # the runner's default --Lx (the solver default)


@pytest.fixture(scope="module")
def runs(golden, tmp_path_factory, cuda):
    """Run all 21 cases through the executable, to full length."""
    out = tmp_path_factory.mktemp("verification")
    for case, c in sorted(golden["cases"].items()):
        exe = os.path.join(PKG, "nse2d_freeslip" if c["exe"] == "nse2d_freeslip" else "nse2d")
        d = out / case
        p = subprocess.run([exe] + list(c["args"]) + ["--outdir", str(d)], capture_output=True, text=True,
                           timeout=900)
        assert p.returncode == 0, (case, p.stderr[-2000:])
    return out


class Snap:
    pass


def snaps(d):
    """All HDF5 snapshots of a run, by time: omega, psi [Ny, Nx], y, x."""
    out = []
    for fn in sorted((d / "snaps").glob("snap_t*.h5")):
        f = H5File(str(fn))
        s = Snap()
        s.t, s.Nx, s.Ny = float(f.attrs["t"]), int(f.attrs["Nx"]), int(f.attrs["Ny"])
        s.Lx, s.h = float(f.attrs["Lx"]), float(f.attrs["h"])
        s.omega = f.read("omega").astype(float)
        s.psi = f.read("psi").astype(float) if "psi" in f.links else None
        s.y = f.read("y").ravel() if "y" in f.links else np.linspace(-s.h, s.h, s.Ny)
        s.x = np.arange(s.Nx) * (s.Lx / s.Nx)
        out.append(s)
    assert out, f"no HDF5 snapshots in {d}"
    return sorted(out, key=lambda s: s.t)


def last_snap(d, t):
    s = snaps(d)[-1]
    assert abs(s.t - t) <= 1e-6 * max(1.0, abs(t)), (d, s.t, t)
    return s


def l2_norm(err, y):
    """Trapezoid weights in y, mean in x (run_tests.py:185-201)."""
    w = np.zeros_like(y)
    w[1:] += 0.5 * np.diff(y)
    w[:-1] += 0.5 * np.diff(y)
    return math.sqrt(float(np.sum(w[:, None] * err ** 2) / (err.shape[1] * np.sum(w)))), float(np.max(np.abs(err)))


def observed_order(e):
    return [math.log(e[k] / e[k + 1]) / math.log(2.0) for k in range(len(e) - 1)]


def diag(d):
    return np.atleast_1d(np.genfromtxt(d / "diagnostics.csv", delimiter=",", names=True))


# ---- the six tests: (metrics, [(description, passed)]) ----
def eigenmode_space(out):
    m, checks, nu, T = {}, [], 1e-2, 2.0
    mu = math.pi / H
    for b in (0, 2):
        e2 = []
        for ny in (33, 65, 129):
            s = last_snap(out / f"eig_space_Ny{ny}_b{b}", T)
            decay = math.exp(-nu * mu * mu * s.t)
            prof = -mu * np.cos(mu * (s.y + H)) * decay
            l2, li = l2_norm(s.omega - prof[:, None], s.y)
            wall = 0.5 * (s.omega[0].mean() + s.omega[-1].mean())
            m[f"E2_Ny{ny}_b{b}"], m[f"Einf_Ny{ny}_b{b}"] = l2, li
            m[f"wall_rel_Ny{ny}_b{b}"] = abs(wall + mu * decay) / abs(mu * decay)
            e2.append(l2)
        p = observed_order(e2)
        checks.append((f"beta={b}: orders in space {['%.3f' % q for q in p]}", 1.7 <= p[-1] <= 2.3))
    return m, checks


def eigenmode_time(out):
    m, checks, T = {}, [], 10.24
    ref = last_snap(out / "eig_time_ref", T)
    e2 = []
    for dt in (0.64, 0.32, 0.16, 0.08):
        s = last_snap(out / f"eig_time_dt{dt:g}", T)
        m[f"E2_dt{dt:g}"] = l2_norm(s.omega - ref.omega, s.y)[0]
        e2.append(m[f"E2_dt{dt:g}"])
    p = observed_order(e2)
    checks.append((f"orders in time {['%.3f' % q for q in p]}", 2.5 <= 0.5 * (p[0] + p[1]) <= 3.5))
    return m, checks


def poiseuille(out):
    m, checks = {}, []
    r = diag(out / "poiseuille")[-1]
    Ub, nu = 1.0, 2.0 * H * 1.0 / 500.0
    exact = {"tauw_bot": 3 * nu * Ub / H, "tauw_top": -3 * nu * Ub / H, "dpdx": -3 * nu * Ub / H ** 2,
             "epsilon": 3 * nu * Ub ** 2 / H ** 2, "K": 0.6 * Ub ** 2}
    for k, ex in exact.items():
        m[f"dev_{k}"] = abs(float(r[k]) - ex) / abs(ex)
        checks.append((f"{k} = {float(r[k]):+.8e} (exact {ex:+.8e})", m[f"dev_{k}"] < 5e-3))
    m["energy_balance"] = abs(-Ub * float(r["dpdx"]) - float(r["epsilon"])) / exact["epsilon"]
    checks.append(("energy balance", m["energy_balance"] < 5e-3))
    return m, checks


def mms(out):
    m, checks = {}, []
    A0, eps, Om, kx, T = 1.0, 0.1, 1.0, 2, 1.0
    k, c = 2.0 * math.pi * kx / LX, math.pi / (2.0 * H)
    for b in (0, 2):
        e2 = []
        for n in (64, 128, 256):
            s = last_snap(out / f"mms_N{n}_b{b}", T)
            th = c * (s.y + H)
            g = k * k * np.sin(th) ** 2 - 2.0 * c * c * np.cos(2.0 * th)
            ex = A0 * (1.0 + eps * math.sin(Om * s.t)) * g[:, None] * np.sin(k * s.x)[None, :]
            m[f"E2_N{n}_b{b}"], m[f"Einf_N{n}_b{b}"] = l2_norm(s.omega - ex, s.y)
            e2.append(m[f"E2_N{n}_b{b}"])
        p = observed_order(e2)
        checks.append((f"beta={b}: MMS orders {['%.3f' % q for q in p]}", 1.7 <= p[-1] <= 2.3))
    return m, checks


def conservation(out):
    m, checks, drift = {}, [], {}
    for dt in (4e-3, 2e-3):
        ss = snaps(out / f"cons_dt{dt:g}")
        dy = 2.0 * H / (ss[0].Ny - 1)
        Z = np.array([0.5 * dy * np.sum(s.omega ** 2) / s.Nx for s in ss])
        E = np.array([0.5 * dy * np.sum(s.psi * s.omega) / s.Nx for s in ss])
        dZ, dE = float(np.max(np.abs(Z / Z[0] - 1.0))), float(np.max(np.abs(E / E[0] - 1.0)))
        m[f"drift_enstrophy_dt{dt:g}"], m[f"drift_energy_dt{dt:g}"] = dZ, dE
        drift[dt] = (dE, dZ)
        checks.append((f"dt={dt:g}: drifts energy {dE:.3e}, enstrophy {dZ:.3e} over {len(ss)} snapshots",
                       dE < 1e-6 and dZ < 1e-6))
    a, b = drift[4e-3], drift[2e-3]
    checks.append(("drift falls when dt is halved", b[0] < a[0] and b[1] < a[1]))
    return m, checks


def channel(out):
    m, checks, drag, T, dsave, tref = {}, [], 1e-3, 20.0, 0.05, 2.0
    d = diag(out / "channel")
    r = d[np.isfinite(d["eta_h"])]
    resid = r["dOmega_same_int_w"] - (r["A_w"] - r["eta_h"] + r["Phi_h"] + r["P_int_w"] - 2.0 * drag * r["Omega_int_w"])
    m["identity_max_over_eta_h"] = float(np.max(np.abs(resid)) / np.mean(np.abs(r["eta_h"])))
    # every output time after t = 0 (the t = 0 row holds no closure columns: nan, src/main.cu:417)
    checks.append((f"enstrophy identity at {len(r)} output times: {m['identity_max_over_eta_h']:.3e}",
                   m["identity_max_over_eta_h"] < 1e-6 and len(r) == len(d) - 1))
    late = r[r["t"] >= 0.5 * T]
    m["eta_h_over_eta_late"] = float(np.mean(late["eta_h"]) / np.mean(late["eta"]))
    m["Phi_h_over_Phi_late"] = float(np.mean(late["Phi_h"]) / np.mean(late["BOmega_wall"]))
    early = d[(d["t"] > 0) & (d["t"] <= tref + 1e-9)]
    for col in ("K", "Omega", "eta", "epsilon"):
        m[f"early_mean_{col}"] = float(np.mean(early[col]))
    m[f"K_at_t{tref:g}"] = float(early["K"][-1])
    m[f"Omega_at_t{tref:g}"] = float(early["Omega"][-1])
    fin = all(np.all(np.isfinite(d[c][1:])) for c in ("K", "Omega", "eta", "epsilon", "Re_tau"))
    checks.append((f"reached t = {float(d['t'][-1]):g} with finite diagnostics ({len(d)} rows)",
                   fin and float(d["t"][-1]) > T - dsave - 1e-6))
    return m, checks


TESTS = {"eigenmode_space": eigenmode_space, "eigenmode_time": eigenmode_time, "poiseuille": poiseuille,
         "mms": mms, "conservation": conservation, "channel": channel}
REF_SKIP = {"channel": ("identity_max_over_eta_h", "eta_h_over_eta_late", "Phi_h_over_Phi_late")}


@pytest.mark.parametrize("name", list(TESTS))
def test_reference_verification(runs, golden, name):
    metrics, checks = TESTS[name](runs)
    for desc, ok in checks:
        print(f"[{'ok' if ok else 'FAILED'}] {name}: {desc}")
    failed = [desc for desc, ok in checks if not ok]
    # against the reference's published values, at the runner's tolerance
    tol, floor = golden["ref_tol"][name], golden["ref_abs_floor"]
    ref = golden["reference_json"][name]
    bad = []
    for k, v in metrics.items():
        if k in REF_SKIP.get(name, ()) or k not in ref:
            continue
        r = ref[k]
        if max(abs(v), abs(r)) < floor:
            continue
        if abs(v - r) > tol * max(abs(r), floor):
            bad.append(f"{k}: {v:.6e} vs reference {r:.6e}")
    print(f"{name}: {len(metrics)} values against the reference (relative tolerance {tol:g}); "
          + ("all within" if not bad else "; ".join(bad)))
    assert not failed and not bad, (failed, bad)
