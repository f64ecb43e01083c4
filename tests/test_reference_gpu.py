"""This build against the reference's own CUDA code, both on the same B200.

oracle/_ref holds the reference compiled from its sources for sm_100a by oracle/ref.mk (its own
flags, HDF5 off). The tests skip when it was not built (the reference's sources are not on every
machine that runs the tests).

1. The seven C-linkage operators of the reference's test API (src/test_api.cu:8-92) and this
   library's, on the same device inputs: 1e-13 relative to the output's maximum (the same
   formulas up to FMA contraction).
2. The reference executable and nse2d on the same command lines: every diagnostics column of
   every row equal to the 9 significant digits the CSV prints: 1e-8 of the value plus 2e-9 of
   the column's scale (columns such as dOmega_rhs are small differences of O(1) sums), or 1e-13
   absolute for columns that are round-off in both (tau_w at Ub = 0). The two
   differ only by the order of the reductions and the FFT (cuFFT there, this project's here).
3. Fields against the reference's own time loop (oracle/_ref/libnse2d_refloop.so: the
   reference's src/main.cu:197-213 and 434-541 driven through its own launchers, built from its
   sources by oracle/ref.mk), from the same seeded initial vorticity. The small-channel
   configuration (256 x 257, Lx = 2 pi, tanh beta = 2, Ub = 1, Re_b = 500, Poiseuille plus a
   seed-0 Gaussian perturbation of 1e-3 of the wall vorticity, zero at the walls, no forcing):
   - one step at dt = 1e-3 (as configured) and at 1e-4: psi, and omega away from the walls,
     within 1e-11 relative to the field's maximum;
   - 1000 steps at dt = 1e-4: within 1e-8;
   - 1000 steps at dt = 1e-3 as configured: the step lies beyond the stability limit of SSPRK(3,3)
     for the mapped Laplacian on this grid (nu dt lambda_min = -9.7 against -2.51), so both builds
     blow up; both must reach non-finite values within two steps of each other.
   The wall rows are the Thom closure's (thom_gain ~1.5e6 times the round-off of psi at rows 1-2),
   held as in the oracle parity tests. An adaptive forced channel (512 x 257, Re_b 5000, F0 0.05 at
   mode 12, drag 1e-3) is stepped 20 times in both: dt of every step within 1e-12, fields within
   1e-10.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ORACLE, PKG, load_oracle_module
from test_parity_gpu import assert_fields_close, laminar_perturbed, relerr, thom_gain

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(ORACLE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libnse2d_ref.so")
REF_EXE = os.path.join(REF_DIR, "nse2d_ref")

need_ref = pytest.mark.skipif(not (os.path.isfile(REF_LIB) and os.path.isfile(REF_EXE)),
                              reason="the reference was not compiled here (oracle/ref.mk)")


def ref_lib():
    L = ctypes.CDLL(REF_LIB)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    sig = {
        "testapi_uv_from_psi_mapped": [P, P, P, I, I, D, D, P, P],
        "testapi_omega_from_psi_interior_mapped": [P, P, I, I, D, D, P, P, P],
        "testapi_thom_wall_vorticity_mapped": [P, P, I, I, P, D, D, P],
        "testapi_arakawa_J_mapped": [P, P, P, I, I, D, D, P, P],
        "testapi_compute_adv_from_uv_mapped": [P, P, P, P, I, I, D, D, P, P],
        "testapi_compute_adv_flux_mapped": [P, P, P, P, I, I, D, D, P, P],
        "testapi_arakawa_J_mapped_split": [P, P, P, P, P, P, I, I, D, D, P, P],
    }
    for n, a in sig.items():
        getattr(L, n).argtypes = a
        getattr(L, n).restype = None
    return L


@need_ref
def test_testapi_matches_reference(nse, cuda):
    torch = cuda
    mine = nse.load()
    ref = ref_lib()
    Nx, Ny = 256, 129
    g = nse.Solver(Nx=Nx, Ny=Ny, Lx=2 * np.pi, stretch=1, beta=2.0)
    an, ae, de = (torch.tensor(g.metric(k), dtype=torch.float64, device="cuda") for k in (1, 2, 3))
    dx, deta = g.scalar(1), g.scalar(2)
    gen = torch.Generator(device="cuda").manual_seed(5)
    psi, w, u, v = (torch.randn(Ny, Nx, dtype=torch.float64, device="cuda", generator=gen) for _ in range(4))
    P = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None   # noqa: E731
    out = lambda: torch.zeros(Ny, Nx, dtype=torch.float64, device="cuda")   # noqa: E731

    def both(fn):
        a, b = fn(mine), fn(ref)
        torch.cuda.synchronize()
        for x, y in zip(a, b):
            scale = float(y.abs().max())
            assert float((x - y).abs().max()) <= 1e-13 * max(scale, 1e-300), (float((x - y).abs().max()), scale)

    def uv(L):
        a, b = out(), out()
        L.testapi_uv_from_psi_mapped(P(psi), P(a), P(b), Nx, Ny, 1 / dx, 1 / deta, P(an), None)
        return a, b

    def om(L):
        a = out()
        L.testapi_omega_from_psi_interior_mapped(P(a), P(psi), Nx, Ny, 1 / dx**2, 1 / deta**2, P(an), P(ae), None)
        return (a[1:-1],)

    def thom(L):
        a = w.clone()
        L.testapi_thom_wall_vorticity_mapped(P(a), P(psi), Nx, Ny, P(de), 0.0, 2.0, None)
        return (a,)

    def jac(L):
        a = out()
        L.testapi_arakawa_J_mapped(P(psi), P(w), P(a), Nx, Ny, 1 / dx, 1 / deta, P(an), None)
        return (a,)

    def adv(L):
        a, b = out(), out()
        L.testapi_compute_adv_from_uv_mapped(P(u), P(v), P(w), P(a), Nx, Ny, 1 / dx, 1 / deta, P(an), None)
        L.testapi_compute_adv_flux_mapped(P(u), P(v), P(w), P(b), Nx, Ny, 1 / dx, 1 / deta, P(an), None)
        return a, b

    def split(L):
        r = [out() for _ in range(4)]
        L.testapi_arakawa_J_mapped_split(P(psi), P(w), *[P(x) for x in r], Nx, Ny, 1 / dx, 1 / deta, P(an), None)
        return r

    for fn in (uv, om, thom, jac, adv, split):
        both(fn)
    g.close()


CASES = {
    "channel": ["--Nx", "512", "--Ny", "257", "--Ub", "1", "--Reb", "5000.0", "--init", "mix", "--amp", "0.05",
                "--F0", "0.05", "--nforce", "12", "--drag", "0.001", "--stretch", "tanh", "--beta", "2",
                "--tend", "0.2", "--diag_save", "0.05", "--closure_diag"],
    "mms": ["--Nx", "128", "--Ny", "129", "--Ub", "0", "--nu", "0.01", "--init", "mms", "--mmsA0", "1.0",
            "--mmsEps", "0.1", "--mmsOm", "1.0", "--mmsKx", "2", "--stretch", "tanh", "--beta", "2", "--no-adapt",
            "--dt", "0.000125", "--tend", "0.25", "--diag_save", "0.05"],
    "poiseuille": ["--Nx", "64", "--Ny", "129", "--Ub", "1.0", "--Reb", "500.0", "--init", "laminar", "--stretch",
                   "tanh", "--beta", "2", "--tend", "1.0", "--diag_save", "0.25"],
    "diffusion2d": ["--Nx", "64", "--Ny", "65", "--Ub", "0", "--nu", "0.01", "--init", "diffusion2d", "--amp", "0.5",
                    "--my", "2", "--stretch", "none", "--no-adapt", "--dt", "0.001", "--tend", "0.1",
                    "--diag_save", "0.025"],
}


def run(exe, args, out):
    p = subprocess.run([exe] + args + ["--snap_save", "0", "--outdir", out], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return np.atleast_1d(np.genfromtxt(os.path.join(out, "diagnostics.csv"), delimiter=",", names=True))


@need_ref
@pytest.mark.parametrize("case", sorted(CASES))
def test_runs_match_reference_executable(cuda, tmp_path, case):
    a = CASES[case]
    ref = run(REF_EXE, a, str(tmp_path / "ref"))
    mine = run(os.path.join(PKG, "nse2d"), a, str(tmp_path / "mine"))
    assert len(mine) == len(ref) and len(ref) >= 3
    for name in ref.dtype.names:
        r, m = ref[name], mine[name]
        fin = np.isfinite(r)
        assert np.array_equal(fin, np.isfinite(m)), name
        if name in ("utau_avg", "Cf", "Re_tau") and np.max(np.abs(ref["tauw_bot"])) < 1e-13:
            continue
        scale = max(float(np.max(np.abs(r[fin]))) if fin.any() else 0.0, 1e-300)
        err = np.abs(m[fin] - r[fin])
        # a column that is round-off in both (e.g. tau_w of a flow with Ub = 0) is held to 1e-13
        tol = 1e-8 * np.abs(r[fin]) + max(2e-9 * scale, 1e-13)
        assert np.all(err <= tol), (name, float(np.max(err)), scale)


refloop = load_oracle_module("ref_loop")
need_loop = pytest.mark.skipif(not refloop.available(),
                               reason="the reference's loop harness was not compiled here (oracle/ref.mk)")
SMALL = dict(Nx=256, Ny=257, Lx=2 * np.pi, h=1.0, stretch=1, beta=2.0, Ub=1.0, Reb=500.0, adapt=0)


def _both(nse, dt, **kw):
    cfg = dict(SMALL, dt_init=dt, **kw)
    g = nse.Solver(**cfg)
    r = refloop.RefLoop(**cfg)
    w0 = laminar_perturbed(cfg["Nx"], cfg["Ny"], g.metric(0), seed=0, amp=1e-3)
    g.set_omega(w0)
    r.set_omega(w0)
    return g, r


@need_loop
@pytest.mark.parametrize("dt", [1e-3, 1e-4])
def test_small_channel_one_step_matches_reference_loop(nse, cuda, dt):
    """One step. At dt = 1e-4: psi and omega to 1e-11, the wall rows to the Thom-gain bound. At
    dt = 1e-3, past the stability limit, the step multiplies the stiffest wall-normal mode by
    |R(nu dt lambda_min)| = |1 + z + z^2/2 + z^3/6| ~ 115 (z = -9.7), and the Thom closure's
    round-off in the wall rows (thom_gain ulp(psi)) reaches the first rows inside through the
    Laplacian of stages 2 and 3: psi and omega beyond 4 rows of a wall are held to 1e-11, the 4 rows
    next to each wall to 115 times the Thom-gain bound."""
    g, r = _both(nse, dt)
    wg, pg = g.fields()
    wr, pr = r.fields()
    assert_fields_close(wg, pg, wr, pr, g.metric(3), 1e-12)          # the initial solve and closure
    g.step(1)
    r.step(1)
    wg, pg = g.fields()
    wr, pr = r.fields()
    rows = np.max(np.abs(wg - wr), axis=1) / np.max(np.abs(wr))
    print(f"dt={dt:g}: one step, psi {relerr(pg, pr):.2e}; omega by row (first 6): "
          + " ".join(f"{e:.1e}" for e in rows[:6]) + f"; rows 4..Ny-5 {rows[4:-4].max():.2e}")
    if dt == 1e-4:
        assert_fields_close(wg, pg, wr, pr, g.metric(3), 1e-11)
    else:
        assert relerr(pg, pr) < 1e-11
        assert rows[4:-4].max() < 1e-11, rows[4:-4].max()
        bound = 115.0 * thom_gain(g.metric(3)) * 8 * np.finfo(float).eps * np.max(np.abs(pr)) / np.max(np.abs(wr))
        near = np.concatenate([rows[:4], rows[-4:]])
        assert near.max() < bound, (near, bound)
    g.close()
    r.close()


@need_loop
def test_small_channel_1000_steps_matches_reference_loop(nse, cuda):
    g, r = _both(nse, 1e-4)
    g.step(1000, use_graph=True)
    r.step(1000)
    wg, pg = g.fields()
    wr, pr = r.fields()
    assert_fields_close(wg, pg, wr, pr, g.metric(3), 1e-8)
    assert abs(g.time()[0] - r.time()[0]) < 1e-15
    print(f"1000 steps at dt=1e-4: psi {relerr(pg, pr):.2e}, omega {relerr(wg, wr):.2e}")
    g.close()
    r.close()


@need_loop
def test_small_channel_as_configured_blows_up_in_both(nse, cuda):
    """dt = 1e-3 for up to 1000 steps: the first step with a non-finite omega in each build."""
    g, r = _both(nse, 1e-3)
    first = {}
    for n in range(1, 1001):
        if "ours" not in first:
            g.step(1)
            if not np.all(np.isfinite(g.fields()[0])):
                first["ours"] = n
        if "reference" not in first:
            r.step(1)
            if not np.all(np.isfinite(r.fields()[0])):
                first["reference"] = n
        if len(first) == 2:
            break
    print(f"dt=1e-3: first non-finite omega at step {first.get('ours')} (this build), "
          f"{first.get('reference')} (the reference's loop)")
    assert len(first) == 2, first
    assert abs(first["ours"] - first["reference"]) <= 2, first
    g.close()
    r.close()


@need_loop
def test_adaptive_forced_channel_matches_reference_loop(nse, cuda):
    cfg = dict(Nx=512, Ny=257, Lx=4.0 * np.pi, h=1.0, stretch=1, beta=2.0, Ub=1.0, Reb=5000.0, F0=0.05, nforce=12,
               lin_drag=1e-3, adapt=1, cfl=0.5, dt_max=1e-2, dt_init=1e-3)
    g = nse.Solver(**cfg)
    r = refloop.RefLoop(**cfg)
    w0 = laminar_perturbed(512, 257, g.metric(0), seed=4, amp=5e-2)
    g.set_omega(w0)
    r.set_omega(w0)
    for n in range(20):
        g.step(1)
        r.step(1)
        tg, dtg = g.time()[:2]
        tr, dtr = r.time()[:2]
        assert abs(dtg - dtr) <= 1e-12 * dtr, (n, dtg, dtr)
        assert abs(tg - tr) <= 1e-12 * tr, (n, tg, tr)
    wg, pg = g.fields()
    wr, pr = r.fields()
    assert_fields_close(wg, pg, wr, pr, g.metric(3), 1e-10)
    g.close()
    r.close()
