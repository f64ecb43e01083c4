"""The FP32-bulk variant (precision 32) against the FP64 path and the oracle, on a B200.

The variant steps FP32 fluctuations about fixed FP64 base profiles (the x-means of the initial
state) with an FP32 spectral buffer and the tridiagonal solve's arithmetic and table in FP64. Its
error is FP32 rounding of the fluctuations, so the bars here are FP32-level:
  - split and export of the initial state: 1e-6 of max |omega| / max |psi|;
  - one step: 2e-5 of max |omega| and 1e-5 of max |psi|;
  - 200 steps of a forced turbulent-ish channel: 1e-3 of max |omega|, and the diagnostics K,
    Omega, u_tau, Re_tau, C_f and the wall enstrophy flux BOmega_wall within 1e-3 relative;
  - against the oracle (the CPU restatement of the reference's FP64 algorithm) at a fixed dt, at
    256x129 (200 steps) and 4096x2049 (20 steps): omega within 1e-4 of its max away from the walls
    (the two rows next to each wall within 1e-3: they carry the Thom gain), psi within 1e-6,
    K and Omega within 1e-6 relative, u_tau, Re_tau and C_f within 1e-5, BOmega_wall within 1e-3;
    the FP64 path within 1e-9, and 1e-7 for the quantities taken at the walls (the wall vorticity
    and shear carry the Thom gain on the round-off of psi next to the walls).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(Nx=256, Ny=129, Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=5000.0, F0=0.05, nforce=8,
           lin_drag=1e-3, adapt=1, cfl=0.5)


def omega0(Nx, Ny, y, seed=4, amp=0.1):
    rng = np.random.default_rng(seed)
    x = np.arange(Nx) * (2 * np.pi / Nx)
    w = np.repeat((3.0 * y)[:, None], Nx, axis=1)
    for m in range(1, 17):
        w += amp * rng.standard_normal() * np.cos(m * x + 2 * np.pi * rng.random())[None, :] * \
            np.sin(rng.integers(1, 7) * np.pi * (y + 1) / 2)[:, None]
    w[0], w[-1] = 3.0 * y[0], 3.0 * y[-1]
    return w


def pair(nse, **kw):
    cfg = dict(CFG, **kw)
    a = nse.Solver(**cfg)
    b = nse.Solver(precision=32, **cfg)
    w0 = omega0(a.Nx, a.Ny, a.metric(0))
    a.set_omega(w0)
    b.set_omega(w0)
    return a, b


def rel(x, ref):
    return float(np.max(np.abs(x - ref)) / np.max(np.abs(ref)))


def test_split_and_export(nse, cuda):
    a, b = pair(nse)
    wa, pa = a.fields()
    wb, pb = b.fields()
    assert rel(wb, wa) < 1e-6 and rel(pb, pa) < 1e-6


def test_one_step(nse, cuda):
    a, b = pair(nse)
    a.step(1)
    b.step(1)
    assert b.time()[:3] == pytest.approx(a.time()[:3], rel=1e-6)
    wa, pa = a.fields()
    wb, pb = b.fields()
    assert rel(wb, wa) < 2e-5, rel(wb, wa)
    assert rel(pb, pa) < 1e-5, rel(pb, pa)


@pytest.mark.parametrize("walls", ["no_slip", "free_slip"])
def test_200_steps_and_diagnostics(nse, cuda, walls):
    a, b = pair(nse, free_slip=1 if walls == "free_slip" else 0)
    a.step(200, use_graph=True)
    b.step(200, use_graph=True)
    wa, _ = a.fields()
    wb, _ = b.fields()
    assert rel(wb, wa) < 1e-3, rel(wb, wa)
    da, db = a.diagnostics(), b.diagnostics()
    for k in ("K", "Omega", "utau_avg", "Re_tau", "Cf", "BOmega_wall"):
        if walls == "free_slip" and k in ("utau_avg", "Re_tau", "Cf"):
            continue
        assert abs(db[k] - da[k]) <= 1e-3 * abs(da[k]) + 1e-12, (k, db[k], da[k])


def test_run_loop_and_ensemble(nse, cuda):
    a, b = pair(nse)
    r = b.run(stats_every=25)
    assert r == nse.HALT_STATS and b.time()[2] == 25
    c = nse.Solver(precision=32, **CFG)
    c.set_omega(omega0(c.Nx, c.Ny, c.metric(0)))
    e = nse.Ensemble([c])
    e.step(25)
    assert np.array_equal(c.fields()[0], b.fields()[0])
    e.close()


SIX = ("K", "Omega", "utau_avg", "Re_tau", "Cf", "BOmega_wall")


@pytest.mark.parametrize("Nx,Ny,steps", [(256, 129, 200), (4096, 2049, 20)])
def test_against_oracle(nse, oracle, cuda, Nx, Ny, steps):
    import os
    oracle.lib().or_set_threads(os.cpu_count() or 1)
    cfg = dict(CFG, Nx=Nx, Ny=Ny, adapt=0)
    o = oracle.OracleSolver(**cfg)
    y = o.metric(0)
    w0 = omega0(Nx, Ny, y)
    o.set_omega(w0)
    dt = 0.9 * o.adapt_dt()[0]                     # a fixed step below the CFL and viscous limits
    cfg["dt_init"] = dt
    t = 0.0
    for _ in range(steps):
        o.step(t, dt)
        t += dt
    wo, po = o.fields()
    do = dict(zip(nse.DIAG_COLUMNS, o.diag_row(t, t0_row=True)))
    o.close()
    # the wall enstrophy flux takes the wall vorticity, which carries the Thom closure's gain on the
    # round-off of psi next to the walls (1e-7 in FP64)
    # (as do u_tau, Re_tau and C_f, through the wall shear)
    bars = {64: dict(omega=1e-9, psi=1e-9, bulk=1e-9, wall=1e-7, bw=1e-7),
            32: dict(omega=1e-4, psi=1e-6, bulk=1e-6, wall=1e-5, bw=1e-3)}
    for P in (64, 32):
        g = nse.Solver(precision=P, **cfg)
        g.set_omega(w0)
        g.step(steps, use_graph=True)
        assert g.time()[1] == dt
        wg, pg = g.fields()
        dg = g.diagnostics(t0_row=True)
        g.close()
        b = bars[P]
        # omega away from the walls; the wall rows and their neighbours carry the Thom gain
        # (2/dy_1^2 = 1e8 on the 4096x2049 grid) on the round-off of psi next to the walls
        scale = np.max(np.abs(wo))
        e_int = np.max(np.abs(wg[2:-2] - wo[2:-2])) / scale
        e_wall = np.max(np.abs(wg[[0, 1, -2, -1]] - wo[[0, 1, -2, -1]])) / scale
        assert e_int < b["omega"], (P, e_int)
        assert e_wall < max(b["omega"], b["bw"]), (P, e_wall)
        assert rel(pg, po) < b["psi"], (P, rel(pg, po))
        for k in SIX:
            e = abs(dg[k] - do[k]) / abs(do[k])
            bar = b["bw"] if k == "BOmega_wall" else (b["bulk"] if k in ("K", "Omega") else b["wall"])
            assert e < bar, (P, k, e, dg[k], do[k])


def test_fp32_plan_forms_agree(nse, cuda):
    """The FP32-bulk step's kernel forms (TMA stage kernel or a CTA per tile, cluster or two-pass
    tridiagonal solve over the FP32 spectra) agree to FP32 round-off after 20 steps at 512x257."""
    cfg = dict(CFG, Nx=512, Ny=257)
    out = {}
    for st in (1, 0):
        for cl in (1, 0):
            g = nse.Solver(precision=32, **cfg)
            g.set_plan(stage_tma=st, tridiag_clusters=cl)
            p = g.plan()
            assert (p["stage_tma"], p["tridiag_clusters"]) == (st, cl)
            g.set_omega(omega0(g.Nx, g.Ny, g.metric(0)))
            g.step(20, use_graph=True)
            out[(st, cl)] = g.fields()
            g.close()
    wr, pr = out[(1, 1)]
    for key, (w, psi) in out.items():
        assert rel(w, wr) < 1e-5, (key, rel(w, wr))
        assert rel(psi, pr) < 1e-6, (key, rel(psi, pr))
