"""The headline grid, 4096 x 2049 with the bench workload's physics, on a B200.

The row transforms are compiled per length (M = Nx / 2 = 2048 here), and the 4096-point rows
take code paths that the smaller parity grids do not reach: the staged rows of the inverse
transforms, their shared-memory layout, full tile rows of the persistent TMA stage kernels and
the strip/band items of the max reductions. These tests hold them to the bars of the small grids:
  - Poisson solve against the oracle: 1e-12 relative to max |psi|;
  - 10 SSPRK(3,3) steps with the adaptive dt against the oracle: every dt and max |u|, |v|,
    |v| a within 1e-12 relative; psi within 1e-10, and omega within 1e-10 away from the walls.
    On this grid the first spacing is 1.4e-4, so the Thom closure multiplies round-off in psi
    at the first interior rows by ~1e8 into the wall vorticity (thom_gain), and viscosity carries
    that into the next rows over the 30 stages. Omega within WALL_ROWS rows of a wall is held to
    thom_gain * 8 ulp(max |psi|) relative to max |omega| (as the parity tests hold the wall rows);
  - max |u|, |v|, |v| a of a state: exactly the per-point maxima (numpy);
  - the FP32-bulk variant, one step against FP64: 2e-5 of max |omega|, 1e-5 of max |psi|.
"""
import numpy as np
import pytest

from test_parity_gpu import laminar_perturbed, relerr, thom_gain
from test_zz_no_alloc import _numpy_max_uv

pytestmark = pytest.mark.gpu

WALL_ROWS = 16
CFG = dict(Nx=4096, Ny=2049, Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=2.0e4, F0=0.05, nforce=12,
           lin_drag=1e-3, adapt=1, cfl=0.5, dt_max=1e-2, dt_init=1e-3)


def test_poisson_fullsize(nse, oracle, cuda):
    torch = cuda
    Nx, Ny, Lx = CFG["Nx"], CFG["Ny"], CFG["Lx"]
    s = nse.Solver(**CFG)
    m = oracle.metrics(Nx, Ny, Lx, 1.0, 1, 2.0)
    rng = np.random.default_rng(2049)
    w = rng.standard_normal((Ny, Nx))
    psi_ref = oracle.poisson_solve(w, Lx, m, 0.0, 2.0)
    wd = torch.from_numpy(w).cuda()
    pd = torch.zeros_like(wd)
    s.poisson_solve(wd, pd)
    torch.cuda.synchronize()
    assert relerr(pd.cpu().numpy(), psi_ref) < 1e-12
    s.close()


def test_steps_fullsize(nse, oracle, cuda):
    g = nse.Solver(**CFG)
    o = oracle.OracleSolver(**CFG)
    w0 = laminar_perturbed(CFG["Nx"], CFG["Ny"], o.metric(0), seed=5, amp=5e-2)
    g.set_omega(w0)
    o.set_omega(w0)
    t = 0.0
    for n in range(10):
        dto, mo = o.adapt_dt()
        o.step(t, dto)
        t += dto
        g.step(1)
        tg, dtg, st, mg = g.time()
        assert abs(dtg - dto) <= 1e-12 * dto, (n, dtg, dto)
        assert np.allclose(mg, mo, rtol=1e-12, atol=0), (n, mg, mo)
    wg, pg = g.fields()
    wo, po = o.fields()
    assert relerr(pg, po) < 1e-10, ("psi", relerr(pg, po))
    scale = np.max(np.abs(wo))
    err_rows = np.max(np.abs(wg - wo), axis=1) / scale
    far = err_rows[WALL_ROWS:-WALL_ROWS]
    assert far.max() < 1e-10, ("omega away from the walls", far.max(), WALL_ROWS + int(far.argmax()))
    near = np.concatenate([err_rows[:WALL_ROWS], err_rows[-WALL_ROWS:]])
    bound = thom_gain(o.metric(3)) * 8 * np.finfo(float).eps * np.max(np.abs(po)) / scale
    assert near.max() < bound, ("omega near the walls", near.max(), bound)
    # the reduction of the final state, against the per-point maxima
    um = np.array(g.max_uv())
    exp = np.array(_numpy_max_uv(pg, g.metric(1), 1.0 / g.scalar(1), 1.0 / g.scalar(2)))
    np.testing.assert_array_equal(um, exp)
    g.close()
    o.close()


def test_fp32_one_step_fullsize(nse, cuda):
    a = nse.Solver(**CFG)
    b = nse.Solver(precision=32, **CFG)
    w0 = laminar_perturbed(CFG["Nx"], CFG["Ny"], a.metric(0), seed=6, amp=5e-2)
    a.set_omega(w0)
    b.set_omega(w0)
    a.step(1)
    b.step(1)
    wa, pa = a.fields()
    wb, pb = b.fields()
    assert relerr(wb, wa) < 2e-5
    assert relerr(pb, pa) < 1e-5
    a.close()
    b.close()
