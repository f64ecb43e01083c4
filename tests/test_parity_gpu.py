"""Parity of the CUDA path (through the C ABI) with the CPU oracle, on a B200.

Tolerances (FP64): single operators 1e-13 relative to the field's max (the same arithmetic up
to FMA contraction); Poisson solve 1e-12 (FFT and the segmented Thomas sweep reassociate
sums); one SSPRK(3,3) step 1e-11 and 1000 steps 1e-8 relative to max|field| (the bars of the
specification; omega near the walls also carries the Thom closure gain, see assert_fields_close);
diagnostics rows 1e-9 relative per column with an absolute floor of 1e-12
times the column scale (reductions in a different order).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRIDS = [(8, 5, 0, 0.0), (16, 9, 1, 2.0), (64, 33, 0, 0.0), (64, 65, 1, 2.0), (128, 129, 1, 2.0),
         (256, 257, 1, 2.0), (512, 257, 1, 2.0),
         # the longest rows the row transforms take (M = 4096 and 8192), with few rows
         (8192, 65, 1, 2.0), (16384, 33, 0, 0.0),
         # row counts that are not 2^k + 1 (partial stage tiles, uneven Thomas segments and bands)
         (128, 50, 1, 2.0), (256, 301, 1, 1.5), (1024, 777, 0, 0.0)]


def laminar_perturbed(Nx, Ny, y, seed=0, amp=1e-3, Ub=1.0, h=1.0):
    """Poiseuille vorticity 3 Ub y / h^2 plus a seeded Gaussian perturbation of amplitude amp times
    the wall vorticity 3 Ub / h, zero on the wall rows (the small-channel configuration)."""
    rng = np.random.default_rng(seed)
    w = np.repeat((3.0 * Ub * y / (h * h))[:, None], Nx, axis=1)
    pert = amp * (3.0 * Ub / h) * rng.standard_normal((Ny, Nx))
    pert[0, :] = 0.0
    pert[-1, :] = 0.0
    return w + pert


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def thom_gain(dy_edge):
    """Largest factor by which the Thom closure (src/ops.cu:121-149) multiplies a difference in psi
    at the first interior rows into the wall vorticity: |A| + |B| at either wall."""
    g = 0.0
    for d1, d2 in ((dy_edge[0], dy_edge[1]), (dy_edge[-1], dy_edge[-2])):
        A = 2.0 * (1.0 / (d1 * d1) + 1.0 / (d1 * d2))
        B = -2.0 * d1 / (d2 * (d1 + d2) * (d1 + d2))
        g = max(g, abs(A) + abs(B))
    return g


def assert_fields_close(wg, pg, wo, po, dy_edge, tol):
    """psi and omega away from the walls (rows 2 .. Ny-3) within tol, relative to the field's max.
    The wall rows come from the Thom closure, which multiplies round-off differences of psi at the
    first interior rows by thom_gain (~2/dy_1^2, 1.5e6 on the 257-row tanh grid), and the next rows
    take those wall differences through the Laplacian in the following stage; these four rows are
    held to tol plus thom_gain * 8 ulp(max |psi|), relative to max |omega|."""
    assert relerr(pg, po) < tol, ("psi", relerr(pg, po))
    scale = np.max(np.abs(wo))
    e_int = np.max(np.abs(wg[2:-2] - wo[2:-2])) / scale
    assert e_int < tol, ("omega interior", e_int)
    e_wall = np.max(np.abs(wg[[0, 1, -2, -1]] - wo[[0, 1, -2, -1]])) / scale
    bound = tol + thom_gain(dy_edge) * 8 * np.finfo(float).eps * np.max(np.abs(po)) / scale
    assert e_wall < bound, ("omega near the walls", e_wall, bound)


@pytest.mark.parametrize("Nx,Ny,stretch,beta", GRIDS)
def test_poisson_parity(nse, oracle, cuda, Nx, Ny, stretch, beta):
    torch = cuda
    Lx = 2 * np.pi
    s = nse.Solver(Nx=Nx, Ny=Ny, Lx=Lx, stretch=stretch, beta=beta, Ub=1.0, Reb=500.0)
    m = oracle.metrics(Nx, Ny, Lx, 1.0, stretch, beta)
    for which, name in enumerate(["y", "a_node", "a_edge", "dy_edge", "w_node"]):
        assert np.array_equal(s.metric(which), m[name]), name
    rng = np.random.default_rng(Nx * 1000 + Ny)
    w = rng.standard_normal((Ny, Nx))
    psi_ref = oracle.poisson_solve(w, Lx, m, 0.0, 2.0)
    wd = torch.from_numpy(w).cuda()
    pd = torch.zeros_like(wd)
    s.poisson_solve(wd, pd)
    torch.cuda.synchronize()
    assert relerr(pd.cpu().numpy(), psi_ref) < 1e-12
    s.close()


def test_testapi_operators(nse, oracle, cuda):
    torch = cuda
    Nx, Ny, Lx = 128, 65, 2 * np.pi
    m = oracle.metrics(Nx, Ny, Lx, 1.0, 1, 2.0)
    rng = np.random.default_rng(7)
    psi, w, u, v = (rng.standard_normal((Ny, Nx)) for _ in range(4))
    inv_dx, deta = Nx / Lx, 2.0 / (Ny - 1)
    inv_deta = 1.0 / deta
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    an, ae, de = T(m["a_node"]), T(m["a_edge"]), T(m["dy_edge"])
    api = nse.Testapi()
    P = oracle.p
    L = oracle.lib()
    # Arakawa
    Jd = torch.zeros((Ny, Nx), dtype=torch.float64, device="cuda")
    api.arakawa_J_mapped(T(psi), T(w), Jd, Nx, Ny, inv_dx, inv_deta, an)
    Jr = np.empty((Ny, Nx)); L.or_arakawa(P(psi), P(w), P(Jr), Nx, Ny, inv_dx, inv_deta, P(m["a_node"]))
    torch.cuda.synchronize()
    assert relerr(Jd.cpu().numpy(), Jr) < 1e-13
    # split, with one output omitted
    outs = [torch.zeros((Ny, Nx), dtype=torch.float64, device="cuda") for _ in range(3)]
    api.arakawa_J_mapped_split(T(psi), T(w), outs[0], None, outs[1], outs[2], Nx, Ny, inv_dx, inv_deta, an)
    J1, J3, Ja = (np.empty((Ny, Nx)) for _ in range(3))
    L.or_arakawa_split(P(psi), P(w), P(J1), None, P(J3), P(Ja), Nx, Ny, inv_dx, inv_deta, P(m["a_node"]))
    torch.cuda.synchronize()
    for a, b in zip(outs, (J1, J3, Ja)):
        assert relerr(a.cpu().numpy(), b) < 1e-13
    # u, v
    ud, vd = (torch.zeros((Ny, Nx), dtype=torch.float64, device="cuda") for _ in range(2))
    api.uv_from_psi_mapped(T(psi), ud, vd, Nx, Ny, inv_dx, inv_deta, an)
    ur, vr = np.empty((Ny, Nx)), np.empty((Ny, Nx))
    L.or_uv_from_psi(P(psi), P(ur), P(vr), Nx, Ny, inv_dx, inv_deta, P(m["a_node"]))
    torch.cuda.synchronize()
    assert relerr(ud.cpu().numpy(), ur) < 1e-14 and relerr(vd.cpu().numpy(), vr) < 1e-14
    # omega from psi (interior rows only are written)
    wd = T(w.copy())
    api.omega_from_psi_interior_mapped(wd, T(psi), Nx, Ny, inv_dx ** 2, inv_deta ** 2, an, ae)
    wr = w.copy()
    L.or_omega_from_psi_interior(P(wr), P(psi), Nx, Ny, inv_dx ** 2, inv_deta ** 2, P(m["a_node"]), P(m["a_edge"]))
    torch.cuda.synchronize()
    assert relerr(wd.cpu().numpy(), wr) < 1e-13
    # advective and flux references
    for gname, oname in (("compute_adv_from_uv_mapped", "or_adv_from_uv"), ("compute_adv_flux_mapped", "or_adv_flux")):
        od = torch.zeros((Ny, Nx), dtype=torch.float64, device="cuda")
        getattr(api, gname)(T(u), T(v), T(w), od, Nx, Ny, inv_dx, inv_deta, an)
        orr = np.empty((Ny, Nx))
        getattr(L, oname)(P(u), P(v), P(w), P(orr), Nx, Ny, inv_dx, inv_deta, P(m["a_node"]))
        torch.cuda.synchronize()
        assert relerr(od.cpu().numpy(), orr) < 1e-13, gname
    # Thom, no-slip then free-slip
    for fs in (0, 1):
        nse.load().nse2d_testapi_set_free_slip(fs)
        wd = T(w.copy())
        api.thom_wall_vorticity_mapped(wd, T(psi), Nx, Ny, de, 0.0, 2.0)
        wr = w.copy()
        L.or_thom(P(wr), P(psi), Nx, Ny, P(m["dy_edge"]), 0.0, 2.0, fs)
        torch.cuda.synchronize()
        assert relerr(wd.cpu().numpy(), wr) < 1e-13
    nse.load().nse2d_testapi_set_free_slip(0)


def _pair(nse, oracle, **cfg):
    g = nse.Solver(**cfg)
    o = oracle.OracleSolver(**cfg)
    return g, o


CASES = {
    # the small plain-method configuration (256 x 257, tanh 2, Re_b 500), at a stable dt
    "small": dict(Nx=256, Ny=257, Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=500.0, adapt=0, dt_init=1e-4),
    # forced channel with drag, uniform grid
    "forced": dict(Nx=128, Ny=65, Lx=4 * np.pi, stretch=0, beta=0.0, Ub=1.0, Reb=2000.0, F0=0.05, nforce=4,
                   lin_drag=1e-3, adapt=0, dt_init=5e-4),
    # manufactured solution (forcing evaluated at the three stage times)
    "mms": dict(Nx=64, Ny=65, Lx=4 * np.pi, stretch=1, beta=2.0, Ub=0.0, nu_override=1e-2, mms=1, mms_A0=1.0,
                mms_eps=0.1, mms_Om=1.0, mms_kx=2, adapt=0, dt_init=5e-4),
    # free-slip walls
    "freeslip": dict(Nx=64, Ny=33, Lx=2 * np.pi, stretch=0, Ub=0.0, nu_override=0.0, free_slip=1, adapt=0,
                     dt_init=2e-3),
}


@pytest.mark.parametrize("case", list(CASES))
def test_one_step(nse, oracle, cuda, case):
    cfg = CASES[case]
    g, o = _pair(nse, oracle, **cfg)
    y = o.metric(0)
    w0 = laminar_perturbed(cfg["Nx"], cfg["Ny"], y, seed=0, amp=1e-3, Ub=max(cfg["Ub"], 1.0))
    g.set_omega(w0)
    o.set_omega(w0)
    de = o.metric(3)
    wg, pg = g.fields()
    wo, po = o.fields()
    assert_fields_close(wg, pg, wo, po, de, 1e-12)
    g.step(1)
    o.step(0.0, cfg["dt_init"])
    wg, pg = g.fields()
    wo, po = o.fields()
    assert_fields_close(wg, pg, wo, po, de, 1e-11)
    t, dt, st, _ = g.time()
    assert st == 1 and abs(t - cfg["dt_init"]) < 1e-18


def test_1000_steps_small_channel(nse, oracle, cuda):
    """256 x 257 tanh channel, Re_b 500, dt 1e-4: 1000 steps within 1e-8 of the oracle."""
    cfg = CASES["small"]
    g, o = _pair(nse, oracle, **cfg)
    w0 = laminar_perturbed(cfg["Nx"], cfg["Ny"], o.metric(0), seed=0, amp=1e-3)
    g.set_omega(w0)
    o.set_omega(w0)
    g.step(1000, use_graph=True)
    for n in range(1000):
        o.step(n * 1e-4, 1e-4)
    wg, pg = g.fields()
    wo, po = o.fields()
    assert_fields_close(wg, pg, wo, po, o.metric(3), 1e-8)


def test_adaptive_dt_sequence(nse, oracle, cuda):
    """Device-side adaptive dt (max |u|, |v|, CFL, viscous limit) matches the oracle's, step by step."""
    cfg = dict(Nx=128, Ny=129, Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=5000.0, F0=0.05, nforce=8,
               lin_drag=1e-3, adapt=1, cfl=0.5, dt_max=1e-2)
    g, o = _pair(nse, oracle, **cfg)
    w0 = laminar_perturbed(128, 129, o.metric(0), seed=3, amp=5e-2)
    g.set_omega(w0)
    o.set_omega(w0)
    t = 0.0
    for n in range(20):
        dto, mo = o.adapt_dt()
        o.step(t, dto)
        t += dto
        g.step(1)
        tg, dtg, st, mg = g.time()
        assert abs(dtg - dto) <= 1e-13 * dto, (n, dtg, dto)
        assert np.allclose(mg, mo, rtol=1e-12, atol=0)
        assert abs(tg - t) <= 1e-13 * max(t, 1.0)
    wg, pg = g.fields()
    wo, po = o.fields()
    assert_fields_close(wg, pg, wo, po, o.metric(3), 1e-10)


DIAG_CASES = {
    "channel_closure": dict(Nx=128, Ny=129, Lx=4 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=5000.0, F0=0.05,
                            nforce=12, lin_drag=1e-3, adapt=0, dt_init=2e-4, closure_diag=1),
    "mms": CASES["mms"],
}


@pytest.mark.parametrize("case", list(DIAG_CASES))
def test_diagnostics_rows(nse, oracle, cuda, case):
    cfg = DIAG_CASES[case]
    g, o = _pair(nse, oracle, **cfg)
    w0 = laminar_perturbed(cfg["Nx"], cfg["Ny"], o.metric(0), seed=5, amp=1e-2, Ub=1.0)
    g.set_omega(w0)
    o.set_omega(w0)
    names = nse.DIAG_COLUMNS

    def check(rg, ro):
        for k, name in enumerate(names):
            a, b = rg[name], ro[k]
            if np.isnan(b):
                assert np.isnan(a), name
                continue
            assert abs(a - b) <= 1e-9 * abs(b) + 1e-12 * max(1.0, abs(b)), (name, a, b)

    check(g.diagnostics(t0_row=True), o.diag_row(0.0, t0_row=True))
    dt = cfg["dt_init"]
    g.step(9)
    g.step_store_rhs(1)
    for n in range(10):
        o.step(n * dt, dt)
    check(g.diagnostics(t0_row=False), o.diag_row(10 * dt, t0_row=False))


@pytest.mark.parametrize("Nx,Ny", [(8192, 65), (16384, 33)])
def test_steps_long_rows(nse, oracle, cuda, Nx, Ny):
    """Three adaptive steps on the longest rows the row transforms take, against the oracle:
    dt and the maxima of every step to 1e-12, the fields to 1e-10."""
    cfg = dict(Nx=Nx, Ny=Ny, Lx=4 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=2000.0, F0=0.05, nforce=8,
               lin_drag=1e-3, adapt=1, cfl=0.5)
    g, o = _pair(nse, oracle, **cfg)
    w0 = laminar_perturbed(Nx, Ny, o.metric(0), seed=7, amp=1e-2)
    g.set_omega(w0)
    o.set_omega(w0)
    t = 0.0
    for _ in range(3):
        dto, mo = o.adapt_dt()
        o.step(t, dto)
        t += dto
        g.step(1)
        tg, dtg, st, mg = g.time()
        assert abs(dtg - dto) <= 1e-12 * dto, (dtg, dto)
        assert np.allclose(mg, mo, rtol=1e-12, atol=0)
    wg, pg = g.fields()
    wo, po = o.fields()
    assert_fields_close(wg, pg, wo, po, o.metric(3), 1e-10)


@pytest.mark.parametrize("Nx,Ny,precision", [(128, 50, 64), (256, 301, 64), (1024, 777, 64), (256, 301, 32)])
def test_steps_uneven_rows(nse, oracle, cuda, Nx, Ny, precision):
    """Five adaptive steps on row counts that are not 2^k + 1, against the oracle: dt to 1e-12 and
    the fields to 1e-10 in FP64 (FP32 bulk: dt to 1e-6, omega to 1e-5 of its max, psi to 1e-6)."""
    cfg = dict(Nx=Nx, Ny=Ny, Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=2000.0, F0=0.05, nforce=4,
               lin_drag=1e-3, adapt=1, cfl=0.5)
    g = nse.Solver(precision=precision, **cfg)
    o = oracle.OracleSolver(**cfg)
    w0 = laminar_perturbed(Nx, Ny, o.metric(0), seed=11, amp=1e-2)
    g.set_omega(w0)
    o.set_omega(w0)
    t = 0.0
    for _ in range(5):
        dto, mo = o.adapt_dt()
        o.step(t, dto)
        t += dto
        g.step(1)
        dtg = g.time()[1]
        assert abs(dtg - dto) <= (1e-12 if precision == 64 else 1e-6) * dto, (dtg, dto)
    wg, pg = g.fields()
    wo, po = o.fields()
    if precision == 64:
        assert_fields_close(wg, pg, wo, po, o.metric(3), 1e-10)
    else:
        assert relerr(pg, po) < 1e-6, relerr(pg, po)
        assert np.max(np.abs(wg - wo)) / np.max(np.abs(wo)) < 1e-5
