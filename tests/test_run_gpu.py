"""The device-side run loop (nse2d_run), the profile row moments and the 1-D spectra, on a B200.

nse2d_run replays the same captured step as nse2d_step inside a WHILE graph node, so the fields
after a run must equal those after the same number of plain steps to the bit. Its stop
conditions mirror the reference's loop (src/main.cu:434-566, 695): an output time, a statistics
step, t_end, a step budget. The row moments (src/diag.cu:468-499) are checked against the
oracle at 1e-12 relative to the size of their terms; the spectra (src/diag.cu:868-898) against numpy's
FFT of the same u, v at 1e-12 relative to the spectrum's maximum.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(Nx=128, Ny=129, Lx=2.0 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=2000.0, F0=0.05, nforce=4,
           lin_drag=1e-3, adapt=1, cfl=0.5)


def omega0(Nx, Ny, y, seed=3, amp=0.05):
    rng = np.random.default_rng(seed)
    x = np.arange(Nx) * (2 * np.pi / Nx)
    w = np.repeat((3.0 * y)[:, None], Nx, axis=1)
    for m in range(1, 9):
        w += amp * rng.standard_normal() * np.cos(m * x + 2 * np.pi * rng.random())[None, :] * \
            np.sin(rng.integers(1, 5) * np.pi * (y + 1) / 2)[:, None]
    w[0] = 3.0 * y[0]
    w[-1] = 3.0 * y[-1]
    return w


def pair(nse):
    a = nse.Solver(**CFG)
    b = nse.Solver(**CFG)
    w0 = omega0(a.Nx, a.Ny, a.metric(0))
    a.set_omega(w0)
    b.set_omega(w0)
    return a, b


def test_run_budget_matches_steps(nse, cuda):
    a, b = pair(nse)
    r = a.run(max_steps=37)
    b.step(37, use_graph=True)
    assert r == nse.HALT_BUDGET
    wa, pa = a.fields()
    wb, pb = b.fields()
    assert np.array_equal(wa, wb) and np.array_equal(pa, pb)
    ta, tb = a.time(), b.time()
    assert ta == tb


def test_run_stats_and_end(nse, cuda):
    a, b = pair(nse)
    assert a.run(stats_every=10) == nse.HALT_STATS
    assert a.time()[2] == 10
    assert a.run(stats_every=10) == nse.HALT_STATS
    assert a.time()[2] == 20
    b.step(20, use_graph=True)
    assert np.array_equal(a.fields()[0], b.fields()[0])
    t, dt = a.time()[:2]
    t_end = t + 7.5 * dt
    r = a.run(t_end=t_end)
    t2, dt2 = a.time()[:2]
    assert r & nse.HALT_END
    assert not (t2 < t_end - 0.5 * dt2)


def test_run_stops_at_output_time(nse, cuda):
    """The run stops after the first step whose t reaches the output time (src/main.cu:566);
    a replay one step at a time with the same schedule gives the same step count and t."""
    a, b = pair(nse)
    a.step(1, use_graph=True)
    b.step(1, use_graph=True)
    for frac in (5.3, 7.8):
        t, dt = a.time()[:2]
        t_out = t + frac * dt
        r = a.run(next_diag=t_out)
        assert r & nse.HALT_OUTPUT
        t2, _, n2 = a.time()[:3]
        b.set_schedule(1e300, t_out)
        while True:
            b.step(1)
            tb, dtb, nb = b.time()[:3]
            if tb + max(64 * np.finfo(float).eps * max(1.0, abs(tb)), 1e-6 * dtb) >= t_out:
                break
        assert (t2, n2) == (tb, nb)
        assert np.array_equal(a.fields()[0], b.fields()[0])


def test_row_moments_match_oracle(nse, oracle, cuda):
    a, _ = pair(nse)
    a.step(5, use_graph=True)
    _, psi = a.fields()
    got = a.row_moments()
    Nx, Ny = a.Nx, a.Ny
    ref = [np.empty(Ny) for _ in range(5)]
    L = oracle.lib()
    L.or_row_moments(oracle.p(np.ascontiguousarray(psi)), Nx, Ny, 1.0 / a.scalar(1), 1.0 / a.scalar(2),
                     oracle.p(a.metric(1)), *[oracle.p(r) for r in ref])
    ref = np.array(ref)
    # each row sum against the size of its terms: sum_i v telescopes to zero, so its value is
    # round-off and only the term scale is meaningful
    su2, sv2 = np.abs(ref[2]), np.abs(ref[3])
    scale = np.array([np.sqrt(Nx * su2), np.sqrt(Nx * sv2), su2, sv2, np.sqrt(su2 * sv2)])
    scale = np.maximum(scale, 1e-300).max(axis=1, keepdims=True)
    assert np.max(np.abs(got - ref) / scale) < 1e-12


def test_spectra_match_numpy(nse, cuda):
    a, _ = pair(nse)
    Nx, Ny = a.Nx, a.Ny
    a.step(3, use_graph=True)
    acc_u = np.zeros(Nx // 2 + 1)
    acc_v = np.zeros(Nx // 2 + 1)
    an = a.metric(1)
    inv_dx, inv_deta = 1.0 / a.scalar(1), 1.0 / a.scalar(2)
    for _ in range(2):
        a.spectra_accumulate()
        _, psi = a.fields()
        ym = np.r_[0, np.arange(Ny - 1)]
        yp = np.r_[np.arange(1, Ny), Ny - 1]
        u = an[:, None] * (psi[yp] - psi[ym]) * (0.5 * inv_deta)
        v = -(np.roll(psi, -1, axis=1) - np.roll(psi, 1, axis=1)) * (0.5 * inv_dx)
        w = np.full(Nx // 2 + 1, 2.0)
        w[0] = w[-1] = 1.0
        norm = 1.0 / (Nx * Nx * Ny)
        acc_u += norm * w * np.sum(np.abs(np.fft.rfft(u, axis=1)) ** 2, axis=0)
        acc_v += norm * w * np.sum(np.abs(np.fft.rfft(v, axis=1)) ** 2, axis=0)
        a.step(2, use_graph=True)
    kx, eu, ev, n = a.spectra()
    assert n == 2
    np.testing.assert_allclose(kx, 2 * np.pi * np.arange(Nx // 2 + 1) / a.cfg.Lx, rtol=1e-15)
    assert np.max(np.abs(eu - acc_u / 2)) < 1e-12 * np.max(acc_u / 2)
    assert np.max(np.abs(ev - acc_v / 2)) < 1e-12 * np.max(acc_v / 2)


def test_device_statistics_match_host_accumulation(nse, cuda):
    """nse2d_stats_device: the time-weighted row statistics of the reference's loop
    (src/main.cu:695-733) accumulated inside the run's graph, with no halt, equal the host's
    accumulation of nse2d_row_moments at the same steps (H += mom / Nx * dtw) to the bit."""
    a, b = pair(nse)
    Nx = a.Nx
    a.stats_device(10)
    assert a.run(max_steps=50) == nse.HALT_BUDGET          # one launch, no statistics halts
    H = np.zeros((5, a.Ny))
    T, last = 0.0, 0.0
    for k in range(5):
        assert b.run(stats_every=10) == nse.HALT_STATS
        t = b.time()[0]
        dtw = t - last
        H += b.row_moments() / Nx * dtw
        T += dtw
        last = t
    Ha, Ta = a.stats_read()
    assert Ta == T
    assert np.array_equal(Ha, H)
    assert np.array_equal(a.fields()[0], b.fields()[0])
    a.stats_device(0)
    assert a.stats_read()[1] == 0.0
