"""Failure detection without a GPU fault: NaN put into a host-prepared initial vorticity.

The reference runs on with non-finite fields and never reports them. Here the max reduction of
an adaptive step raises bit 0 of the context's non-finite flag (nse2d_nonfinite) when psi holds
NaN or Inf, and a device-side run (nse2d_run) halts once for it with NSE2D_HALT_NONFINITE, so the
host learns of it at the next return; a later run goes on, as the reference's loop would. Bit 1
(a bounded wait that ran out) is not raised by a NaN. Nothing here faults, traps or hangs the GPU:
the bad value is a NaN in an ordinary host array.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(Nx=128, Ny=65, Lx=2.0 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=2000.0, F0=0.05, nforce=4,
           lin_drag=1e-3, adapt=1, cfl=0.5)


def laminar(g):
    y = g.metric(0)
    return np.repeat((3.0 * y)[:, None], g.Nx, axis=1)


@pytest.mark.parametrize("precision", [64, 32])
def test_nan_in_initial_omega_halts_the_run_once(nse, cuda, precision):
    g = nse.Solver(precision=precision, **CFG)
    w0 = laminar(g)
    w0[g.Ny // 3, 40] = np.nan
    g.set_omega(w0)
    # FP64: setting the state runs the max reduction on psi (the next step's maxima), which flags
    # the NaN at once; FP32 flags it in the first step
    assert g.nonfinite() == (1 if precision == 64 else 0)
    r = g.run(t_end=1.0, max_steps=50)
    assert r & nse.HALT_NONFINITE, r
    assert g.time()[2] == 1                        # halted after the first step
    flags = g.nonfinite()
    assert flags & 1 and not flags & 2, flags
    # a second run is not stopped again by the same NaN: it runs to its budget
    r2 = g.run(t_end=1.0, max_steps=5)
    assert r2 == nse.HALT_BUDGET, r2
    assert g.time()[2] == 6
    g.close()


def test_finite_state_raises_no_flag(nse, cuda):
    g = nse.Solver(**CFG)
    g.set_omega(laminar(g))
    assert g.run(t_end=1.0, max_steps=20) == nse.HALT_BUDGET
    assert g.nonfinite() == 0
    g.close()


def test_max_uv_reports_nan_through_the_flag(nse, cuda):
    """nse2d_max_uv on a context whose psi holds a NaN: the maxima skip it, the flag shows it;
    setting a clean state clears the flag."""
    g = nse.Solver(**CFG)
    w0 = laminar(g)
    g.set_omega(w0)
    w, psi = g.fields()
    psi[5, 7] = np.nan
    g.set_state(w, psi, t=0.0)
    m = g.max_uv()
    assert np.all(np.isfinite(m))
    assert g.nonfinite() & 1
    g.set_omega(w0)
    assert g.nonfinite() == 0
    g.max_uv()
    assert g.nonfinite() == 0
    g.close()
