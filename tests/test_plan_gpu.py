"""Kernel plans of a context (nse2d_plan) and their autotuners, on a B200.

The forms of each part of the step compute the same arithmetic:
  - the two stage kernels (TMA-fed persistent tiles, or a CTA per tile with plain loads) share the
    per-point arithmetic, so their steps agree to the bit;
  - the row transforms with prefetched rows (Nx = 4096) apply the same merge, DFTs and split in
    the same order as the plain ones, compiled in other kernels (where the compiler may fuse
    other multiply-adds): dt, maxima and fields to round-off (1e-12, the wall rows to the
    Thom-gain bound);
  - the two tridiagonal forms reassociate the recurrences differently: round-off (1e-12);
  - the two max forms and the two launch forms (programmatic dependent launch or stream order)
    give the same bits.
nse2d_autotune_plan restores the state it tried the plans on (to the bit), and after
nse2d_ensemble_autotune_plans every member steps exactly as a solo channel with its plan.
"""
import numpy as np
import pytest

from test_parity_gpu import assert_fields_close, laminar_perturbed

pytestmark = pytest.mark.gpu

SMALL = dict(Nx=256, Ny=129, Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=5000.0, F0=0.05, nforce=8, lin_drag=1e-3,
             adapt=1, cfl=0.5, dt_max=1e-2)


def run_with(nse, cfg, w0, steps, **plan):
    g = nse.Solver(**cfg)
    g.set_plan(**plan)
    g.set_omega(w0)
    g.step(steps, use_graph=True)
    out = g.fields(), g.time()[:2], g.plan()
    g.close()
    return out


def test_plan_forms_agree(nse, cuda):
    w0 = laminar_perturbed(256, 129, np.tanh(2.0 * np.linspace(-1, 1, 129)) / np.tanh(2.0), seed=3, amp=5e-2)
    ref, tref, p = run_with(nse, SMALL, w0, 5, stage_tma=1, tridiag_clusters=1)
    assert p["stage_tma"] == 1
    (w, psi), t, p = run_with(nse, SMALL, w0, 5, stage_tma=0, tridiag_clusters=1)
    assert p["stage_tma"] == 0
    assert np.array_equal(w, ref[0]) and np.array_equal(psi, ref[1]) and t == tref
    (w, psi), t, p = run_with(nse, SMALL, w0, 5, stage_tma=1, tridiag_clusters=0)
    assert p["tridiag_clusters"] == 0
    assert np.max(np.abs(psi - ref[1])) <= 1e-12 * np.max(np.abs(ref[1]))
    assert np.max(np.abs(w[2:-2] - ref[0][2:-2])) <= 1e-11 * np.max(np.abs(ref[0]))


def test_rowfft_prefetch_matches_plain_at_4096(nse, cuda):
    cfg = dict(SMALL, Nx=4096, Ny=2049, Reb=2e4, nforce=12)
    y = np.tanh(2.0 * np.linspace(-1, 1, 2049)) / np.tanh(2.0)
    w0 = laminar_perturbed(4096, 2049, y, seed=5, amp=5e-2)
    (wa, pa), ta, p = run_with(nse, cfg, w0, 2, rowfft_prefetch=1)
    assert p["rowfft_prefetch"] == 1
    (wb, pb), tb, p = run_with(nse, cfg, w0, 2, rowfft_prefetch=0)
    assert p["rowfft_prefetch"] == 0
    assert np.allclose(ta, tb, rtol=1e-13, atol=0)    # t and dt after both steps
    de = np.diff(y)
    assert_fields_close(wa, pa, wb, pb, de, 1e-12)


def test_autotune_plan_restores_state(nse, cuda):
    g = nse.Solver(**SMALL)
    w0 = laminar_perturbed(256, 129, g.metric(0), seed=4, amp=5e-2)
    g.set_omega(w0)
    g.step(3)
    before, tb = g.fields(), g.time()
    best, ms = g.autotune_plan(trial_steps=4)
    assert ms > 0 and g.plan() == best
    after, ta = g.fields(), g.time()
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1]) and tb == ta
    # the context then steps as a fresh one with the same plan
    g.step(4, use_graph=True)
    h = nse.Solver(**SMALL)
    h.set_plan(**best)
    h.set_omega(w0)
    h.step(3)
    h.step(4, use_graph=True)
    assert np.array_equal(g.fields()[0], h.fields()[0])
    g.close()
    h.close()


def test_ensemble_autotune_plans_matches_solo(nse, cuda):
    grids = [(256, 129), (256, 129), (512, 257), (512, 257), (256, 257)]
    members, w0s = [], []
    for k, (Nx, Ny) in enumerate(grids):
        cfg = dict(SMALL, Nx=Nx, Ny=Ny)
        m = nse.Solver(**cfg)
        w0 = laminar_perturbed(Nx, Ny, m.metric(0), seed=10 + k, amp=5e-2)
        m.set_omega(w0)
        members.append((m, cfg))
        w0s.append(w0)
    ens = nse.Ensemble([m for m, _ in members])
    groups, ms = ens.autotune_plans(trial_steps=2)
    assert 1 <= groups <= len(grids) and ms > 0
    for (m, _), w0 in zip(members, w0s):
        m.set_omega(w0)
    ens.step(6)
    for (m, cfg), w0 in zip(members, w0s):
        h = nse.Solver(**cfg)
        h.set_plan(**m.plan())
        assert h.plan() == m.plan()
        h.set_omega(w0)
        h.step(6, use_graph=True)
        assert np.array_equal(m.fields()[0], h.fields()[0]), (cfg["Nx"], cfg["Ny"], m.plan())
        h.close()
    ens.close()
    for m, _ in members:
        m.close()


def test_switching_row_transform_form_mid_run(nse, cuda):
    """At Nx = 4096 an adaptive FP64 step with the prefetching row transforms takes its max
    reduction inside the stage-3 inverse transform, and the next step's dt from the maxima it left;
    the other form reduces at the start of the step. Switching forms between steps (the plan change
    refreshes the maxima of the current psi) gives the same dt and maxima at every step to
    round-off, and the maxima the host reads are those the last step's dt came from in either form."""
    cfg = dict(SMALL, Nx=4096, Ny=2049, Reb=2e4, nforce=12)
    y = np.tanh(2.0 * np.linspace(-1, 1, 2049)) / np.tanh(2.0)
    w0 = laminar_perturbed(4096, 2049, y, seed=8, amp=5e-2)
    a = nse.Solver(**cfg)
    a.set_plan(rowfft_prefetch=1, max_fused=1)
    assert a.plan()["max_fused"] == 1
    a.set_omega(w0)
    b = nse.Solver(**cfg)
    b.set_plan(rowfft_prefetch=1, max_fused=1)
    b.set_omega(w0)
    seq_a, seq_b = [], []
    for k, pf in enumerate((1, 0, 1, 1, 0)):
        a.step(1, use_graph=True)
        b.set_plan(rowfft_prefetch=pf, max_fused=1)
        b.step(1, use_graph=True)
        seq_a.append(a.time())
        seq_b.append(b.time())
    # t, dt, steps and the maxima of every step (maxima read a step late would differ by ~1e-4)
    assert [r[2] for r in seq_a] == [r[2] for r in seq_b]
    flat = lambda seq: np.array([(t, dt) + tuple(m) for t, dt, _, m in seq])
    assert np.allclose(flat(seq_a), flat(seq_b), rtol=1e-12, atol=0)
    (wa, pa), (wb, pb) = a.fields(), b.fields()
    assert_fields_close(wa, pa, wb, pb, np.diff(y), 1e-12)
    a.close()
    b.close()


def test_fused_max_same_bits_at_4096(nse, cuda):
    """The max reduction inside the stage-3 inverse transform evaluates the per-point maxima of the
    separate reduction, and the stage kernel's dt the same adaptive_dt: the same steps to the bit."""
    cfg = dict(SMALL, Nx=4096, Ny=2049, Reb=2e4, nforce=12)
    y = np.tanh(2.0 * np.linspace(-1, 1, 2049)) / np.tanh(2.0)
    w0 = laminar_perturbed(4096, 2049, y, seed=6, amp=5e-2)
    (wa, pa), ta, p = run_with(nse, cfg, w0, 3, rowfft_prefetch=1, max_fused=1)
    assert p["rowfft_prefetch"] == 1 and p["max_fused"] == 1
    (wb, pb), tb, p = run_with(nse, cfg, w0, 3, rowfft_prefetch=1, max_fused=0)
    assert p["rowfft_prefetch"] == 1 and p["max_fused"] == 0
    assert ta == tb
    assert np.array_equal(wa, wb) and np.array_equal(pa, pb)


@pytest.mark.parametrize("Nx,Ny,precision", [(256, 129, 64), (4096, 2049, 64), (256, 129, 32), (4096, 2049, 32)])
def test_programmatic_launch_same_bits(nse, cuda, Nx, Ny, precision):
    """With programmatic dependent launch every step kernel waits on the device for the kernel
    before it to complete before it reads or writes anything: the same steps to the bit, through
    plain launches, the one-step graph and the run graph (a WHILE node)."""
    cfg = dict(SMALL, Nx=Nx, Ny=Ny, Reb=2e4 if Nx == 4096 else SMALL["Reb"], nforce=12 if Nx == 4096 else 8)
    y = np.tanh(2.0 * np.linspace(-1, 1, Ny)) / np.tanh(2.0)
    w0 = laminar_perturbed(Nx, Ny, y, seed=9, amp=5e-2)
    out = {}
    for pdl in (1, 0):
        g = nse.Solver(precision=precision, **cfg)
        g.set_plan(pdl=pdl)
        assert g.plan()["pdl"] == pdl
        g.set_omega(w0)
        g.step(1, use_graph=False)
        g.step(2, use_graph=True)
        g.run(max_steps=3)
        out[pdl] = (g.fields(), g.time())
        g.close()
    (wa, pa), ta = out[1]
    (wb, pb), tb = out[0]
    assert ta == tb and ta[2] == 6
    assert np.array_equal(wa, wb) and np.array_equal(pa, pb)
