"""Batched ensembles (nse2d_ensemble_*) on a B200: one graph launch advances every member, and the
result of each member equals that member stepped alone, to the bit, whatever the grouping of the
members into concurrent branches. Ensemble members take the two-pass tridiagonal solve, so the
solo runs they are compared with do too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(Nx=128, Ny=65, Reb=2000.0, nforce=4),
    dict(Nx=256, Ny=129, Reb=5000.0, nforce=8),
    dict(Nx=64, Ny=33, Reb=3000.0, nforce=12),
    dict(Nx=128, Ny=129, Reb=8000.0, nforce=4, stretch=0, beta=0.0),
    dict(Nx=512, Ny=257, Reb=20000.0, nforce=12),
]


def make(nse, m, seed):
    cfg = dict(Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, F0=0.05, lin_drag=1e-3, adapt=1, cfl=0.5)
    cfg.update(m)
    s = nse.Solver(**cfg)
    y = s.metric(0)
    rng = np.random.default_rng(seed)
    w = np.repeat((3.0 * y)[:, None], s.Nx, axis=1)
    x = np.arange(s.Nx) * (2 * np.pi / s.Nx)
    for k in range(1, 7):
        w += 0.05 * rng.standard_normal() * np.cos(k * x + rng.random() * 6.28)[None, :] * \
            np.sin(rng.integers(1, 5) * np.pi * (y + 1) / 2)[:, None]
    w[0], w[-1] = 3.0 * y[0], 3.0 * y[-1]
    s.set_omega(w)
    return s


def test_ensemble_matches_solo_runs(nse, cuda):
    ens_m = [make(nse, m, 10 + i) for i, m in enumerate(MEMBERS)]
    solo = [make(nse, m, 10 + i) for i, m in enumerate(MEMBERS)]
    for s in solo:
        s.set_tridiag_form(False)
    e = nse.Ensemble(ens_m)
    groups, ms = e.autotune(trial_steps=2)
    assert 1 <= groups <= len(MEMBERS) and ms > 0
    ncand = len([g for g in (1, 2, 4) if g < len(MEMBERS)]) + 1
    e.step(7)
    for s in solo:
        s.step(ncand * 3 + 7, use_graph=True)
    for a, b in zip(ens_m, solo):
        wa, pa = a.fields()
        wb, pb = b.fields()
        assert np.array_equal(wa, wb) and np.array_equal(pa, pb)
        assert a.time()[:3] == b.time()[:3]
    # another grouping, same results
    e.set_groups(2)
    e.step(3)
    for s in solo:
        s.step(3, use_graph=True)
    for a, b in zip(ens_m, solo):
        assert np.array_equal(a.fields()[0], b.fields()[0])
    e.close()


def test_tridiag_forms_agree(nse, cuda):
    """The cluster and the two-pass tridiagonal solves of the same channel agree to round-off, and
    switching the form between steps (the step graph is captured again) keeps stepping."""
    m = MEMBERS[4]
    a, b = make(nse, m, 3), make(nse, m, 3)
    b.set_tridiag_form(False)
    a.step(5, use_graph=True)
    b.step(5, use_graph=True)
    wa, pa = a.fields()
    wb, pb = b.fields()
    assert np.max(np.abs(pa - pb)) <= 1e-12 * np.max(np.abs(pa))
    assert np.max(np.abs(wa[2:-2] - wb[2:-2])) <= 1e-10 * np.max(np.abs(wa))
    b.set_tridiag_form(True)
    b.step(2, use_graph=True)
    a.step(2, use_graph=True)
    assert np.max(np.abs(a.fields()[1] - b.fields()[1])) <= 1e-12 * np.max(np.abs(pa))
    a.close()
    b.close()
