"""nse2d_max_uv_noalloc (a context-free max |u|, |v|, |v| a that allocates no device memory)
against the context entry point nse2d_max_uv, through the C ABI on a B200.

Both run the same reduction kernel over the same psi; maxima do not depend on the order in
which the partials are folded, so the results agree to the bit. The tolerance (1e-15
relative) leaves one ulp. Each case calls the no-alloc entry point twice in a row, since
its scratch is reused from call to call and must be cleared in between, and checks that the
device's free memory does not change across those calls.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    dict(Nx=256, Ny=257, stretch=1, beta=2.0),      # fewer interior rows than CTAs at 4 per SM
    dict(Nx=4096, Ny=2049, stretch=1, beta=2.0),    # CTAs stride over the rows
    dict(Nx=64, Ny=33, stretch=0, beta=0.0),
]


def _omega(Nx, Ny, y, seed):
    rng = np.random.default_rng(seed)
    w = np.repeat((3.0 * y)[:, None], Nx, axis=1)
    w += 1e-2 * rng.standard_normal((Ny, Nx))
    return w


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['Nx']}x{c['Ny']}")
def test_max_uv_noalloc_matches_context(nse, cuda, case):
    torch = cuda
    g = nse.Solver(Lx=2.0 * np.pi, Ub=1.0, Reb=500.0, **case)
    Nx, Ny = g.Nx, g.Ny
    y, a_node = g.metric(0), g.metric(1)
    g.set_omega(_omega(Nx, Ny, y, seed=Nx + Ny))
    ref = np.array(g.max_uv())
    assert np.all(np.isfinite(ref)) and ref[0] > 0

    # the caller's own device buffers: psi of the context, a_node copied by the test
    psi_ptr = g.field_ptr(1)
    d_a_node = torch.tensor(a_node, dtype=torch.float64, device="cuda")
    dx, deta = g.scalar(1), g.scalar(2)
    torch.cuda.synchronize()

    first = np.array(nse.max_uv_noalloc(psi_ptr, d_a_node, Nx, Ny, 1.0 / dx, 1.0 / deta))
    free_before = torch.cuda.mem_get_info()[0]
    second = np.array(nse.max_uv_noalloc(psi_ptr, d_a_node, Nx, Ny, 1.0 / dx, 1.0 / deta))
    third = np.array(nse.max_uv_noalloc(psi_ptr, d_a_node, Nx, Ny, 1.0 / dx, 1.0 / deta))
    free_after = torch.cuda.mem_get_info()[0]

    for r in (first, second, third):
        np.testing.assert_allclose(r, ref, rtol=1e-15, atol=0.0)
    assert free_after == free_before, (free_before, free_after)
    g.close()


def test_max_uv_noalloc_rejects_bad_sizes(nse, cuda):
    torch = cuda
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(nse.Nse2dError, match="too small"):
        nse.max_uv_noalloc(buf, buf, 8, 2, 1.0, 1.0)
    with pytest.raises(nse.Nse2dError, match="exceeds the maximum"):
        nse.max_uv_noalloc(buf, buf, (1 << 30) + 1, 8, 1.0, 1.0)
