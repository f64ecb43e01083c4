"""nse2d_max_uv_noalloc (a context-free max |u|, |v|, |v| a that allocates no device memory)
against the context entry point nse2d_max_uv, through the C ABI on a B200.

Both run the same reduction kernel over the same psi; maxima do not depend on the order in
which the partials are folded, so the results agree to the bit. The tolerance (1e-15
relative) leaves one ulp. Each case calls the no-alloc entry point twice in a row, since
its scratch is reused from call to call and must be cleared in between, and checks that the
device's free memory does not change across those calls.

The entry point takes any Nx >= 2 and any 8-byte-aligned psi: sizes that are not a multiple of
two, and a psi that starts 8 bytes past a 16-byte boundary, use the kernel's 8-byte-load form.
Those cases are checked against the per-point maxima computed with numpy from the same psi.
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


def _numpy_max_uv(psi, a_node, inv_dx, inv_deta):
    """max |u|, |v|, |v| a with u = a (psi_{j+1} - psi_{j-1}) inv_deta / 2 and
    v = (psi_{i+1} - psi_{i-1}) inv_dx / 2 (periodic in x), over the interior rows, evaluated
    in the kernel's order: the difference times 0.5 inv first, then times a."""
    cy, cx = 0.5 * inv_deta, 0.5 * inv_dx
    a = a_node[1:-1, None]
    dy = np.abs(psi[2:] - psi[:-2])
    dxd = np.abs(np.roll(psi, -1, axis=1) - np.roll(psi, 1, axis=1))[1:-1]
    return (a * (dy * cy)).max(), (dxd * cx).max(), ((dxd * cx) * a).max()


@pytest.mark.parametrize("Nx,Ny,offset", [(2, 3, 0), (5, 7, 0), (6, 9, 1), (7, 4, 1), (1030, 11, 0), (1031, 12, 1),
                                          (600, 40, 1), (4096, 23, 1)])
def test_max_uv_noalloc_any_nx_and_offset(nse, cuda, Nx, Ny, offset):
    """Odd and non-power-of-two Nx, and psi at an 8-byte (not 16-byte) aligned address."""
    torch = cuda
    rng = np.random.default_rng(Nx * 31 + Ny)
    psi = rng.standard_normal((Ny, Nx))
    a_node = rng.uniform(0.5, 2.0, Ny)
    inv_dx, inv_deta = 3.0, 0.7
    buf = torch.zeros(Ny * Nx + 2, dtype=torch.float64, device="cuda")
    assert buf.data_ptr() % 16 == 0
    buf[offset:offset + Ny * Nx] = torch.from_numpy(psi.ravel()).to("cuda")
    d_a = torch.tensor(a_node, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    got = np.array(nse.max_uv_noalloc(buf.data_ptr() + 8 * offset, d_a, Nx, Ny, inv_dx, inv_deta))
    exp = np.array(_numpy_max_uv(psi, a_node, inv_dx, inv_deta))
    np.testing.assert_array_equal(got, exp)


def test_max_uv_noalloc_rejects_unaligned_pointer(nse, cuda):
    torch = cuda
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(nse.Nse2dError, match="8-byte aligned"):
        nse.max_uv_noalloc(buf.data_ptr() + 4, buf, 4, 4, 1.0, 1.0)
