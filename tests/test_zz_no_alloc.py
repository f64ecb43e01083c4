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

A psi holding NaN must be reported (status NSE2D_STATUS_NONFINITE): the maxima skip NaN, so the
returned values alone would not show it. In a fresh process, the first call may make CUDA place
the library's code and the static scratch on the device (CUDA loads kernels on first use); that
one-time change of free device memory is bounded, and the calls after it change nothing.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG

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


def test_max_uv_noalloc_reports_nan(nse, cuda):
    """NaN in psi: status NSE2D_STATUS_NONFINITE (an error from the Python mirror), then a clean
    psi on the same scratch gives the numpy maxima again (the flag does not stick)."""
    torch = cuda
    Nx, Ny = 256, 65
    rng = np.random.default_rng(3)
    psi = rng.standard_normal((Ny, Nx))
    a_node = rng.uniform(0.5, 2.0, Ny)
    d_psi = torch.tensor(psi, dtype=torch.float64, device="cuda")
    d_a = torch.tensor(a_node, dtype=torch.float64, device="cuda")
    d_psi[Ny // 2, 17] = float("nan")
    torch.cuda.synchronize()
    assert nse.STATUS_NONFINITE == 2
    with pytest.raises(nse.Nse2dError, match="NaN or Inf"):
        nse.max_uv_noalloc(d_psi, d_a, Nx, Ny, 3.0, 0.7)
    d_psi[Ny // 2, 17] = float(psi[Ny // 2, 17])
    torch.cuda.synchronize()
    got = np.array(nse.max_uv_noalloc(d_psi, d_a, Nx, Ny, 3.0, 0.7))
    np.testing.assert_array_equal(got, np.array(_numpy_max_uv(psi, a_node, 3.0, 0.7)))


_FRESH = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import nse2d_b200 as nse
Nx, Ny = 1024, 513
rng = np.random.default_rng(11)
psi = torch.tensor(rng.standard_normal((Ny, Nx)), dtype=torch.float64, device="cuda")
a = torch.tensor(rng.uniform(0.5, 2.0, Ny), dtype=torch.float64, device="cuda")
torch.cuda.synchronize()
f0 = torch.cuda.mem_get_info()[0]
r1 = nse.max_uv_noalloc(psi, a, Nx, Ny, 3.0, 0.7)
f1 = torch.cuda.mem_get_info()[0]
r2 = nse.max_uv_noalloc(psi, a, Nx, Ny, 3.0, 0.7)
r3 = nse.max_uv_noalloc(psi, a, Nx, Ny, 3.0, 0.7)
f2 = torch.cuda.mem_get_info()[0]
print(json.dumps(dict(f0=f0, f1=f1, f2=f2, r=[list(r1), list(r2), list(r3)])))
"""


def test_max_uv_noalloc_first_call_in_fresh_process(cuda):
    """Free device memory across the first call of a fresh process (where CUDA may place this
    library's code and the static scratch on the device, once) and across the calls after it."""
    p = subprocess.run([sys.executable, "-c", _FRESH, PKG], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    d = json.loads(p.stdout.strip().splitlines()[-1])
    first = d["f0"] - d["f1"]
    print(f"free device memory: first call {first} bytes, later calls {d['f1'] - d['f2']} bytes")
    assert 0 <= first <= 16 << 20, first          # a one-time placement of code and scratch
    assert d["f2"] == d["f1"], (d["f1"], d["f2"])  # no change at all after the first call
    assert d["r"][0] == d["r"][1] == d["r"][2]
