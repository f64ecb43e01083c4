"""The reference's C++ driver-side API as this library exports it (include/nse2d/*.hpp), on a B200.

1. Every operator and diagnostic launcher of the reference's src/ops.cuh:12-81 and
   src/diag.cuh:12-113, called in this library and in the reference's own build
   (oracle/_ref/libnse2d_ref.so, compiled from its sources) through the same C++ symbol, on the
   same device inputs: fields equal to 1e-13 of their maximum (the same formulas up to FMA
   contraction), sums to 1e-12 relative (both add CTA partials with atomics, in different orders),
   maxima and row moments to 1e-13.
2. A driver written against the headers in the shape of the reference's time loop
   (tests/compat_driver.cu: build_y_metrics, Poisson2D_Z2Z, the launchers, adaptive dt), compiled
   with nvcc and linked with libnse2d_b200.so alone: after 10 adaptive steps of a forced tanh
   channel its fields match this library's own step (nse2d_step) to 1e-11 (the wall rows to the
   Thom-gain bound of the parity tests), and its diagnostic sums match the reference's launchers on
   the same final state.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ORACLE, PKG, ROOT
from test_parity_gpu import assert_fields_close, laminar_perturbed

pytestmark = pytest.mark.gpu

REF_LIB = os.path.join(ORACLE, "_ref", "libnse2d_ref.so")
need_ref = pytest.mark.skipif(not os.path.isfile(REF_LIB), reason="the reference was not compiled here")


def cpp_symbols(path):
    """{function name: mangled symbol} of the C++ functions a shared library defines."""
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    syms = {}
    for ln in out.splitlines():
        parts = ln.split()
        if len(parts) == 3 and parts[1] == "T" and parts[2].startswith("_Z") and parts[2][2:3].isdigit():
            m = parts[2]                                # a global function (not a nested name, _ZN...)
            k = 2
            while m[k].isdigit():
                k += 1
            n = int(m[2:k])
            syms.setdefault(m[k:k + n], m)
    return syms


def bind(path):
    lib = ctypes.CDLL(path)
    syms = cpp_symbols(path)

    def fn(name):
        f = getattr(lib, syms[name])
        f.restype = None
        return f
    return fn


P = lambda t: ctypes.c_void_p(t.data_ptr())   # noqa: E731
D = ctypes.c_double
I = ctypes.c_int


@need_ref
def test_launchers_match_reference(nse, cuda):
    torch = cuda
    ours, ref = bind(os.path.join(PKG, "libnse2d_b200.so")), bind(REF_LIB)
    Nx, Ny = 128, 97
    g = nse.Solver(Nx=Nx, Ny=Ny, Lx=2 * np.pi, stretch=1, beta=2.0)
    met = {k: torch.tensor(g.metric(i), dtype=torch.float64, device="cuda")
           for i, k in enumerate(["y", "a_node", "a_edge", "dy_edge", "w_node"])}
    wt = torch.zeros(Ny, dtype=torch.float64, device="cuda")
    wt[1:-1] = g.scalar(2) / met["a_node"][1:-1]
    dx, deta = g.scalar(1), g.scalar(2)
    idx, ide = 1.0 / dx, 1.0 / deta
    gen = torch.Generator(device="cuda").manual_seed(11)
    psi, w, rhs, u, v = (torch.randn(Ny, Nx, dtype=torch.float64, device="cuda", generator=gen) for _ in range(5))
    N = Nx * Ny

    def field_case(call):
        a = [torch.zeros(Ny, Nx, dtype=torch.float64, device="cuda") for _ in range(3)]
        b = [torch.zeros(Ny, Nx, dtype=torch.float64, device="cuda") for _ in range(3)]
        call(ours, a)
        call(ref, b)
        torch.cuda.synchronize()
        for x, y in zip(a, b):
            assert float((x - y).abs().max()) <= 1e-13 * max(float(y.abs().max()), 1e-300)

    field_case(lambda L, o: L("launch_laplacian_fd_mapped")(P(w), P(o[0]), I(Nx), I(Ny), D(idx ** 2), D(ide ** 2),
                                                           P(met["a_node"]), P(met["a_edge"]), None))
    field_case(lambda L, o: L("launch_rhs_mapped")(P(u), P(v), P(w), P(o[0]), I(Nx), I(Ny), D(1e-3), D(0.05), I(12),
                                                   D(1.0), D(1e-3), P(met["y"]), None))

    def mms(L, o):
        o[0].copy_(rhs)
        L("launch_mms_add_forcing")(P(o[0]), I(Nx), I(Ny), D(2 * np.pi), D(1.0), D(0.3), D(1e-2), D(1e-3), D(1.0),
                                    D(0.1), D(1.0), I(2), P(met["y"]), None)
    field_case(mms)
    field_case(lambda L, o: L("launch_axpy")(P(o[0]), P(w), P(rhs), D(0.01), ctypes.c_size_t(N), None))
    field_case(lambda L, o: L("launch_ssprk2")(P(o[0]), P(w), P(u), P(rhs), D(0.01), ctypes.c_size_t(N), None))
    field_case(lambda L, o: L("launch_ssprk3")(P(o[0]), P(w), P(u), P(rhs), D(0.01), ctypes.c_size_t(N), None))
    field_case(lambda L, o: L("launch_uv_from_psi_mapped")(P(psi), P(o[0]), P(o[1]), I(Nx), I(Ny), D(idx), D(ide),
                                                           P(met["a_node"]), None))
    field_case(lambda L, o: L("launch_arakawa_J_mapped")(P(psi), P(w), P(o[0]), I(Nx), I(Ny), D(idx), D(ide),
                                                         P(met["a_node"]), None))

    def thom(L, o):
        o[0].copy_(w)
        L("launch_thom_wall_vorticity_mapped")(P(o[0]), P(psi), I(Nx), I(Ny), P(met["dy_edge"]), D(0.0), D(2.0), None)
    field_case(thom)

    def interior(L, o):
        L("launch_omega_from_psi_interior_mapped")(P(o[0]), P(psi), I(Nx), I(Ny), D(idx ** 2), D(ide ** 2),
                                                   P(met["a_node"]), P(met["a_edge"]), None)
        o[0][0].zero_()
        o[0][-1].zero_()
    field_case(interior)

    # reductions into device scalars / rows
    def sums(call, n, tol=1e-12):
        a = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
        b = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
        call(ours, a)
        call(ref, b)
        torch.cuda.synchronize()
        # relative to the largest value of the output (row sums of u, v come out near zero)
        scale = max(float(b.abs().max()), 1e-300)
        assert float((a - b).abs().max()) <= tol * scale, (a.tolist(), b.tolist())

    def at(t, k):
        return ctypes.c_void_p(t.data_ptr() + 8 * k)
    an, ae, wn, yy = P(met["a_node"]), P(met["a_edge"]), P(met["w_node"]), P(met["y"])
    sums(lambda L, o: L("launch_enstrophy_diss_mapped")(P(w), I(Nx), I(Ny), D(idx), D(ide), an, wn, at(o, 0), at(o, 1),
                                                        None), 2)
    sums(lambda L, o: L("launch_enstrophy_diss_mapped_full")(P(w), I(Nx), I(Ny), D(idx), D(ide), an, wn, at(o, 0),
                                                             at(o, 1), None), 2)
    sums(lambda L, o: L("launch_enstrophy_sbp_mapped")(P(w), I(Nx), I(Ny), D(idx), D(ide), ae, P(wt), at(o, 0),
                                                       at(o, 1), None), 2)
    sums(lambda L, o: L("launch_kinetic_energy_mapped")(P(psi), I(Nx), I(Ny), D(idx), D(ide), an, wn, at(o, 0), None), 1)
    sums(lambda L, o: L("launch_energy_dissipation_mapped")(P(psi), P(w), I(Nx), I(Ny), D(idx), D(ide), an, ae, wn,
                                                            at(o, 0), None), 1)
    sums(lambda L, o: L("launch_power_input_mapped")(P(psi), I(Nx), I(Ny), D(ide), D(1.0), D(0.05), I(12), an, yy, wn,
                                                     at(o, 0), None), 1)
    sums(lambda L, o: L("launch_enstrophy_input_mapped_full")(P(w), I(Nx), I(Ny), D(1.0), D(0.05), I(12), yy, wn,
                                                              at(o, 0), None), 1)
    sums(lambda L, o: L("launch_enstrophy_input_mapped")(P(w), I(Nx), I(Ny), D(1.0), D(0.05), I(12), yy, wn, at(o, 0),
                                                         None), 1)
    sums(lambda L, o: L("launch_enstrophy_diss_balance_mapped")(P(w), I(Nx), I(Ny), D(idx ** 2), D(ide ** 2), an, ae,
                                                                wn, at(o, 0), at(o, 1), None), 2)
    sums(lambda L, o: L("launch_omega_rhs_balance_mapped")(P(w), P(rhs), I(Nx), I(Ny), wn, at(o, 0), None), 1)
    sums(lambda L, o: L("launch_mean_wall_omega")(P(w), I(Nx), I(Ny), at(o, 0), at(o, 1), None), 2, 1e-13)
    sums(lambda L, o: L("launch_mean_wall_omega_omegay_mapped")(P(w), I(Nx), I(Ny), D(ide), an, at(o, 0), at(o, 1),
                                                                None), 2, 1e-13)
    sums(lambda L, o: L("launch_max_uv_from_psi_mapped")(P(psi), I(Nx), I(Ny), D(idx), D(ide), an, at(o, 0), at(o, 1),
                                                         at(o, 2), None), 3, 0.0)
    sums(lambda L, o: L("launch_row_moments_from_psi_mapped")(P(psi), I(Nx), I(Ny), D(idx), D(ide), an, at(o, 0),
                                                              at(o, Ny), at(o, 2 * Ny), at(o, 3 * Ny), at(o, 4 * Ny),
                                                              None), 5 * Ny, 1e-12)
    g.close()


def test_cpp_driver_against_the_step(nse, cuda, tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "compat_driver"
    subprocess.run([nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "compat_driver.cu"), "-L", PKG,
                    "-lnse2d_b200", "-Xlinker", "-rpath", "-Xlinker", PKG, "-o", str(exe)], check=True,
                   capture_output=True, timeout=600)
    Nx, Ny, Lx, beta, Reb, F0, nf, drag, steps = 256, 129, 2 * np.pi, 2.0, 5000.0, 0.05, 8, 1e-3, 10
    g = nse.Solver(Nx=Nx, Ny=Ny, Lx=Lx, stretch=1, beta=beta, Ub=1.0, Reb=Reb, F0=F0, nforce=nf, lin_drag=drag,
                   adapt=1, cfl=0.5, dt_max=1e-2)
    w0 = laminar_perturbed(Nx, Ny, g.metric(0), seed=9, amp=5e-2)
    w0.tofile(tmp_path / "w0.bin")
    subprocess.run([str(exe), str(tmp_path / "w0.bin"), str(tmp_path / "out.bin"), str(Nx), str(Ny), repr(Lx),
                    repr(beta), repr(Reb), repr(F0), str(nf), repr(drag), str(steps)], check=True, capture_output=True,
                   timeout=300)
    out = np.fromfile(tmp_path / "out.bin")
    wd, pd = out[:Nx * Ny].reshape(Ny, Nx), out[Nx * Ny:2 * Nx * Ny].reshape(Ny, Nx)
    t_d, sums_d = out[2 * Nx * Ny], out[2 * Nx * Ny + 1:]
    g.set_omega(w0)
    g.step(steps)
    wg, pg = g.fields()
    assert abs(g.time()[0] - t_d) <= 1e-12 * t_d
    assert_fields_close(wg, pg, wd, pd, g.metric(3), 1e-11)
    # the driver's diagnostic sums of its final state against the reference's launchers on it
    if os.path.isfile(REF_LIB):
        torch = cuda
        ref = bind(REF_LIB)
        met = {k: torch.tensor(g.metric(i), dtype=torch.float64, device="cuda")
               for i, k in enumerate(["y", "a_node", "a_edge", "dy_edge", "w_node"])}
        wt, pt = torch.from_numpy(wd).cuda(), torch.from_numpy(pd).cuda()
        o = torch.zeros(6, dtype=torch.float64, device="cuda")
        at = lambda k: ctypes.c_void_p(o.data_ptr() + 8 * k)   # noqa: E731
        idx, ide = 1.0 / g.scalar(1), 1.0 / g.scalar(2)
        an, ae, wn, yy = P(met["a_node"]), P(met["a_edge"]), P(met["w_node"]), P(met["y"])
        ref("launch_kinetic_energy_mapped")(P(pt), I(Nx), I(Ny), D(idx), D(ide), an, wn, at(0), None)
        ref("launch_enstrophy_diss_mapped")(P(wt), I(Nx), I(Ny), D(idx), D(ide), an, wn, at(1), at(2), None)
        ref("launch_energy_dissipation_mapped")(P(pt), P(wt), I(Nx), I(Ny), D(idx), D(ide), an, ae, wn, at(3), None)
        ref("launch_power_input_mapped")(P(pt), I(Nx), I(Ny), D(ide), D(1.0), D(F0), I(nf), an, yy, wn, at(4), None)
        ref("launch_enstrophy_input_mapped_full")(P(wt), I(Nx), I(Ny), D(1.0), D(F0), I(nf), yy, wn, at(5), None)
        torch.cuda.synchronize()
        np.testing.assert_allclose(sums_d, o.cpu().numpy(), rtol=1e-12, atol=0)
    g.close()
