"""The C ABI library on the CPU: it loads and exports every function include/nse2d.h declares
(no compute calls: there is no GPU here), and the reference's seven test-API symbols are there
with the reference's names (src/test_api.cu:8-92)."""
import ctypes
import os

from conftest import PKG, ROOT

REFERENCE_TESTAPI = ["testapi_uv_from_psi_mapped", "testapi_omega_from_psi_interior_mapped",
                     "testapi_thom_wall_vorticity_mapped", "testapi_arakawa_J_mapped",
                     "testapi_compute_adv_from_uv_mapped", "testapi_compute_adv_flux_mapped",
                     "testapi_arakawa_J_mapped_split"]


def test_library_exports_header(nse):
    lib = nse.load()
    names = nse.header_functions(os.path.join(ROOT, "include", "nse2d.h"))
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    for n in REFERENCE_TESTAPI:
        assert n in names


def test_config_defaults_match_reference(nse):
    cfg = nse.default_config()
    # src/common.cuh:42-114 defaults
    assert (cfg.Nx, cfg.Ny) == (1024, 1025)
    assert cfg.Lx == 12.566370612 and cfg.h == 1.0
    assert cfg.Ub == 1.0 and cfg.Reb == 10000.0 and cfg.nu_override == -1.0
    assert (cfg.dt_init, cfg.dt_max, cfg.cfl, cfg.cvisc) == (1e-3, 1e-2, 0.5, 0.5)
    assert cfg.adapt == 1 and cfg.t_end == 200.0 and cfg.nforce == 1
    assert (cfg.mms_A0, cfg.mms_eps, cfg.mms_Om, cfg.mms_kx) == (1e-3, 0.1, 1.0, 1)
    assert ctypes.sizeof(cfg) > 0


def test_bad_config_fails_loudly(nse):
    """Invalid grids are rejected with a message, before any device work."""
    import pytest
    with pytest.raises(nse.Nse2dError, match="power of two"):
        nse.Solver(Nx=100, Ny=65)
    with pytest.raises(nse.Nse2dError, match="Ny"):
        nse.Solver(Nx=64, Ny=4)
    assert os.path.isfile(os.path.join(PKG, "libnse2d_b200.so"))
