"""Host logic of bench.py that needs no GPU: the byte models behind the roofline numbers and
the traffic table it reads from the committed ncu summaries."""
import importlib.util
import os

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_bytes", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_step_byte_models():
    b = _bench()
    # FP64 step: 8-byte fields, 16-byte spectra, 8-byte elimination table
    assert b.algorithmic_bytes_per_step(4096, 2049) == 1_645_117_512
    # FP32 bulk: 4-byte fields, FP64 spectra and table
    assert b.algorithmic_bytes_per_step(4096, 2049, 4, 16, 8) == 1_074_413_640
    # the all-FP32 count
    assert b.algorithmic_bytes_per_step(4096, 2049, 4) == 822_558_756


def test_kernel_byte_models():
    b = _bench()
    Nx, Ny = 4096, 2049
    N, H, Ni = Nx * Ny, Nx // 2 + 1, Ny - 2
    # stage kernels: psi and omega^(s) in (+ omega^n in stages 2 and 3), omega^(s+1) out
    for name in ("k_stage_tma", "k_stage"):
        assert b.kernel_bytes(name, 1, Nx, Ny) == 24 * N
        assert b.kernel_bytes(name, 2, Nx, Ny) == 32 * N
    # the FP32 stage kernels (both the TMA and the plain one) count 4-byte fields
    for name in ("k_stage32_tma", "k_stage32"):
        assert b.kernel_bytes(name, 1, Nx, Ny) == 12 * N
        assert b.kernel_bytes(name, 3, Nx, Ny) == 16 * N
    assert b.kernel_bytes("k_fft_fwd", 1, Nx, Ny) == 8 * Nx * Ni + 16 * H * Ni
    # the FP32-bulk step's spectra are FP32 (8 bytes per complex value), its cp table FP64
    assert b.kernel_bytes("k_fft_fwd32", 1, Nx, Ny, 32) == 4 * Nx * Ni + 8 * H * Ni
    assert b.kernel_bytes("k_ifft_thom32", 1, Nx, Ny, 32) == 8 * H * Ni + 4 * N + 24 * Nx
    assert b.kernel_bytes("k_thomas_cluster", 1, Nx, Ny) == 16 * H * Ni + 8 * H * Ni + 16 * H * Ny
    assert b.kernel_bytes("k_thomas_cluster", 1, Nx, Ny, 32) == 8 * H * Ni + 8 * H * Ni + 8 * H * Ny
    assert b.kernel_bytes("k_ifft_thom", 1, Nx, Ny) == 16 * H * Ni + 8 * N + 48 * Nx
    assert b.kernel_bytes("k_maxuv_dt", 0, Nx, Ny) == 8 * N
    assert b.kernel_bytes("k_maxuv32", 0, Nx, Ny) == 4 * N
    assert b.kernel_bytes("k_unknown", 0, Nx, Ny) == 0


def test_traffic_tables_cover_the_step_kernels():
    b = _bench()
    t64 = b.read_traffic(4096, 2049, 64)
    t32 = b.read_traffic(4096, 2049, 32)
    for k in ("k_maxuv_dt", "k_stage_tma", "k_fft_fwd", "k_thomas_cluster", "k_ifft_thom"):
        assert t64.get(k, 0) > 0, k
    for k in ("k_maxuv32", "k_stage32_tma", "k_fft_fwd32", "k_thomas_cluster", "k_ifft_thom32"):
        assert t32.get(k, 0) > 0, k
    assert b.read_traffic(64, 33, 64) == {}
