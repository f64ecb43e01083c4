#!/usr/bin/env python3
"""Benchmark: SSPRK(3,3) steps/s of the channel time step at 4096 x 2049, FP64.

Workload (the production-size plain-method configuration): Nx = 4096, Ny = 2049, Lx = 2 pi,
h = 1, tanh stretching beta = 2, Ub = 1, Re_b = 2e4, Kolmogorov forcing F0 = 0.05 at mode 12,
linear drag 1e-3, adaptive dt at CFL 0.5. Synthetic initial state: Poiseuille vorticity plus a
seeded (seed 1) random vorticity over streamwise modes 1-64 of amplitude 0.05 Ub/h, zero at
the walls (see initial_vorticity()).

One "step" = one SSPRK(3,3) step: device-side adaptive dt, three stages of (stage + forward FFT,
segmented Thomas solve, inverse FFT, Thom closure), time advance.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl ours (default): `value` = steps/s with the state resident in HBM (CUDA graph of one step
replayed K times, device events, max over ranks); `e2e` = the same metric through the public C
ABI with host buffers (initial vorticity copied from pinned host memory, every step's t/dt/max
read back to the host, final omega and psi copied back), all inside the timed region.
--impl reference: the CPU restatement of the reference algorithm (the oracle, C++/OpenMP, all
host threads) on the same configuration; the reference itself has no CPU path. Where the
reference was compiled from its sources (oracle/_ref), the line also carries
`reference_cuda_b200`: the reference's own CUDA executable timed on this GPU, beside this
project's executable in the same harness.
Under torchrun (N > 1) every rank advances its own replica (the time step does not shard):
value = steps of all ranks / max-over-ranks time.
"""
import argparse
import ctypes
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "nse2d-channel-gpu_b200")
ORACLE = os.path.join(ROOT, "oracle")

WORKLOAD = dict(Nx=4096, Ny=2049, Lx=2 * np.pi, h=1.0, stretch=1, beta=2.0, Ub=1.0, Reb=2.0e4, F0=0.05,
                nforce=12, lin_drag=1e-3, adapt=1, cfl=0.5, dt_max=1e-2, dt_init=1e-3)
METRIC = "SSPRK3 steps/s at 4096x2049 FP64"
METRIC32 = "SSPRK3 steps/s at 4096x2049 FP32-bulk"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def tanh_y(Ny, beta=2.0, h=1.0):
    e = -1.0 + 2.0 * np.arange(Ny) / (Ny - 1)
    return h * np.tanh(beta * e) / np.tanh(beta)


def initial_vorticity(Nx, Ny, Lx, y, seed=1, amp=0.05, modes=64, Ub=1.0, h=1.0):
    """Poiseuille vorticity 3 Ub y/h^2 plus sum_m A_m cos(k_m x + phi_m) sin(p_m pi (y+h)/(2h)),
    m = 1..modes, A_m ~ amp (Ub/h) N(0,1)/sqrt(modes), phi_m ~ U[0, 2 pi), p_m ~ U{1..8};
    the wall rows keep the Poiseuille value."""
    rng = np.random.default_rng(seed)
    M = min(modes, Nx // 2 - 1)
    A = amp * (Ub / h) * rng.standard_normal(M) / np.sqrt(M)
    phi = 2 * np.pi * rng.random(M)
    p = rng.integers(1, 9, size=M)
    x = np.arange(Nx) * (Lx / Nx)
    k = 2 * np.pi * np.arange(1, M + 1) / Lx
    C = A[:, None] * np.cos(k[:, None] * x[None, :] + phi[:, None])          # [M, Nx]
    S = np.sin(p[:, None] * np.pi * (y[None, :] + h) / (2 * h))               # [M, Ny]
    w = np.repeat((3.0 * Ub * y / (h * h))[:, None], Nx, axis=1) + S.T @ C
    w[0] = 3.0 * Ub * y[0] / (h * h)
    w[-1] = 3.0 * Ub * y[-1] / (h * h)
    return np.ascontiguousarray(w)


def algorithmic_bytes_per_step(Nx, Ny, real_bytes=8, spectral_bytes=None, table_bytes=None):
    """Algorithmic HBM bytes of one step (every input read once, every output written once):
    stage kernels read psi and omega^(s) (+ omega^n in stages 2, 3) and write omega^(s+1);
    each Poisson solve reads omega^(s+1), writes psi-hat and reads the elimination table cp;
    each inverse transform reads psi-hat and writes psi. The FP32-bulk variant has 4-byte fields
    and an FP32 spectral buffer (8 bytes per complex) but keeps cp (8 bytes) in FP64."""
    N, H = Nx * Ny, Nx // 2 + 1
    Rf = real_bytes
    Cf = spectral_bytes if spectral_bytes is not None else 2 * real_bytes
    Tf = table_bytes if table_bytes is not None else real_bytes
    return (Rf * N * (3 + 4 + 4) + 3 * (Rf * N + Cf * H * Ny + Tf * H * (Ny - 2)) + 3 * (Cf * H * Ny + Rf * N))


def kernel_bytes(name, stage, Nx, Ny, precision=64):
    """Algorithmic bytes of one launch of each kernel of this implementation (inputs read
    once, outputs written once); FP32-bulk kernels end in 32 (4-byte fields, 8-byte spectra),
    and the tridiagonal kernels of the FP32-bulk step read and write 8-byte spectra."""
    N, H, Ni = Nx * Ny, Nx // 2 + 1, Ny - 2
    C = 8 if precision == 32 else 16                            # bytes per spectral value
    if name.startswith("k_stage32"):                              # k_stage32, k_stage32_tma
        return 4 * N * (2 if stage == 1 else 3) + 4 * N
    if name.startswith("k_fft_fwd32"):
        return 4 * Nx * Ni + 8 * H * Ni
    if name.startswith("k_ifft_thom32"):
        return 8 * H * Ni + 4 * N + 4 * 6 * Nx
    if name == "k_maxuv32":
        return 4 * N
    if name.startswith("k_stage"):
        return 8 * N * (2 if stage == 1 else 3) + 8 * N          # psi, omega^(s) [, omega^n] -> omega^(s+1)
    if name == "k_fft_fwd":
        return 8 * Nx * Ni + 16 * H * Ni                         # omega^(s+1) rows -> omega-hat
    if name == "k_thomas_cluster":
        return C * H * Ni + 8 * H * Ni + C * H * Ny              # omega-hat and cp read, psi-hat written
    if name == "k_thomas_maps":
        return C * H * Ni + 8 * H * Ni                           # omega-hat, cp read once
    if name == "k_thomas_apply":
        return C * H * Ni                                        # psi-hat written (its re-read of
                                                                 # omega-hat and cp is not counted)
    if name == "k_ifft_thom":
        return 16 * H * Ni + 8 * N + 8 * 6 * Nx                  # psi-hat -> psi, + Thom rows
    if name == "k_maxuv_dt":
        return 8 * N
    return 0


def read_traffic(Nx, Ny, precision=64):
    """DRAM bytes (read + write) per launch of each kernel from the committed ncu summary of
    this grid and precision (lines `kernel bytes`), or {} when there is none."""
    tag = "step" if precision == 64 else "step32"
    path = os.path.join(ROOT, "profiles", f"traffic_{tag}_{Nx}x{Ny}.txt")
    out = {}
    if os.path.isfile(path):
        for ln in open(path):
            parts = ln.split()
            if len(parts) == 2 and not ln.startswith("#"):
                out[parts[0]] = int(parts[1])
    return out


def hbm_peak():
    try:
        d = json.load(open(MEASURED_PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


class NvmlClock:
    """SM clock and clock-event reasons of this process's GPU read in-process through NVML (a
    read-only query): one sample when the timed region starts, then samples every ~2 ms while
    its work runs on the device, so that even a region of a few ms has readings under load.
    The GPU is found by its UUID, since NVML numbers every GPU of the machine."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, device_index):
        self.samples, self.bits, self.h, self.nvml = [], 0, None, None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.nvml = pynvml
        except Exception:
            self.h = None

    def sample(self):
        if self.h is None:
            return
        try:
            self.samples.append(self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
            self.bits |= int(self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.h))
        except Exception:
            pass

    def poll_until(self, stream, every_s=0.002):
        """Sample until the work queued on `stream` has finished."""
        while not stream.query():
            self.sample()
            time.sleep(every_s)
        self.sample()

    def result(self):
        if self.h is None or not self.samples:
            return {"nvml_samples": 0}
        return {"nvml_sm_mhz": float(np.median(self.samples)), "nvml_sm_min_mhz": float(min(self.samples)),
                "nvml_sm_max_mhz": float(self.max_mhz), "nvml_samples": len(self.samples),
                "nvml_reasons": sorted(v for k, v in self.REASONS.items() if self.bits & k)}


def dist_setup(backend="nccl"):
    """One process per GPU under torchrun (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_* from the env).
    The ranks run independent replicas of the channel: the process group carries only the barrier
    around the timed region and the max over ranks of its time. `backend="gloo"` runs the same
    host logic on CPU ranks."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, steps, ms_max):
    """Whole-job steps/s of `world` replicas that each took `steps` steps, the slowest in ms_max."""
    return round(world * steps / (ms_max * 1e-3), 3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def fp32_accuracy(nse, W, w0, steps=200):
    """The FP32-bulk variant against FP64 from the same initial state after `steps` steps: relative
    differences of the fields and of the diagnostics K, Omega, u_tau, Re_tau, C_f and the wall
    enstrophy flux."""
    a = nse.Solver(precision=64, **W)
    b = nse.Solver(precision=32, **W)
    a.set_omega(w0)
    b.set_omega(w0)
    a.step(steps, use_graph=True)
    b.step(steps, use_graph=True)
    wa, pa = a.fields()
    wb, pb = b.fields()
    da, db = a.diagnostics(), b.diagnostics()
    out = {"steps": steps,
           "omega_rel_max": float(np.max(np.abs(wb - wa)) / np.max(np.abs(wa))),
           "psi_rel_max": float(np.max(np.abs(pb - pa)) / np.max(np.abs(pa)))}
    for k in ("K", "Omega", "utau_avg", "Re_tau", "Cf", "BOmega_wall"):
        out[k + "_rel"] = float(abs(db[k] - da[k]) / max(abs(da[k]), 1e-300))
    a.close()
    b.close()
    return out


SIX = ("K", "Omega", "utau_avg", "Re_tau", "Cf", "BOmega_wall")


def against_oracle(nse, W, w0, steps=100, dt=5e-5):
    """FP64 and FP32-bulk GPU steps against the oracle (the CPU restatement of the reference's
    FP64 algorithm) from the same initial state, at a fixed dt (the workload's viscous limit is
    5.06e-5) so that the three take the same steps: relative differences of the fields and of
    the diagnostics K, Omega, u_tau, Re_tau, C_f and the wall enstrophy flux (rows rebuilt at the
    final state in both)."""
    ora = _load("nse2d_oracle_py", os.path.join(ORACLE, "oracle.py"))
    ora.lib().or_set_threads(os.cpu_count() or 1)
    cfg = dict(W, adapt=0, dt_init=dt)
    o = ora.OracleSolver(**cfg)
    o.set_omega(w0)
    t = 0.0
    for _ in range(steps):
        o.step(t, dt)
        t += dt
    wo, po = o.fields()
    do = dict(zip(nse.DIAG_COLUMNS, o.diag_row(t, t0_row=True)))
    o.close()
    out = {"steps": steps, "dt": dt, "t": t}
    for P in (64, 32):
        g = nse.Solver(precision=P, **cfg)
        g.set_omega(w0)
        g.step(steps, use_graph=True)
        wg, pg = g.fields()
        dg = g.diagnostics(t0_row=True)
        g.close()
        r = {"omega_rel_max": float(np.max(np.abs(wg - wo)) / np.max(np.abs(wo))),
             "psi_rel_max": float(np.max(np.abs(pg - po)) / np.max(np.abs(po)))}
        for k in SIX:
            r[k + "_rel"] = float(abs(dg[k] - do[k]) / max(abs(do[k]), 1e-300))
        out[f"fp{P}"] = r
    return out


def run_ours(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    nse = _load("nse2d_b200", os.path.join(PKG, "nse2d_b200.py"))
    W = WORKLOAD
    Nx, Ny = W["Nx"], W["Ny"]
    y = tanh_y(Ny, W["beta"], W["h"])
    w0 = initial_vorticity(Nx, Ny, W["Lx"], y, seed=1 + rank)
    pinned_w0 = torch.from_numpy(w0).pin_memory()
    stream = torch.cuda.Stream()
    P = args.precision
    solver = nse.Solver(precision=P, **W)
    solver.set_omega(pinned_w0.numpy(), stream=stream)
    # the fastest kernel plan for this grid (every plan timed from this state, which is restored)
    plan, plan_ms = solver.autotune_plan(trial_steps=args.plan_trials, stream=stream) if args.plan_trials > 0 \
        else (solver.plan(), None)
    with torch.cuda.stream(stream):
        solver.step(args.warmup, use_graph=True, stream=stream)
    stream.synchronize()
    # ---- timed region (resident state): K graph replays ----
    sampler = ClockSampler(local)
    sampler.start()
    nv = NvmlClock(local)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        solver.step(args.steps, use_graph=True, stream=stream)
        e1.record(stream)
    nv.poll_until(stream)                        # NVML samples while the replays run
    stream.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    clocks.update(nv.result())
    if clocks.get("sm_mhz") is None and clocks.get("nvml_samples"):
        clocks["sm_mhz"], clocks["sm_max_mhz"] = clocks["nvml_sm_mhz"], clocks["nvml_sm_max_mhz"]
        clocks["reasons"] = clocks["nvml_reasons"]
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    t_sim, dt_last, nsteps_done, umax = solver.time(stream=stream)
    bad = solver.nonfinite(stream=stream)
    # ---- per-kernel timing pass (device events around every kernel of every step) ----
    per_kernel = solver.step_timed(args.steps, stream=stream)
    # ---- e2e through the public API with host buffers ----
    host_w = torch.empty((Ny, Nx), dtype=torch.float64).pin_memory()
    host_psi = torch.empty((Ny, Nx), dtype=torch.float64).pin_memory()
    solver2 = nse.Solver(precision=P, **W)
    solver2.set_plan(**plan)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        c0.record(stream)
        solver2.set_omega(pinned_w0.numpy(), stream=stream)
        for _ in range(args.steps):
            solver2.step(1, use_graph=True, stream=stream)
            solver2.time(stream=stream)          # per-step D2H of t, dt, step, max |u|, |v|
        solver2.lib.nse2d_get_fields(solver2.h, ctypes.c_void_p(host_w.data_ptr()),
                                     ctypes.c_void_p(host_psi.data_ptr()), 0, ctypes.c_void_p(stream.cuda_stream))
        c1.record(stream)
    stream.synchronize()
    e2e_ms = max_over_ranks(c0.elapsed_time(c1), world)
    wall_e2e = time.perf_counter() - t0
    solver2.close()
    launches = solver.launches_per_step()
    solver.close()

    accuracy = fp32_accuracy(nse, W, w0) if P == 32 else None
    vs_oracle = against_oracle(nse, W, w0) if (P == 32 and not args.no_cpu_baseline) else None
    N = Nx * Ny
    B_step = algorithmic_bytes_per_step(Nx, Ny) if P == 64 else algorithmic_bytes_per_step(Nx, Ny, 4, 8, 8)
    peak, peak_kind = hbm_peak()
    step_ms = ms_max / args.steps
    # per-kernel table; the dominant kernel carries the roofline object
    agg = {}
    stage = 0
    for name, tot in per_kernel:
        if name.startswith("k_stage"):
            stage += 1
        b = kernel_bytes(name, stage, Nx, Ny, P)
        a = agg.setdefault(name, {"launches": 0, "ms": 0.0, "bytes": 0.0})
        a["launches"] += args.steps
        a["ms"] += tot
        a["bytes"] += b * args.steps
    total_ms = sum(v["ms"] for v in agg.values())
    kernels = {}
    for name, a in agg.items():
        avg_ms = a["ms"] / a["launches"]
        gbs = (a["bytes"] / a["launches"]) / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
        kernels[name] = {"launches_per_step": a["launches"] // args.steps, "avg_us": round(avg_ms * 1e3, 2),
                         "share": round(a["ms"] / total_ms, 4), "achieved_gbs": round(gbs, 1),
                         "algorithmic_bytes_per_launch": int(a["bytes"] / a["launches"])}
    dom = max(agg, key=lambda k: agg[k]["ms"])
    dk = kernels[dom]
    traffic = read_traffic(Nx, Ny, P).get(dom)
    step_gbs = B_step / (step_ms * 1e-3) / 1e9
    h2d = N * 8 / args.steps + 8 * 3
    d2h = 2 * N * 8 / args.steps + 128
    line = {
        "metric": METRIC if P == 64 else METRIC32, "value": replica_rate(world, args.steps, ms_max),
        "unit": "steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if P == 64 else "f32 (FP64 base profiles, spectral buffer and tridiagonal solve)",
        "data": DATA,
        "config": bench_config(P, world),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": dk["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": round(dk["achieved_gbs"] / peak, 4), "traffic": traffic, "peak_kind": peak_kind},
        "step_roofline": {"algorithmic_bytes_per_step": B_step, "achieved": round(step_gbs, 1), "peak": peak,
                          "unit": "GB/s", "frac": round(step_gbs / peak, 4), "frac_of_8TBs": round(step_gbs / 8000.0, 4)},
        "kernels": kernels,
        **({"fp32_vs_fp64": accuracy, "vs_oracle": vs_oracle,
            "all_fp32_bytes_per_step": algorithmic_bytes_per_step(Nx, Ny, 4)} if P == 32 else {}),
        "e2e": {"value": replica_rate(world, args.steps, e2e_ms), "unit": "steps/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "wall_s": round(wall_e2e, 3)},
        "plan": {**plan, "tuned_ms_per_step": plan_ms,
                 "how": "nse2d_autotune_plan: every kernel plan timed over a few graph-replayed steps before "
                        "the timed region (state restored), the fastest kept"},
        "gpu_launches": int(launches * args.steps),
        "clocks": clocks,
        "sim": {"t": t_sim, "dt_last": dt_last, "steps_done": nsteps_done, "umax": umax[0], "nonfinite": bad},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, sample_steps=args.cpu_steps)
    return line


DATA = "synthetic (seeded Poiseuille + random vorticity over x-modes 1-64)"


def bench_config(precision, world):
    """The `config` object of both arms' lines (the same workload)."""
    return {"workload": f"channel SSPRK3 step 4096x2049 {'FP64' if precision == 64 else 'FP32-bulk'}, tanh beta=2, "
                        "Re_b=2e4, F0=0.05 n=12, drag 1e-3, adaptive dt CFL 0.5",
            "Nx": WORKLOAD["Nx"], "Ny": WORKLOAD["Ny"],
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (each field 67 MB, step working set ~0.5 GB)",
            "graph": "one CUDA graph per step, replayed"}


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(args, sample_steps=3, max_seconds=60.0, warmup=1, single_thread=True):
    """The oracle (C++/OpenMP CPU restatement of the reference algorithm) on the same workload."""
    ora = _load("nse2d_oracle_py", os.path.join(ORACLE, "oracle.py"))
    W = WORKLOAD
    L = ora.lib()
    threads = os.cpu_count() or 1
    L.or_set_threads(threads)
    o = ora.OracleSolver(**{k: W[k] for k in W})
    y = o.metric(0)
    o.set_omega(initial_vorticity(W["Nx"], W["Ny"], W["Lx"], y, seed=1))
    t = 0.0

    def steps(n_max, seconds):
        nonlocal t
        n, t0 = 0, time.perf_counter()
        while n < n_max and time.perf_counter() - t0 < seconds:
            dt, _ = o.adapt_dt()
            o.step(t, dt)
            t += dt
            n += 1
        return n, time.perf_counter() - t0

    steps(max(1, warmup), max_seconds)             # warm-up steps
    n, el = steps(sample_steps, max_seconds)
    cores = int(L.or_get_threads())
    out = {"value": round(n / el, 4), "unit": "steps/s", "cores": cores, "kind": "port", "cpu_model": cpu_model(),
           "host_threads": os.cpu_count(),
           "sample": f"{n} full SSPRK3 steps of the 4096x2049 workload (adaptive dt) after {max(1, warmup)} warm-up "
                     f"step(s), {cores} threads"}
    if single_thread:
        L.or_set_threads(1)
        n1, el1 = steps(1, max_seconds)
        out["single_thread"] = {"value": round(n1 / el1, 4), "unit": "steps/s", "cores": 1,
                                "sample": f"{n1} step(s) of the same run on one thread"}
        L.or_set_threads(threads)
    o.close()
    return out


def exe_step_ms(exe, steps, warm=5):
    """Median t_step_ms of the executable's --profile timing.csv (CUDA events around every step)
    on the bench workload's grid and physics, started from --init mix (the reference's executable
    has no way to take the seeded initial field); ~steps steps after the dt-limited start."""
    import tempfile
    W = WORKLOAD
    dt_est = 5.06e-5                     # the viscous limit of this grid (cvisc 0.5), which sets dt
    with tempfile.TemporaryDirectory() as out:
        cmd = [exe, "--Nx", str(W["Nx"]), "--Ny", str(W["Ny"]), "--Lx", repr(W["Lx"]), "--h", "1", "--Ub", "1",
               "--Reb", repr(W["Reb"]), "--stretch", "tanh", "--beta", repr(W["beta"]), "--F0", repr(W["F0"]),
               "--nforce", str(W["nforce"]), "--drag", repr(W["lin_drag"]), "--cfl", repr(W["cfl"]),
               "--dtmax", repr(W["dt_max"]), "--dt", repr(W["dt_init"]), "--init", "mix", "--amp", "0.05",
               "--profile", "--timeEvery", "1", "--statsEvery", "100000000", "--snap_save", "0", "--diag_save", "0",
               "--tend", repr((steps + warm) * dt_est), "--outdir", out]
        subprocess.run(cmd, check=True, capture_output=True, timeout=900)
        a = np.atleast_1d(np.genfromtxt(os.path.join(out, "timing.csv"), delimiter=",", names=True))
    ms = a["t_step_ms"][warm:] if len(a) > warm else a["t_step_ms"]
    return float(np.median(ms)), int(len(ms))


def reference_cuda(steps):
    """The reference's own CUDA solver compiled for sm_100a (oracle/_ref, by oracle/ref.mk) and this
    project's nse2d executable, timed the same way on this GPU."""
    exe = os.path.join(ORACLE, "_ref", "nse2d_ref")
    if not os.path.isfile(exe):
        return {"unavailable": "oracle/_ref/nse2d_ref was not built (the reference sources are not on this machine)"}
    ref_ms, n = exe_step_ms(exe, steps)
    ours_ms, _ = exe_step_ms(os.path.join(PKG, "nse2d"), steps)
    return {"value": round(1e3 / ref_ms, 3), "unit": "steps/s", "ms_per_step": round(ref_ms, 4), "steps": n,
            "ours_same_harness": {"value": round(1e3 / ours_ms, 3), "ms_per_step": round(ours_ms, 4)},
            "how": "median t_step_ms of each executable's --profile timing.csv (CUDA events around each "
                   "step; the reference's includes its three blocking max-reduction copies, ours the "
                   "per-kernel events of a profiled step) at 4096x2049, --init mix, after 5 steps"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    steps = max(1, min(args.steps, args.ref_steps))
    cb = cpu_baseline(args, sample_steps=steps, max_seconds=args.ref_seconds, warmup=min(args.warmup, 5))
    extra = {}
    if args.ref_cuda_steps > 0:
        try:
            extra["reference_cuda_b200"] = reference_cuda(args.ref_cuda_steps)
        except Exception as e:                                         # informational only
            extra["reference_cuda_b200"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    return {**extra, "metric": METRIC, "value": cb["value"], "unit": "steps/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 / cb["value"], 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA, "config": bench_config(64, world),
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


ENSEMBLE_SEED = 20261203


def ensemble_members(n=64, seed=ENSEMBLE_SEED):
    """The 64-channel ensemble workload: (Nx, Ny) uniform on {256, 512, 1024} x {129, 257, 513},
    Re_b log-uniform on [2e3, 2e4], forcing mode in {4, 8, 12}; initial seeds 100 + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(dict(Nx=int(rng.choice([256, 512, 1024])), Ny=int(rng.choice([129, 257, 513])),
                        Reb=float(np.exp(rng.uniform(np.log(2e3), np.log(2e4)))), nforce=int(rng.choice([4, 8, 12])),
                        seed=100 + i))
    return out


def run_ensemble(args):
    """64 channels advanced by one graph launch per K steps (nse2d_ensemble, branch count chosen
    by its autotuner) against the same 64 channels stepped one after another (each its own
    graph replay). Metric: grid-point updates per second, sum_i Nx_i Ny_i K / time."""
    import torch
    nse = _load("nse2d_b200", os.path.join(PKG, "nse2d_b200.py"))
    spec = ensemble_members()

    def build():
        sol = []
        for m in spec:
            W = dict(Lx=2 * np.pi, h=1.0, stretch=1, beta=2.0, Ub=1.0, F0=0.05, lin_drag=1e-3, adapt=1, cfl=0.5,
                     dt_max=1e-2, dt_init=1e-3, Nx=m["Nx"], Ny=m["Ny"], Reb=m["Reb"], nforce=m["nforce"])
            s = nse.Solver(precision=args.precision, **W)
            s.set_omega(initial_vorticity(m["Nx"], m["Ny"], W["Lx"], tanh_y(m["Ny"]), seed=m["seed"]))
            sol.append(s)
        return sol

    K = args.steps
    pts = sum(m["Nx"] * m["Ny"] for m in spec)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    members = build()
    ens = nse.Ensemble(members)
    groups, _ = ens.autotune_plans(trial_steps=3, stream=stream)
    plans = {}
    for m, sm in zip(spec, members):
        plans.setdefault(f"{m['Nx']}x{m['Ny']}", sm.plan())
    ens.step(args.warmup, stream=stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    a.record(stream)
    ens.step(K, stream=stream)
    b.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    ens_ms = a.elapsed_time(b)
    ens.close()
    seq = build()
    for m, s in zip(spec, seq):
        s.set_plan(**plans[f"{m['Nx']}x{m['Ny']}"])
        s.step(args.warmup, use_graph=True, stream=stream)
    torch.cuda.synchronize()
    a.record(stream)
    for s in seq:
        s.step(K, use_graph=True, stream=stream)
    b.record(stream)
    torch.cuda.synchronize()
    seq_ms = a.elapsed_time(b)
    for s in members + seq:
        s.close()
    prec = "FP64" if args.precision == 64 else "FP32-bulk"
    return {"metric": f"ensemble grid-point updates/s (64 channels, configuration 3, {prec})",
            "value": round(pts * K / (ens_ms * 1e-3), 1), "unit": "points/s", "n_gpus": 1, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(ens_ms / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == 64 else "f32 bulk (FP64 base profiles, FP64 tridiagonal arithmetic and table)",
            "data": "synthetic (seeded laminar + random modes per member)", "plans": plans,
            "config": {"workload": "64 channels, (Nx,Ny) on {256,512,1024}x{129,257,513}, Re_b log-uniform "
                                   "[2e3,2e4], nforce {4,8,12}, tanh beta=2, adaptive dt", "members": len(spec),
                       "points": pts, "master_seed": ENSEMBLE_SEED, "branches": groups},
            "sequential": {"value": round(pts * K / (seq_ms * 1e-3), 1), "unit": "points/s",
                           "ms_per_step": round(seq_ms / K, 4),
                           "how": "the same 64 channels with the same plans, each replaying its own one-step graph "
                                  "K times, one after another"},
            "speedup_vs_sequential": round(seq_ms / ens_ms, 3), "clocks": ck}


def run_closure(args):
    """The learned-closure workflow (closure_pipeline): a 2048x1025 FP64 DNS (Re_b=1e4, tanh
    beta=2, F0=0.05 at n=8, drag 1e-3, seeded mix) filtered to 256x129 every 0.1 units; the
    4-layer BF16 CNN trained on it with AdamW; its gain chosen against a validation DNS (seed 5);
    then, from the filtered state of a fresh seed (7), the DNS, the coarse solve with the model
    and the plain coarse solve over the same span. Metric: DNS GPU seconds / GPU seconds of the
    accepted coarse solve (the closure run if within 2% of the DNS on the time-averaged Re_tau
    and mean-velocity profile, else the plain coarse run if it is, else 1: the DNS itself)."""
    import torch
    sys.path.insert(0, PKG)
    nse = _load("nse2d_b200", os.path.join(PKG, "nse2d_b200.py"))
    cp = _load("closure_pipeline", os.path.join(PKG, "closure_pipeline.py"))
    log = lambda m: print(m, file=sys.stderr, flush=True)
    T = args.closure_span
    data, y, gen_s = cp.generate(torch, cp.DNS_CFG, seed=1, t_spinup=args.closure_spinup, t_span=T, dt_snap=0.1, log=log)
    net, hist, train_s = cp.train(torch, data, y, steps=args.closure_train_steps, batch=8, lr=1e-3, hidden=32, seed=0,
                                  log=log)
    ref_val = cp.reference(torch, cp.DNS_CFG, seed=5, t_spinup=args.closure_spinup, t_span=args.closure_val_span,
                           dt_stat=0.5, log=log)
    gain = cp.select_gain(torch, net, ref_val, log=log)
    out = cp.a_posteriori(torch, net, cp.DNS_CFG, seed=7, t_spinup=args.closure_spinup, t_span=T, dt_stat=0.5, log=log)
    dns_s = out["dns"]["gpu_s"]
    acc = {"none": "closure", "coarse": "coarse", "dns": "dns"}[out["fallback"]]
    acc_s = dns_s if acc == "dns" else out[acc]["gpu_s"]

    def brief(r):
        return {"gpu_s": round(r["gpu_s"], 3), "finite": r["finite"], "re_tau": round(float(np.mean(r["re_tau"])), 3),
                "re_tau_err": round(r.get("re_tau_err", 0.0), 5), "profile_err": round(r.get("profile_err", 0.0), 5)}
    return {
        "metric": "closure vs DNS time at 2% Re_tau", "value": round(dns_s / acc_s, 2), "unit": "x (DNS GPU s / accepted coarse GPU s)",
        "higher_is_better": True, "n_gpus": 1, "steps": args.closure_train_steps, "warmup": 0, "scaling": "none",
        "vs_baseline": None, "dtype": "bf16 model (FP32 accumulate), FP64 solver", "data": "self-generated DNS",
        "accepted": acc, "gain": gain, "model_mode": "x-mean of tau on every row",
        "a_priori": {"val_loss_untrained": round(hist["val0"], 4), "val_loss": round(hist["val"], 4),
                     "note": "loss normalised by the variance of tau: predicting tau = 0 scores ~1"},
        "dns": brief(out["dns"]), "closure": brief(out["closure"]), "coarse": brief(out["coarse"]),
        "gpu_seconds": {"data_generation": round(gen_s, 2), "training": round(train_s, 2),
                        "validation_dns": round(ref_val["gpu_s"], 2)},
        "config": {"workload": f"learned closure: DNS 2048x1025 -> 256x129, span {T} units after {args.closure_spinup} "
                               f"of spin-up, snapshots every 0.1, {args.closure_train_steps} AdamW steps of batch 8",
                   "Re_b": 1e4, "seeds": {"train": 1, "validation": 5, "test": 7}},
    }


def profile_steps(args):
    """A short, untimed run of the workload for profilers: initial solve, then K plain steps
    (no graph), so that every kernel launch is visible separately."""
    import torch
    nse = _load("nse2d_b200", os.path.join(PKG, "nse2d_b200.py"))
    W = dict(WORKLOAD)
    if args.nx:
        W["Nx"], W["Ny"] = args.nx, args.ny
    y = tanh_y(W["Ny"], W["beta"], W["h"])
    s = nse.Solver(precision=args.precision, **W)
    if args.plan:
        s.set_plan(**{k: int(v) for k, v in (kv.split("=") for kv in args.plan.split(","))})
    s.set_omega(initial_vorticity(W["Nx"], W["Ny"], W["Lx"], y, seed=1))
    s.step(args.profile_steps, use_graph=False)
    torch.cuda.synchronize()
    t, dt, n, m = s.time()
    print(json.dumps({"profile_steps": n, "t": t, "dt": dt, "umax": m[0], "nonfinite": s.nonfinite(), "plan": s.plan()}))
    s.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="untimed run of K plain steps for a profiler (no JSON bench line)")
    ap.add_argument("--plan", default="",
                    help="profile runs: kernel forms as key=value pairs, e.g. rowfft_prefetch=1,max_fused=0")
    ap.add_argument("--nx", type=int, default=0)
    ap.add_argument("--ny", type=int, default=0)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--ref-steps", type=int, default=20)
    ap.add_argument("--ref-seconds", type=float, default=120.0)
    ap.add_argument("--ref-cuda-steps", type=int, default=40,
                    help="reference arm: also time the reference's CUDA build (oracle/_ref) for K steps (0: off)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plan-trials", type=int, default=20,
                    help="steps per candidate of the kernel-plan autotuner before the timed region (0: default plan)")
    ap.add_argument("--precision", type=int, choices=[64, 32], default=64,
                    help="32: the FP32-bulk variant (its own metric line)")
    ap.add_argument("--workload", choices=["channel", "ensemble", "closure"], default="channel",
                    help="ensemble: the 64-channel batched ensemble; closure: the learned-closure workflow "
                         "(each its own JSON line, 1 GPU)")
    ap.add_argument("--closure-span", type=float, default=200.0,
                    help="closure: convective units of data and of the test runs (200: the specified configuration, "
                         "about 15 minutes on one B200)")
    ap.add_argument("--closure-val-span", type=float, default=50.0)
    ap.add_argument("--closure-spinup", type=float, default=20.0)
    ap.add_argument("--closure-train-steps", type=int, default=2000)
    args = ap.parse_args()
    if args.profile_steps > 0:
        profile_steps(args)
        return
    if args.workload == "ensemble":
        print(json.dumps(run_ensemble(args)))
        return
    if args.workload == "closure":
        print(json.dumps(run_closure(args)))
        return
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup() if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                    int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        line = run_reference(args, world, rank)
    else:
        line = run_ours(args, world, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if args.impl == "ours" and world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
