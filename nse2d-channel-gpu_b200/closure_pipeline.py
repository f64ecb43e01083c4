"""The learned-closure workflow on one GPU: DNS snapshots box-filtered to the coarse grid, the
closure model trained on them, and the a-posteriori comparison of the coarse solve with the
model against the DNS (the reference it is measured against, and its fallback).

Host-side orchestration only: every field operation (time steps, the Jacobians, the filter,
the velocities, training and inference) runs on the GPU through the C ABI (nse2d_b200).
Fields live in torch CUDA tensors.

Data. A DNS (2048 x 1025 by default) starts from a seeded 'mix' state: Poiseuille vorticity
plus a random perturbation over x-modes 1..64; after a spin-up, every dt_snap convective units
the state is filtered to the coarse grid (nse2d_box_filter) and the sample is
  (omega_bar, psi_bar, u_bar, v_bar, tau),  tau = filter(J(psi, omega)) - J(psi_bar, omega_bar),
with u_bar, v_bar the coarse velocities of psi_bar and J the mapped Arakawa Jacobian of each
grid (testapi_arakawa_J_mapped), tau zero on the wall rows.

A posteriori. From a DNS of a fresh seed after its spin-up, the filtered state starts two
coarse runs, with and without the model, and the DNS continues; all three run for the same
time and sample Re_tau and the mean-velocity profile every dt_stat. The closure run is
accepted when its time-averaged Re_tau and mean-velocity profile are within tol of the DNS
and it stayed finite; otherwise the workflow falls back to the plain coarse run if that one
is within tol, else to the DNS. The model's gain (and whether it acts pointwise or through
the x-mean of tau on every row) is chosen beforehand by a-posteriori runs against a
validation DNS of another seed (select_gain).
"""
import math
import time

import numpy as np

import nse2d_b200 as nse

DNS_CFG = dict(Nx=2048, Ny=1025, Lx=2 * math.pi, stretch=1, beta=2.0, Ub=1.0, Reb=1e4, F0=0.05, nforce=8,
               lin_drag=1e-3, adapt=1, cfl=0.5)


def coarse_cfg(dns_cfg, Nx=256, Ny=129):
    c = dict(dns_cfg)
    c.update(Nx=Nx, Ny=Ny)
    return c


def mix_omega(y, Nx, Lx, amp, seed, modes=64, Ub=1.0, h=1.0):
    """Poiseuille vorticity 3 Ub y / h^2 plus a seeded perturbation of amp times the wall
    vorticity over x-modes 1..modes (random amplitude, phase and wall-normal mode 1..6,
    zero at the walls)."""
    rng = np.random.default_rng(seed)
    x = np.arange(Nx) * Lx / Nx
    eta = (y - y[0]) / (y[-1] - y[0])
    w = np.repeat((3.0 * Ub * y / h ** 2)[:, None], Nx, axis=1)
    pert = np.zeros_like(w)
    for m in range(1, modes + 1):
        a, ph, ky = rng.standard_normal(), 2 * np.pi * rng.random(), int(rng.integers(1, 7))
        pert += a * np.cos(2 * np.pi * m * x / Lx + ph)[None, :] * np.sin(ky * np.pi * eta)[:, None]
    return w + amp * 3.0 * Ub / h * pert / np.sqrt(modes)


def advance_to(solver, t_target, chunk=200000):
    """Step on the device until t reaches t_target (the last dt trimmed onto it)."""
    while True:
        t = solver.time()[0]
        if t >= t_target - 1e-9 * max(1.0, abs(t_target)):
            return
        r = solver.run(next_snap=t_target, max_steps=chunk)
        if r & nse.HALT_NONFINITE:
            raise nse.Nse2dError(f"non-finite state before t = {t_target}")


class CoarseFilter:
    """Filters the state of a fine Solver onto the grid of a coarse one and forms the sample."""

    def __init__(self, torch, fine, coarse):
        self.t, self.fine, self.coarse = torch, fine, coarse
        dev = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
        self.a_f, self.a_c = dev(fine.metric(1)), dev(coarse.metric(1))
        self.fg = (1.0 / fine.scalar(1), 1.0 / fine.scalar(2))
        self.cg = (1.0 / coarse.scalar(1), 1.0 / coarse.scalar(2))
        self.Jf = torch.empty((fine.Ny, fine.Nx), dtype=torch.float64, device="cuda")
        self.Jbar = torch.empty((coarse.Ny, coarse.Nx), dtype=torch.float64, device="cuda")
        self.Jc = torch.empty_like(self.Jbar)
        self.api = nse.Testapi()

    def __call__(self, w, psi, u, v, tau):
        f, c = self.fine, self.coarse
        pw, pp = f.field_ptr(0), f.field_ptr(1)
        self.api.arakawa_J_mapped(pp, pw, self.Jf, f.Nx, f.Ny, self.fg[0], self.fg[1], self.a_f)
        nse.box_filter(pw, f.Nx, f.Ny, w, c.Nx, c.Ny)
        nse.box_filter(pp, f.Nx, f.Ny, psi, c.Nx, c.Ny)
        nse.box_filter(self.Jf, f.Nx, f.Ny, self.Jbar, c.Nx, c.Ny)
        self.api.uv_from_psi_mapped(psi, u, v, c.Nx, c.Ny, self.cg[0], self.cg[1], self.a_c)
        self.api.arakawa_J_mapped(psi, w, self.Jc, c.Nx, c.Ny, self.cg[0], self.cg[1], self.a_c)
        tau.copy_(self.Jbar - self.Jc)
        tau[0].zero_()
        tau[-1].zero_()


def generate(torch, dns_cfg=DNS_CFG, Nxc=256, Nyc=129, seed=1, t_spinup=20.0, t_span=200.0, dt_snap=0.1, log=print):
    """Snapshots [5, S, Nyc, Nxc] (omega, psi, u, v, tau) of a DNS and the GPU seconds it took."""
    dns = nse.Solver(**dns_cfg)
    coarse = nse.Solver(**coarse_cfg(dns_cfg, Nxc, Nyc))
    y = dns.metric(0)
    dns.set_omega(mix_omega(y, dns.Nx, dns_cfg["Lx"], 0.05, seed))
    flt = CoarseFilter(torch, dns, coarse)
    S = int(round(t_span / dt_snap))
    data = torch.empty((5, S, Nyc, Nxc), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    advance_to(dns, t_spinup)
    for s in range(S):
        flt(*[data[k, s] for k in range(5)])
        if s + 1 < S:
            advance_to(dns, t_spinup + (s + 1) * dt_snap)
        if log and (s + 1) % max(1, S // 10) == 0:
            log(f"  DNS t = {dns.time()[0]:.2f}, {s + 1}/{S} snapshots")
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    dns.close()
    return data, coarse.metric(0), secs


def scales_of(data, train_idx):
    """Standard deviations of omega, psi, u, v and of tau over the training samples."""
    sub = data[:, train_idx]
    s = [float(sub[k].std().item()) for k in range(5)]
    return [max(x, 1e-12) for x in s[:4]], max(s[4], 1e-12)


def train(torch, data, y, steps=2000, batch=8, lr=1e-3, weight_decay=1e-4, hidden=32, seed=0, val_frac=0.1,
          wall_rows=1, log=print):
    """Trains a Cnn on the samples (tau left out on the wall_rows rows next to each wall);
    returns it, the train/validation losses and the GPU seconds."""
    S = data.shape[1]
    rng = np.random.default_rng(seed)
    perm = rng.permutation(S)
    nval = max(1, int(round(val_frac * S)))
    val_idx, train_idx = np.sort(perm[:nval]), np.sort(perm[nval:])
    in_s, tau_s = scales_of(data, train_idx)
    net = nse.Cnn(data.shape[3], data.shape[2], y, hidden, batch)
    net.init_params(seed)
    net.set_scales(in_s, tau_s)
    net.set_application(wall_rows, 1.0, False)
    fields = [data[k] for k in range(5)]

    def val_loss():
        tot = 0.0
        for i in range(0, len(val_idx), batch):
            idx = val_idx[i:i + batch]
            tot += net.gradients(*fields, idx=idx) * len(idx)
        return tot / len(val_idx)

    hist = {"val0": val_loss(), "train": []}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(steps):
        lr_t = lr * 0.5 * (1 + math.cos(math.pi * it / steps))
        idx = rng.choice(train_idx, size=batch, replace=False)
        want = (it % 100 == 0) or it == steps - 1
        loss = net.train_step(*fields, lr_t, idx=idx, weight_decay=weight_decay, want_loss=want)
        if want:
            hist["train"].append((it, loss))
            if log and it % 500 == 0:
                log(f"  step {it}: train loss {loss:.4f}")
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    hist["val"] = val_loss()
    return net, hist, secs


def _stats_run(torch, solver, t_end, dt_stat, rows=None):
    """Steps to t_end sampling Re_tau and the mean-velocity profile every dt_stat; returns the
    samples, whether the run stayed finite, and the GPU seconds of the stepping."""
    re, prof = [], []
    t = solver.time()[0]
    n = int(round((t_end - t) / dt_stat))
    secs, finite = 0.0, True
    for s in range(n):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        try:
            advance_to(solver, t + (s + 1) * dt_stat)
        except nse.Nse2dError:
            finite = False
        torch.cuda.synchronize()
        secs += time.perf_counter() - t0
        if not finite:
            break
        d = solver.diagnostics()
        m = solver.row_moments()[0] / solver.Nx
        if not (np.isfinite(d["Re_tau"]) and np.all(np.isfinite(m))):
            finite = False
            break
        re.append(d["Re_tau"])
        prof.append(m if rows is None else m[rows])
    return np.array(re), np.array(prof), finite, secs


def reference(torch, dns_cfg=DNS_CFG, Nxc=256, Nyc=129, seed=7, t_spinup=20.0, t_span=200.0, dt_stat=0.5, log=print):
    """The DNS reference: spin-up from a fresh seed, the filtered state at its end (the coarse
    runs' initial omega), then the DNS statistics over t_span."""
    dns = nse.Solver(**dns_cfg)
    y = dns.metric(0)
    dns.set_omega(mix_omega(y, dns.Nx, dns_cfg["Lx"], 0.05, seed))
    coarse = nse.Solver(**coarse_cfg(dns_cfg, Nxc, Nyc))
    flt = CoarseFilter(torch, dns, coarse)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    advance_to(dns, t_spinup)
    torch.cuda.synchronize()
    spin = time.perf_counter() - t0
    bufs = [torch.empty((Nyc, Nxc), dtype=torch.float64, device="cuda") for _ in range(5)]
    flt(*bufs)
    w0 = bufs[0].cpu().numpy()
    t_start = dns.time()[0]
    rows = np.arange(0, dns.Ny, (dns.Ny - 1) // (Nyc - 1))
    re, prof, finite, secs = _stats_run(torch, dns, t_start + t_span, dt_stat, rows)
    if log:
        log(f"  dns: {secs:.2f} s, finite {finite}, mean Re_tau {re.mean():.2f}")
    dns.close()
    coarse.close()
    return dict(w0=w0, t_start=t_start, t_span=t_span, dt_stat=dt_stat, re_tau=re, profile=prof, finite=finite,
                gpu_s=secs, spinup_s=spin, ccfg=coarse_cfg(dns_cfg, Nxc, Nyc))


def coarse_run(torch, ref, net=None, every_stage=False, log=print, name="coarse"):
    """A coarse run from the reference's filtered state, with the model when net is given."""
    c = nse.Solver(**ref["ccfg"])
    c.set_omega(ref["w0"])               # psi of the filtered omega on the coarse grid, Thom walls
    wc, pc = c.fields()
    c.set_state(wc, pc, t=ref["t_start"])
    if net is not None:
        c.set_closure(net, every_stage=every_stage)
    re, prof, finite, secs = _stats_run(torch, c, ref["t_start"] + ref["t_span"], ref["dt_stat"])
    if log:
        log(f"  {name}: {secs:.2f} s, finite {finite}, mean Re_tau {re.mean() if len(re) else float('nan'):.2f}")
    c.close()
    return dict(re_tau=re, profile=prof, finite=finite, gpu_s=secs)


def compare(ref, run, tol=0.02):
    """Relative errors of the time-averaged Re_tau and mean-velocity profile against the DNS."""
    out = dict(run)
    if run["finite"] and len(run["re_tau"]) == len(ref["re_tau"]):
        rr = ref["re_tau"].mean()
        out["re_tau_err"] = float(abs(run["re_tau"].mean() - rr) / abs(rr))
        p, q = run["profile"].mean(axis=0), ref["profile"].mean(axis=0)
        out["profile_err"] = float(np.max(np.abs(p - q)) / np.max(np.abs(q)))
    else:
        out["re_tau_err"] = out["profile_err"] = float("inf")
    out["within_tol"] = bool(out["finite"] and out["re_tau_err"] <= tol and out["profile_err"] <= tol)
    return out


def select_gain(torch, net, ref_val, gains=(1.0, 0.5, 0.25), row_mean=True, every_stage=False, log=print):
    """The gain (and mode) of the model chosen by a-posteriori runs against a validation DNS of
    another seed: the smallest max(Re_tau error, profile error) among finite runs."""
    best = None
    for g in gains:
        net.set_application(1, g, row_mean)
        r = compare(ref_val, coarse_run(torch, ref_val, net, every_stage, None))
        score = max(r["re_tau_err"], r["profile_err"])
        if log:
            log(f"  gain {g}: Re_tau err {r['re_tau_err']:.4f}, profile err {r['profile_err']:.4f}")
        if best is None or score < best[1]:
            best = (g, score)
    net.set_application(1, best[0], row_mean)
    return best[0]


def a_posteriori(torch, net, dns_cfg=DNS_CFG, Nxc=256, Nyc=129, seed=7, t_spinup=20.0, t_span=200.0, dt_stat=0.5,
                 tol=0.02, every_stage=False, log=print):
    """DNS, coarse + closure and plain coarse runs from the same filtered state (fresh seed).
    Decision: the closure run if it is within tol of the DNS (time-averaged Re_tau and
    mean-velocity profile), else the plain coarse run if it is, else the DNS (fallback)."""
    ref = reference(torch, dns_cfg, Nxc, Nyc, seed, t_spinup, t_span, dt_stat, log)
    out = {"dns": dict(re_tau=ref["re_tau"], profile=ref["profile"], finite=ref["finite"], gpu_s=ref["gpu_s"])}
    out["closure"] = compare(ref, coarse_run(torch, ref, net, every_stage, log, "closure"), tol)
    out["coarse"] = compare(ref, coarse_run(torch, ref, None, False, log, "coarse"), tol)
    out["accepted"] = out["closure"]["within_tol"]
    out["fallback"] = "none" if out["accepted"] else ("coarse" if out["coarse"]["within_tol"] else "dns")
    out["dns_spinup_s"] = ref["spinup_s"]
    return out
