"""Python mirror of the nse2d-b200 C ABI (include/nse2d.h), over ctypes.

This is the host-side interface a Python user (and the tests and bench.py) calls. It binds
libnse2d_b200.so, built in this directory by `make`; there is no fallback: if the library
or a CUDA device is missing, loading fails with an error.

Two layers, as in the C header:
  * the reference's C-linkage operator launchers (src/test_api.cu of the reference), which
    take device pointers; `Testapi` wraps them for torch CUDA tensors;
  * `Solver`, the status-returning solver-context API: the whole SSPRK(3,3) step of the
    reference time loop (src/main.cu:434-541), its Poisson solve and its diagnostics.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnse2d_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "nse2d.h")

DIAG_COLUMNS = ["umax", "vmax", "K", "Omega", "dOmega_rhs", "eta", "BOmega_wall", "Pin", "epsilon", "POmega",
                "tauw_bot", "tauw_top", "dpdx", "utau_avg", "Cf", "Re_tau",
                "dOmega_rhs_same", "dOmega_rhs_same_int", "Omega_int", "eta_int", "Jwall_s1_cum", "Jwall_s2_cum",
                "Jwall_s3_cum", "Omega_int_w", "dOmega_same_int_w", "A_w", "P_int_w", "eta_h", "Phi_h"]


class Nse2dError(RuntimeError):
    pass


class Config(ctypes.Structure):
    """struct nse2d_config: the reference's Grid + Params (src/common.cuh:42-114)."""
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Lx", ctypes.c_double), ("h", ctypes.c_double),
                ("stretch", ctypes.c_int), ("beta", ctypes.c_double), ("Ub", ctypes.c_double),
                ("Reb", ctypes.c_double), ("nu_override", ctypes.c_double), ("dt_init", ctypes.c_double),
                ("dt_max", ctypes.c_double), ("cfl", ctypes.c_double), ("cvisc", ctypes.c_double),
                ("adapt", ctypes.c_int), ("t_end", ctypes.c_double), ("F0", ctypes.c_double),
                ("nforce", ctypes.c_int), ("lin_drag", ctypes.c_double), ("free_slip", ctypes.c_int),
                ("mms", ctypes.c_int), ("mms_A0", ctypes.c_double), ("mms_eps", ctypes.c_double),
                ("mms_Om", ctypes.c_double), ("mms_kx", ctypes.c_int), ("closure_diag", ctypes.c_int),
                ("precision", ctypes.c_int), ("y_table", ctypes.c_void_p)]


class Plan(ctypes.Structure):
    """struct nse2d_plan: the kernel forms of a context's step."""
    _fields_ = [("stage_tma", ctypes.c_int), ("tridiag_clusters", ctypes.c_int), ("rowfft_prefetch", ctypes.c_int),
                ("max_fused", ctypes.c_int), ("pdl", ctypes.c_int)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class SnapshotMeta(ctypes.Structure):
    """struct nse2d_snapshot_meta: the grid and the scalar attributes of a snapshot file."""
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("t", ctypes.c_double), ("Lx", ctypes.c_double),
                ("h", ctypes.c_double), ("nu", ctypes.c_double), ("beta", ctypes.c_double),
                ("stretch_tanh", ctypes.c_int), ("y", ctypes.c_void_p), ("fields", ctypes.c_int)]


_lib = None


def header_functions(path=HEADER):
    """Names of the functions declared in include/nse2d.h."""
    import re
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(?:void|int|const char\*)\s+\**(\w+)\s*\(", txt)))


def load(path=LIB_PATH):
    """Load libnse2d_b200.so and declare the signatures. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(path):
        raise Nse2dError(f"{path} is missing: build it with `make -C {HERE}` (nvcc, sm_100a)")
    lib = ctypes.CDLL(path)
    P, I, D, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, None
    sig = {
        "nse2d_config_default": (V, [ctypes.POINTER(Config)]),
        "nse2d_create": (I, [ctypes.POINTER(Config), ctypes.POINTER(P)]),
        "nse2d_destroy": (I, [P]),
        "nse2d_set_omega": (I, [P, P, I, P]),
        "nse2d_set_state": (I, [P, P, P, I, D, P]),
        "nse2d_get_fields": (I, [P, P, P, I, P]),
        "nse2d_field_ptr": (I, [P, I, ctypes.POINTER(P)]),
        "nse2d_get_field": (I, [P, I, P, P]),
        "nse2d_step": (I, [P, I, I, P]),
        "nse2d_set_tridiag_form": (I, [P, I]),
        "nse2d_step_store_rhs": (I, [P, I, P]),
        "nse2d_launches_per_step": (I, [P]),
        "nse2d_step_timed": (I, [P, I, P, P]),
        "nse2d_step_kernel_name": (ctypes.c_char_p, [P, I]),
        "nse2d_step_profiled": (I, [P, P, P, P, P]),
        "nse2d_ensemble_create": (I, [P, I, ctypes.POINTER(P)]),
        "nse2d_ensemble_destroy": (I, [P]),
        "nse2d_ensemble_step": (I, [P, I, P]),
        "nse2d_ensemble_set_groups": (I, [P, I]),
        "nse2d_ensemble_autotune": (I, [P, I, P, P, P]),
        "nse2d_set_dt": (I, [P, D, P]),
        "nse2d_set_schedule": (I, [P, D, D, P]),
        "nse2d_get_time": (I, [P, P, P, P, P, P]),
        "nse2d_poisson_solve": (I, [P, P, P, P]),
        "nse2d_max_uv": (I, [P, P, P]),
        "nse2d_run": (I, [P, D, D, I, D, ctypes.c_longlong, P, P]),
        "nse2d_row_moments": (I, [P, P, P]),
        "nse2d_spectra_accumulate": (I, [P, P]),
        "nse2d_stats_device": (I, [P, I, P]),
        "nse2d_get_plan": (I, [P, ctypes.POINTER(Plan)]),
        "nse2d_set_plan": (I, [P, ctypes.POINTER(Plan)]),
        "nse2d_autotune_plan": (I, [P, I, ctypes.POINTER(Plan), P, P]),
        "nse2d_ensemble_autotune_plans": (I, [P, I, P, P, P]),
        "nse2d_stats_read": (I, [P, P, P, P]),
        "nse2d_spectra": (I, [P, P, P, P, P, P]),
        "nse2d_max_uv_noalloc": (I, [P, P, I, I, D, D, P, P]),
        "nse2d_diagnostics": (I, [P, I, P, P]),
        "nse2d_rhs_at_state": (I, [P, D, P]),
        "nse2d_uv": (I, [P, P, P, P]),
        "nse2d_nonfinite": (I, [P, P, P]),
        "nse2d_metrics": (I, [P, I, P]),
        "nse2d_scalar": (I, [P, I, P]),
        "nse2d_gemm_bf16": (I, [P, P, P, P, P, I, I, I, I, I, P]),
        "nse2d_box_filter": (I, [P, I, I, P, I, I, P]),
        "nse2d_cnn_create": (I, [I, I, I, I, P, ctypes.POINTER(P)]),
        "nse2d_cnn_destroy": (I, [P]),
        "nse2d_cnn_layer_shape": (I, [P, I, P, P]),
        "nse2d_cnn_set_params": (I, [P, I, P, P]),
        "nse2d_cnn_get_params": (I, [P, I, P, P]),
        "nse2d_cnn_get_grads": (I, [P, I, P, P]),
        "nse2d_cnn_set_scales": (I, [P, P, D]),
        "nse2d_cnn_set_application": (I, [P, I, D, I]),
        "nse2d_cnn_forward": (I, [P, P, P, P, P, P, P]),
        "nse2d_cnn_gradients": (I, [P, P, P, P, P, P, P, I, P, P]),
        "nse2d_cnn_train_step": (I, [P, P, P, P, P, P, P, I, ctypes.c_float, ctypes.c_float, P, P]),
        "nse2d_set_closure": (I, [P, P, I]),
        "nse2d_snapshot_write": (I, [ctypes.c_char_p, I, ctypes.POINTER(SnapshotMeta), I, P, P]),
        "nse2d_snapshot_read": (I, [ctypes.c_char_p, ctypes.POINTER(SnapshotMeta), ctypes.c_char_p, P]),
        "nse2d_last_error": (ctypes.c_char_p, []),
        "nse2d_set_abort_on_error": (V, [I]),
        "nse2d_testapi_set_free_slip": (V, [I]),
        "testapi_uv_from_psi_mapped": (V, [P, P, P, I, I, D, D, P, P]),
        "testapi_omega_from_psi_interior_mapped": (V, [P, P, I, I, D, D, P, P, P]),
        "testapi_thom_wall_vorticity_mapped": (V, [P, P, I, I, P, D, D, P]),
        "testapi_arakawa_J_mapped": (V, [P, P, P, I, I, D, D, P, P]),
        "testapi_compute_adv_from_uv_mapped": (V, [P, P, P, P, I, I, D, D, P, P]),
        "testapi_compute_adv_flux_mapped": (V, [P, P, P, P, I, I, D, D, P, P]),
        "testapi_arakawa_J_mapped_split": (V, [P, P, P, P, P, P, I, I, D, D, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


HALT_OUTPUT, HALT_STATS, HALT_END, HALT_NONFINITE, HALT_BUDGET = 1, 2, 4, 8, 16
STATUS_NONFINITE = 2          # nse2d_max_uv_noalloc: psi holds NaN or Inf


def _check(rc):
    if rc != 0:
        raise Nse2dError(load().nse2d_last_error().decode())


def default_config(**kw):
    cfg = Config()
    load().nse2d_config_default(ctypes.byref(cfg))
    for k, v in kw.items():
        if k == "stretch" and isinstance(v, str):
            v = {"none": 0, "uniform": 0, "tanh": 1, "table": 2}[v]
        if k == "y_table":
            # kept alive with the Config: nse2d_create copies it
            cfg._y_table = np.ascontiguousarray(v, dtype=np.float64)
            v = cfg._y_table.ctypes.data
        setattr(cfg, k, v)
    return cfg


def _ptr(a):
    """Device or host address of a torch tensor or a numpy array."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def _stream(s):
    if s is None:
        return None
    if hasattr(s, "cuda_stream"):
        return ctypes.c_void_p(s.cuda_stream)
    return ctypes.c_void_p(int(s))


def max_uv_noalloc(psi_dev, a_node_dev, Nx, Ny, inv_dx, inv_deta, stream=None):
    """max |u|, |v|, |v| a of a caller-owned psi [Ny, Nx] and a_node [Ny] (CUDA float64)
    through nse2d_max_uv_noalloc, which allocates no device memory. psi_dev and a_node_dev may
    also be raw device addresses (int), such as Solver.field_ptr returns. Raises Nse2dError when
    the arguments are rejected or psi holds NaN or Inf."""
    def dev(a):
        return ctypes.c_void_p(a) if isinstance(a, int) else _ptr(a)
    out = (ctypes.c_double * 3)()
    _check(load().nse2d_max_uv_noalloc(dev(psi_dev), dev(a_node_dev), int(Nx), int(Ny), float(inv_dx),
                                       float(inv_deta), out, _stream(stream)))
    return tuple(out)


def write_snapshot(path, fields, t, Lx, h, nu, beta=0.0, y=None, fmt="h5"):
    """Write a snapshot file: fields = {name: [Ny, Nx] float64 array} (omega, psi, u, v), in the
    reference's HDF5 layout (fmt "h5") or the flat bin layout ("bin"); y (with beta > 0) marks a
    tanh grid and is stored with its attributes."""
    names = list(fields)
    arrs = [np.ascontiguousarray(fields[k], dtype=np.float64) for k in names]
    Ny, Nx = arrs[0].shape
    m = SnapshotMeta(Nx=Nx, Ny=Ny, t=t, Lx=Lx, h=h, nu=nu, beta=beta, stretch_tanh=1 if y is not None else 0)
    yy = None
    if y is not None:
        yy = np.ascontiguousarray(y, dtype=np.float64)
        m.y = yy.ctypes.data
    cn = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
    cf = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    _check(load().nse2d_snapshot_write(str(path).encode(), 0 if fmt == "h5" else 1, ctypes.byref(m), len(names),
                                       ctypes.cast(cn, ctypes.c_void_p), ctypes.cast(cf, ctypes.c_void_p)))


def read_snapshot(path):
    """(meta dict, {name: array}) of a snapshot file of either format: every field present, [Ny, Nx],
    and y when stored."""
    m = SnapshotMeta()
    L = load()
    _check(L.nse2d_snapshot_read(str(path).encode(), ctypes.byref(m), None, None))
    meta = {k: getattr(m, k) for k in ("Nx", "Ny", "t", "Lx", "h", "nu", "beta", "stretch_tanh")}
    out = {}
    for bit, name in ((1, "omega"), (2, "psi"), (4, "u"), (8, "v"), (16, "y")):
        if m.fields & bit:
            a = np.empty(m.Ny if name == "y" else (m.Ny, m.Nx))
            _check(L.nse2d_snapshot_read(str(path).encode(), None, name.encode(), a.ctypes.data_as(ctypes.c_void_p)))
            out[name] = a
    return meta, out


def gemm_bf16(A, B, bias=None, relu=False, out_f32=True, out_bf16=False, stream=None):
    """C = A . B^T (+ bias) on the tensor cores (nse2d_gemm_bf16): A [M, K] and B [N, K] torch
    bfloat16 CUDA tensors (contiguous), FP32 accumulate. Returns (C_f32 or None, act(C)_bf16 or
    None), where act is ReLU when relu is set."""
    import torch
    M, K = A.shape
    N = B.shape[0]
    Cf = torch.empty((M, N), dtype=torch.float32, device=A.device) if out_f32 else None
    Cb = torch.empty((M, N), dtype=torch.bfloat16, device=A.device) if out_bf16 else None
    _check(load().nse2d_gemm_bf16(_ptr(A), _ptr(B), _ptr(bias), _ptr(Cf), _ptr(Cb), int(M), int(N), int(K), int(N),
                                  1 if relu else 0, _stream(stream)))
    return Cf, Cb


def box_filter(fine, Nxf, Nyf, coarse, Nxc, Nyc, stream=None):
    """nse2d_box_filter on device buffers (torch CUDA float64 tensors or raw addresses)."""
    def dev(a):
        return ctypes.c_void_p(a) if isinstance(a, int) else _ptr(a)
    _check(load().nse2d_box_filter(dev(fine), int(Nxf), int(Nyf), dev(coarse), int(Nxc), int(Nyc), _stream(stream)))


class Cnn:
    """The learned closure model (nse2d_cnn_*): BF16 3x3 convolutions on the tensor cores.
    Inputs (omega, psi, u, v) are torch CUDA float64 tensors, one field [Ny, Nx] or samples
    [S, Ny, Nx] with batch indices."""

    def __init__(self, Nx, Ny, y, hidden=32, max_batch=1):
        self.lib = load()
        y = np.ascontiguousarray(y, dtype=np.float64)
        h = ctypes.c_void_p()
        _check(self.lib.nse2d_cnn_create(int(Nx), int(Ny), int(hidden), int(max_batch), _ptr(y), ctypes.byref(h)))
        self.h, self.Nx, self.Ny, self.hidden, self.max_batch = h, Nx, Ny, hidden, max_batch
        self.layers = 4

    def close(self):
        if getattr(self, "h", None):
            self.lib.nse2d_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, layer):
        ci, co = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.nse2d_cnn_layer_shape(self.h, int(layer), ctypes.byref(ci), ctypes.byref(co)))
        return ci.value, co.value

    def set_params(self, layer, w, b):
        ci, co = self.shape(layer)
        w = np.ascontiguousarray(w, dtype=np.float32).reshape(co, 9, ci)
        b = np.ascontiguousarray(b, dtype=np.float32).reshape(co)
        _check(self.lib.nse2d_cnn_set_params(self.h, int(layer), _ptr(w), _ptr(b)))

    def _get(self, fn, layer):
        ci, co = self.shape(layer)
        w = np.zeros((co, 9, ci), np.float32)
        b = np.zeros(co, np.float32)
        _check(fn(self.h, int(layer), _ptr(w), _ptr(b)))
        return w, b

    def get_params(self, layer):
        return self._get(self.lib.nse2d_cnn_get_params, layer)

    def get_grads(self, layer):
        return self._get(self.lib.nse2d_cnn_get_grads, layer)

    def params(self):
        return [self.get_params(l) for l in range(self.layers)]

    def load_params(self, params):
        for l, (w, b) in enumerate(params):
            self.set_params(l, w, b)

    def init_params(self, seed=0, last_gain=0.1):
        """He-uniform weights (bound sqrt(6 / fan_in)), zero biases, from a numpy generator; the
        output layer scaled by last_gain."""
        rng = np.random.default_rng(seed)
        for layer in range(self.layers):
            ci, co = self.shape(layer)
            bound = np.sqrt(6.0 / (9 * ci)) * (last_gain if layer == self.layers - 1 else 1.0)
            self.set_params(layer, rng.uniform(-bound, bound, (co, 9, ci)).astype(np.float32), np.zeros(co, np.float32))

    def set_scales(self, in_scales, tau_scale):
        s = np.ascontiguousarray(in_scales, dtype=np.float64)
        _check(self.lib.nse2d_cnn_set_scales(self.h, _ptr(s), float(tau_scale)))
        self.scales = (tuple(float(x) for x in s), float(tau_scale))

    def set_application(self, wall_rows=1, gain=1.0, row_mean=False):
        """tau = 0 on the wall_rows rows next to each wall (loss and output); output times gain;
        row_mean: every output row replaced by its x-mean."""
        _check(self.lib.nse2d_cnn_set_application(self.h, int(wall_rows), float(gain), 1 if row_mean else 0))

    def forward(self, w, psi, u, v, tau, stream=None):
        _check(self.lib.nse2d_cnn_forward(self.h, _ptr(w), _ptr(psi), _ptr(u), _ptr(v), _ptr(tau), _stream(stream)))

    def gradients(self, w, psi, u, v, tau, idx=(0,), stream=None):
        loss = ctypes.c_float()
        ix = np.ascontiguousarray(idx, dtype=np.int32)
        _check(self.lib.nse2d_cnn_gradients(self.h, _ptr(w), _ptr(psi), _ptr(u), _ptr(v), _ptr(tau), _ptr(ix), len(ix),
                                            ctypes.byref(loss), _stream(stream)))
        return loss.value

    def train_step(self, w, psi, u, v, tau, lr, idx=(0,), weight_decay=0.0, want_loss=True, stream=None):
        loss = ctypes.c_float()
        ix = np.ascontiguousarray(idx, dtype=np.int32)
        _check(self.lib.nse2d_cnn_train_step(self.h, _ptr(w), _ptr(psi), _ptr(u), _ptr(v), _ptr(tau), _ptr(ix), len(ix),
                                             float(lr), float(weight_decay), ctypes.byref(loss) if want_loss else None,
                                             _stream(stream)))
        return loss.value if want_loss else None


class Solver:
    """One channel on one GPU: the reference time loop's state and operators."""

    def __init__(self, cfg=None, **kw):
        self.lib = load()
        self.cfg = cfg if cfg is not None else default_config(**kw)
        h = ctypes.c_void_p()
        _check(self.lib.nse2d_create(ctypes.byref(self.cfg), ctypes.byref(h)))
        self.h = h
        self.Nx, self.Ny = self.cfg.Nx, self.cfg.Ny

    def close(self):
        if getattr(self, "h", None):
            self.lib.nse2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state ----
    def set_closure(self, cnn, every_stage=True):
        """Attach a closure model (Cnn of this grid): evaluated before every stage, or once per
        step and held over its stages; None detaches it."""
        _check(self.lib.nse2d_set_closure(self.h, cnn.h if cnn is not None else None, 1 if every_stage else 0))
        self._closure = cnn

    def set_omega(self, w, stream=None):
        """omega (host numpy [Ny,Nx] or CUDA tensor) -> initial Poisson solve + Thom, t = 0."""
        if hasattr(w, "data_ptr"):
            _check(self.lib.nse2d_set_omega(self.h, _ptr(w), 1, _stream(stream)))
        else:
            w = np.ascontiguousarray(w, dtype=np.float64)
            assert w.size == self.Nx * self.Ny
            _check(self.lib.nse2d_set_omega(self.h, _ptr(w), 0, _stream(stream)))

    def set_state(self, w, psi, t=0.0, stream=None):
        w = np.ascontiguousarray(w, dtype=np.float64)
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        _check(self.lib.nse2d_set_state(self.h, _ptr(w), _ptr(psi), 0, float(t), _stream(stream)))

    def fields(self, stream=None):
        w = np.empty((self.Ny, self.Nx))
        psi = np.empty((self.Ny, self.Nx))
        _check(self.lib.nse2d_get_fields(self.h, _ptr(w), _ptr(psi), 0, _stream(stream)))
        return w, psi

    def field_ptr(self, which):
        p = ctypes.c_void_p()
        _check(self.lib.nse2d_field_ptr(self.h, which, ctypes.byref(p)))
        return p.value

    # ---- time stepping ----
    def step(self, nsteps=1, use_graph=False, stream=None):
        _check(self.lib.nse2d_step(self.h, int(nsteps), 1 if use_graph else 0, _stream(stream)))

    def set_tridiag_form(self, clusters):
        """True: the one-pass cluster tridiagonal solve (the default where it fits); False: the
        two-pass form, which shares the device with concurrent work (ensemble members use it)."""
        _check(self.lib.nse2d_set_tridiag_form(self.h, 1 if clusters else 0))

    def plan(self):
        """The kernel forms in use: {stage_tma, tridiag_clusters, rowfft_prefetch, max_fused, pdl}."""
        pl = Plan()
        _check(self.lib.nse2d_get_plan(self.h, ctypes.byref(pl)))
        return pl.as_dict()

    def set_plan(self, stage_tma=None, tridiag_clusters=None, rowfft_prefetch=None, max_fused=None, pdl=None):
        """Select kernel forms (None keeps the current one, as nse2d_get_plan reports it); forms the
        grid cannot use fall back."""
        cur = self.plan()
        pl = Plan(**{k: int(v if v is not None else cur[k]) for k, v in
                     (("stage_tma", stage_tma), ("tridiag_clusters", tridiag_clusters),
                      ("rowfft_prefetch", rowfft_prefetch), ("max_fused", max_fused), ("pdl", pdl))})
        _check(self.lib.nse2d_set_plan(self.h, ctypes.byref(pl)))

    def autotune_plan(self, trial_steps=10, stream=None):
        """Time every plan the context can use (the state is restored) and keep the fastest;
        returns (plan dict, ms per step)."""
        pl, ms = Plan(), ctypes.c_double()
        _check(self.lib.nse2d_autotune_plan(self.h, int(trial_steps), ctypes.byref(pl), ctypes.byref(ms),
                                            _stream(stream)))
        return pl.as_dict(), ms.value

    def step_store_rhs(self, nsteps=1, stream=None):
        _check(self.lib.nse2d_step_store_rhs(self.h, int(nsteps), _stream(stream)))

    def step_timed(self, nsteps, stream=None):
        """nsteps steps with per-kernel CUDA events; returns [(kernel name, total ms)] in launch order."""
        nk = self.launches_per_step()
        out = (ctypes.c_double * nk)()
        _check(self.lib.nse2d_step_timed(self.h, int(nsteps), out, _stream(stream)))
        return [(self.lib.nse2d_step_kernel_name(self.h, k).decode(), out[k]) for k in range(nk)]

    def launches_per_step(self):
        return self.lib.nse2d_launches_per_step(self.h)

    def set_dt(self, dt, stream=None):
        _check(self.lib.nse2d_set_dt(self.h, float(dt), _stream(stream)))

    def set_schedule(self, next_snap=1e300, next_diag=1e300, stream=None):
        _check(self.lib.nse2d_set_schedule(self.h, float(next_snap), float(next_diag), _stream(stream)))

    def time(self, stream=None):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        um = (ctypes.c_double * 3)()
        _check(self.lib.nse2d_get_time(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st), um,
                                       _stream(stream)))
        return t.value, dt.value, st.value, tuple(um)

    def nonfinite(self, stream=None):
        """Flags since the state was last set: bit 0 a max reduction met NaN/Inf in psi, bit 1
        a bounded wait of a kernel timed out (0: neither)."""
        f = ctypes.c_int()
        _check(self.lib.nse2d_nonfinite(self.h, ctypes.byref(f), _stream(stream)))
        return int(f.value)

    # ---- operators ----
    def poisson_solve(self, w_dev, psi_dev, stream=None):
        """psi from omega (CUDA tensors [Ny,Nx] float64), the reference's Poisson2D_Z2Z::solve."""
        _check(self.lib.nse2d_poisson_solve(self.h, _ptr(w_dev), _ptr(psi_dev), _stream(stream)))

    def run(self, next_snap=1e300, next_diag=1e300, stats_every=0, t_end=1e300, max_steps=1 << 40, stream=None):
        """Step on the device until an output, statistics step, t_end, a non-finite value or
        max_steps stops the run; returns the NSE2D_HALT_* bits."""
        r = ctypes.c_int()
        _check(self.lib.nse2d_run(self.h, float(next_snap), float(next_diag), int(stats_every), float(t_end),
                                  int(max_steps), ctypes.byref(r), _stream(stream)))
        return r.value

    def row_moments(self, stream=None):
        """Row sums over x of u, v, u^2, v^2, u v: array [5, Ny]."""
        out = np.empty((5, self.Ny))
        _check(self.lib.nse2d_row_moments(self.h, _ptr(out), _stream(stream)))
        return out

    def stats_device(self, every, stream=None):
        """Accumulate the time-weighted row statistics on the device every `every` steps of run()
        (0: off); starts from zero at the current t."""
        _check(self.lib.nse2d_stats_device(self.h, int(every), _stream(stream)))

    def stats_read(self, stream=None):
        """(H [5, Ny], T): the accumulated time-weighted row means of u, v, u^2, v^2, u v and the
        total weight."""
        out = np.empty((5, self.Ny))
        T = ctypes.c_double()
        _check(self.lib.nse2d_stats_read(self.h, _ptr(out), ctypes.byref(T), _stream(stream)))
        return out, T.value

    def spectra_accumulate(self, stream=None):
        _check(self.lib.nse2d_spectra_accumulate(self.h, _stream(stream)))

    def spectra(self, stream=None):
        """(kx, E_u, E_v, samples), sample-averaged, k = 0..Nx/2."""
        H = self.Nx // 2 + 1
        kx, eu, ev = np.empty(H), np.empty(H), np.empty(H)
        n = ctypes.c_int()
        _check(self.lib.nse2d_spectra(self.h, _ptr(kx), _ptr(eu), _ptr(ev), ctypes.byref(n), _stream(stream)))
        return kx, eu, ev, n.value

    def max_uv(self, stream=None):
        out = (ctypes.c_double * 3)()
        _check(self.lib.nse2d_max_uv(self.h, out, _stream(stream)))
        return tuple(out)

    def diagnostics(self, t0_row=False, stream=None):
        out = (ctypes.c_double * 29)()
        _check(self.lib.nse2d_diagnostics(self.h, 1 if t0_row else 0, out, _stream(stream)))
        return dict(zip(DIAG_COLUMNS, list(out)))

    def rhs_at_state(self, t, stream=None):
        _check(self.lib.nse2d_rhs_at_state(self.h, float(t), _stream(stream)))

    def metric(self, which):
        n = self.Ny if which in (0, 1, 4) else self.Ny - 1
        out = np.empty(n)
        _check(self.lib.nse2d_metrics(self.h, which, _ptr(out)))
        return out

    def scalar(self, which):
        v = ctypes.c_double()
        _check(self.lib.nse2d_scalar(self.h, which, ctypes.byref(v)))
        return v.value


class Testapi:
    """The reference's C-linkage operator launchers (src/test_api.cu) on torch CUDA tensors."""

    def __init__(self):
        self.lib = load()

    def __getattr__(self, name):
        f = getattr(self.lib, "testapi_" + name)

        def call(*args, stream=None):
            conv = [_ptr(a) if hasattr(a, "data_ptr") or a is None else a for a in args]
            return f(*conv, _stream(stream))
        return call


class Ensemble:
    """Many Solver objects advanced together by one graph launch (nse2d_ensemble_*). The
    solvers must stay alive while the ensemble exists."""

    def __init__(self, solvers):
        self.lib = load()
        self.members = list(solvers)
        arr = (ctypes.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        h = ctypes.c_void_p()
        _check(self.lib.nse2d_ensemble_create(arr, len(self.members), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.nse2d_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, nsteps=1, stream=None):
        _check(self.lib.nse2d_ensemble_step(self.h, int(nsteps), _stream(stream)))

    def set_groups(self, groups):
        _check(self.lib.nse2d_ensemble_set_groups(self.h, int(groups)))

    def autotune_plans(self, trial_steps=5, stream=None):
        """The branch count, then the members' kernel plans by classes of equal grids (coordinate
        descent), then the branch count again: (branches, ms per ensemble step)."""
        g, ms = ctypes.c_int(), ctypes.c_double()
        _check(self.lib.nse2d_ensemble_autotune_plans(self.h, int(trial_steps), ctypes.byref(g), ctypes.byref(ms),
                                                      _stream(stream)))
        return g.value, ms.value

    def autotune(self, trial_steps=5, stream=None):
        """(branches, ms per ensemble step) of the fastest grouping, which stays selected."""
        g, ms = ctypes.c_int(), ctypes.c_double()
        _check(self.lib.nse2d_ensemble_autotune(self.h, int(trial_steps), ctypes.byref(g), ctypes.byref(ms),
                                                _stream(stream)))
        return g.value, ms.value
