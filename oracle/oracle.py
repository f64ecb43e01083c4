"""ctypes wrapper of the CPU FP64 oracle (liboracle.so). TEST INFRASTRUCTURE ONLY.

The oracle is the checker of the CUDA path: a restatement of the reference's algorithm
(see nse2d_oracle.cpp for the file:line citations). Only tests/, the smoke check and the
CPU baseline / reference arm of bench.py use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
EXE = os.path.join(HERE, "_build", "nse2d_oracle")


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


class OrConfig(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Lx", ctypes.c_double), ("h", ctypes.c_double),
                ("stretch", ctypes.c_int), ("beta", ctypes.c_double), ("Ub", ctypes.c_double),
                ("Reb", ctypes.c_double), ("nu_override", ctypes.c_double), ("dt_init", ctypes.c_double),
                ("dt_max", ctypes.c_double), ("cfl", ctypes.c_double), ("cvisc", ctypes.c_double),
                ("adapt", ctypes.c_int), ("t_end", ctypes.c_double), ("F0", ctypes.c_double),
                ("nforce", ctypes.c_int), ("lin_drag", ctypes.c_double), ("free_slip", ctypes.c_int),
                ("mms", ctypes.c_int), ("mms_A0", ctypes.c_double), ("mms_eps", ctypes.c_double),
                ("mms_Om", ctypes.c_double), ("mms_kx", ctypes.c_int), ("closure_diag", ctypes.c_int)]


DEFAULTS = dict(Nx=1024, Ny=1025, Lx=12.566370612, h=1.0, stretch=0, beta=0.0, Ub=1.0, Reb=10000.0,
                nu_override=-1.0, dt_init=1e-3, dt_max=1e-2, cfl=0.5, cvisc=0.5, adapt=1, t_end=200.0, F0=0.0,
                nforce=1, lin_drag=0.0, free_slip=0, mms=0, mms_A0=1e-3, mms_eps=0.1, mms_Om=1.0, mms_kx=1,
                closure_diag=0)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.or_create.restype = P
        L.or_create.argtypes = [ctypes.POINTER(OrConfig)]
        L.or_destroy.argtypes = [P]
        L.or_set_omega.argtypes = [P, P]
        L.or_get_fields.argtypes = [P, P, P]
        L.or_set_fields.argtypes = [P, P, P]
        L.or_metric.restype = ctypes.POINTER(ctypes.c_double)
        L.or_metric.argtypes = [P, I]
        L.or_adapt_dt.restype = D
        L.or_adapt_dt.argtypes = [P, P]
        L.or_step.argtypes = [P, D, D]
        L.or_diag_row.argtypes = [P, D, I, P]
        L.or_nu.restype = D
        L.or_nu.argtypes = [P]
        L.or_jwall.restype = D
        L.or_jwall.argtypes = [P, I]
        L.or_set_threads.argtypes = [I]
        L.or_get_threads.restype = I
        L.or_poisson_solve.argtypes = [P, P, I, I, D, P, P, D, D, D]
        L.or_max_uv.argtypes = [P, I, I, D, D, P, P]
        L.or_rfft_rows.argtypes = [P, P, I, I]
        for name in ("or_uv_from_psi",):
            getattr(L, name).argtypes = [P, P, P, I, I, D, D, P]
        L.or_omega_from_psi_interior.argtypes = [P, P, I, I, D, D, P, P]
        L.or_thom.argtypes = [P, P, I, I, P, D, D, I]
        L.or_arakawa.argtypes = [P, P, P, I, I, D, D, P]
        L.or_adv_from_uv.argtypes = [P, P, P, P, I, I, D, D, P]
        L.or_adv_flux.argtypes = [P, P, P, P, I, I, D, D, P]
        L.or_arakawa_split.argtypes = [P, P, P, P, P, P, I, I, D, D, P]
        L.or_laplacian.argtypes = [P, P, I, I, D, D, P, P]
        L.or_grid_metrics.argtypes = [I, I, D, D, I, D, P, P, P, P, P]
        L.or_row_moments.argtypes = [P, I, I, D, D, P, P, P, P, P, P]
        _lib = L
    return _lib


def p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def metrics(Nx, Ny, Lx, h, stretch, beta):
    y, an, w = np.empty(Ny), np.empty(Ny), np.empty(Ny)
    ae, de = np.empty(Ny - 1), np.empty(Ny - 1)
    rc = lib().or_grid_metrics(Nx, Ny, Lx, h, stretch, beta, p(y), p(an), p(ae), p(de), p(w))
    assert rc == 0
    return dict(y=y, a_node=an, a_edge=ae, dy_edge=de, w_node=w)


class OracleSolver:
    """CPU restatement of the reference time loop on one channel."""

    def __init__(self, **kw):
        c = dict(DEFAULTS)
        c.update(kw)
        self.cfg = OrConfig(**{k: c[k] for k, _ in OrConfig._fields_})
        self.h = lib().or_create(ctypes.byref(self.cfg))
        if not self.h:
            raise ValueError("oracle: bad configuration")
        self.Nx, self.Ny = self.cfg.Nx, self.cfg.Ny

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_omega(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        lib().or_set_omega(self.h, p(w))

    def set_fields(self, w, psi):
        lib().or_set_fields(self.h, p(np.ascontiguousarray(w)), p(np.ascontiguousarray(psi)))

    def fields(self):
        w, psi = np.empty((self.Ny, self.Nx)), np.empty((self.Ny, self.Nx))
        lib().or_get_fields(self.h, p(w), p(psi))
        return w, psi

    def metric(self, which):
        n = self.Ny if which in (0, 1, 4) else self.Ny - 1
        return np.ctypeslib.as_array(lib().or_metric(self.h, which), shape=(n,)).copy()

    def adapt_dt(self):
        m = np.zeros(3)
        dt = lib().or_adapt_dt(self.h, p(m))
        return dt, m

    def step(self, t, dt):
        lib().or_step(self.h, float(t), float(dt))

    def diag_row(self, t, t0_row=False):
        out = np.empty(29)
        lib().or_diag_row(self.h, float(t), 1 if t0_row else 0, p(out))
        return out

    @property
    def nu(self):
        return lib().or_nu(self.h)


def poisson_solve(w, Lx, m, psi_bot, psi_top):
    Ny, Nx = w.shape
    psi = np.empty_like(w)
    deta = 2.0 / (Ny - 1)
    lib().or_poisson_solve(p(np.ascontiguousarray(w)), p(psi), Nx, Ny, Lx, p(m["a_node"]), p(m["a_edge"]),
                           1.0 / deta, psi_bot, psi_top)
    return psi
