"""TEST INFRASTRUCTURE: ctypes wrapper of oracle/_ref/libnse2d_refloop.so, the reference's own time
loop driven through the reference's own launchers (ref_loop.cu). Only tests use it, as the checker
of this project's fields; the library is built from the reference's sources by oracle/ref.mk and
exists only where those sources were present.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libnse2d_refloop.so")
_lib = None


def available():
    return os.path.isfile(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.refloop_create.restype = P
        L.refloop_create.argtypes = [I, I, D, D, I, D, D, D, D, D, I, D, I, D, D, D, D, I, D, D, D, I]
        L.refloop_set_omega.argtypes = [P, P]
        L.refloop_step.argtypes = [P, I]
        L.refloop_get.argtypes = [P, P, P, P, P, P]
        L.refloop_destroy.argtypes = [P]
        for f in ("refloop_set_omega", "refloop_step", "refloop_get", "refloop_destroy"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


class RefLoop:
    """The reference's solver state on the GPU, stepped by its own loop (src/main.cu:434-541).
    Keyword arguments as nse2d_b200.Solver (Grid/Params fields of src/common.cuh:42-114)."""

    def __init__(self, Nx, Ny, Lx=12.566370612, h=1.0, stretch=0, beta=0.0, Ub=1.0, Reb=1e4, nu_override=-1.0,
                 F0=0.0, nforce=1, lin_drag=0.0, adapt=1, cfl=0.5, cvisc=0.5, dt_max=1e-2, dt_init=1e-3, mms=0,
                 mms_A0=1e-3, mms_eps=0.1, mms_Om=1.0, mms_kx=1):
        self.L = lib()
        self.Nx, self.Ny = Nx, Ny
        self.h = self.L.refloop_create(Nx, Ny, Lx, h, int(stretch), beta, Ub, Reb, nu_override, F0, nforce, lin_drag,
                                       int(adapt), cfl, cvisc, dt_max, dt_init, int(mms), mms_A0, mms_eps, mms_Om,
                                       mms_kx)

    def set_omega(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        assert w.shape == (self.Ny, self.Nx)
        self.L.refloop_set_omega(self.h, w.ctypes.data_as(ctypes.c_void_p))

    def step(self, n=1):
        self.L.refloop_step(self.h, int(n))

    def fields(self):
        w = np.empty((self.Ny, self.Nx))
        psi = np.empty((self.Ny, self.Nx))
        self.L.refloop_get(self.h, w.ctypes.data_as(ctypes.c_void_p), psi.ctypes.data_as(ctypes.c_void_p),
                           None, None, None)
        return w, psi

    def time(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        self.L.refloop_get(self.h, None, None, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st))
        return t.value, dt.value, st.value

    def close(self):
        if self.h:
            self.L.refloop_destroy(self.h)
            self.h = None
