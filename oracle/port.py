"""ctypes access to the plain-C restatement oracle (oracle/oracle.c).

Test infrastructure only (see oracle/oracle.c).  The library is built by
``make -C oracle port`` into oracle/_build/liboracle.so; it needs no reference
sources, so it exists wherever the repository is built.  `PortSim` mirrors
`oracle.ref.RefSim` so that tests run the same workload on both.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

MODELS = {"srmhd": 0, "srrmhd": 1}
BCS = {"outflow": 0, "periodic": 1, "flow": 2}
INTEGRATORS = {"rk2": 0, "rksplit": 1, "ssp2": 2, "ssp3": 3, "ssp2322": 4}


class PortConfig(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("endTime", C.c_double), ("cfl", C.c_double), ("Ng", C.c_int),
        ("gamma", C.c_double), ("sigma", C.c_double), ("cp", C.c_double),
        ("weno", C.c_int), ("bcs", C.c_int), ("integrator", C.c_int),
        ("functional_sigma", C.c_int), ("sigma_exp", C.c_double),
    ]


_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    I = C.POINTER(C.c_int)
    L.orc_create.restype = P
    L.orc_create.argtypes = [C.POINTER(PortConfig), D]
    L.orc_destroy.argtypes = [P]
    L.orc_update_time.argtypes = [P, C.c_int]
    L.orc_step.argtypes = [P, C.c_double]
    L.orc_info.argtypes = [P, I, D]
    L.orc_get_state.argtypes = [P, D, D, D]
    L.orc_set_state.argtypes = [P, D, D, D]
    L.orc_flux_F.argtypes = [P, D, D, D, D]
    L.orc_c2p.argtypes = [P, D, D, D]
    L.orc_prims_to_all.argtypes = [P, D, D, D]
    L.orc_apply_bcs.argtypes = [P, D, D, D]
    L.orc_source.argtypes = [P, D, D, D, D]
    L.orc_weno3_upwind.restype = C.c_double
    L.orc_weno3_upwind.argtypes = [C.c_double] * 3
    L.orc_weno5_upwind.restype = C.c_double
    L.orc_weno5_upwind.argtypes = [C.c_double] * 5
    L.orc_hybrd1_kat.argtypes = [C.c_int, C.c_int, D, D, C.c_double, C.c_int]
    L.orc_srmhd_solution.argtypes = [P, D, D]
    L.orc_srmhd_c2p_cells.argtypes = [C.c_int, C.c_double, C.c_double, D, D, D, I, I]
    _LIB = L
    return L


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


class PortSim:
    """The oracle's Simulation: same keywords as oracle.ref.RefSim (prims required)."""

    def __init__(self, prims, **kw):
        self.L = lib()
        c = PortConfig()
        c.model = MODELS[kw.get("model", "srmhd")]
        c.nx, c.ny, c.nz = kw["nx"], kw["ny"], kw.get("nz", 0)
        c.xmin, c.xmax = kw.get("xmin", 0.0), kw.get("xmax", 1.0)
        c.ymin, c.ymax = kw.get("ymin", 0.0), kw.get("ymax", 1.0)
        c.zmin, c.zmax = kw.get("zmin", 0.0), kw.get("zmax", 1.0)
        c.endTime, c.cfl, c.Ng = kw.get("endTime", 1.0), kw.get("cfl", 0.5), kw.get("Ng", 4)
        c.gamma, c.sigma, c.cp = kw.get("gamma", 5.0 / 3.0), kw.get("sigma", 1e3), kw.get("cp", 0.1)
        c.weno = kw.get("weno", 3)
        c.bcs = BCS[kw.get("bcs", "periodic")]
        c.integrator = INTEGRATORS[kw.get("integrator", "rk2")]
        c.functional_sigma = 1 if kw.get("functionalSigma", False) else 0
        c.sigma_exp = kw.get("gam", 12.0)
        self.cfg = c
        prims = np.ascontiguousarray(prims, dtype=np.float64)
        self.h = self.L.orc_create(C.byref(c), _ptr(prims))
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        self._refresh()

    def _refresh(self):
        ints = (C.c_int * 8)()
        dbl = (C.c_double * 5)()
        self.L.orc_info(self.h, ints, dbl)
        self.Nx, self.Ny, self.Nz, self.Ncons, self.Nprims, self.Naux, self.iters, self.dims = list(ints)
        self.t, self.dt, self.dx, self.dy, self.dz = list(dbl)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def zeros(self, nv):
        return np.zeros((nv, self.Nx, self.Ny, self.Nz), dtype=np.float64)

    def update_time(self, n=1):
        rc = self.L.orc_update_time(self.h, n)
        self._refresh()
        return rc

    def step_dt(self, dt):
        rc = self.L.orc_step(self.h, dt)
        self._refresh()
        return rc

    def state(self):
        c, p, a = self.zeros(self.Ncons), self.zeros(self.Nprims), self.zeros(self.Naux)
        self.L.orc_get_state(self.h, _ptr(c), _ptr(p), _ptr(a))
        return c, p, a

    def set_state(self, cons=None, prims=None, aux=None):
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        cons, prims, aux = f(cons), f(prims), f(aux)
        self.L.orc_set_state(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def flux_F(self, cons, prims, aux):
        fnet = self.zeros(self.Ncons)
        self.L.orc_flux_F(self.h, _ptr(cons), _ptr(prims), _ptr(aux), _ptr(fnet))
        return fnet

    def c2p(self, cons, prims, aux):
        return self.L.orc_c2p(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def solution(self, new=None):
        """SRMHD::solution as (2, Nx, Ny, Nz), replaced by `new` when given, and the
        number of cells the last C2P's retry left unconverged."""
        got = np.zeros((2, self.Nx, self.Ny, self.Nz), dtype=np.float64)
        if new is not None:
            new = np.ascontiguousarray(new, dtype=np.float64)
        still = self.L.orc_srmhd_solution(self.h, _ptr(got), _ptr(new))
        return got, still

    def prims_to_all(self, cons, prims, aux):
        self.L.orc_prims_to_all(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def apply_bcs(self, cons, prims, aux):
        self.L.orc_apply_bcs(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def source(self, cons, prims, aux):
        s = self.zeros(self.Ncons)
        self.L.orc_source(self.h, _ptr(cons), _ptr(prims), _ptr(aux), _ptr(s))
        return s


def weno3_upwind(a, b, c):
    return lib().orc_weno3_upwind(a, b, c)


def weno5_upwind(a, b, c, d, e):
    return lib().orc_weno5_upwind(a, b, c, d, e)


def hybrd1_kat(which, x0, tol=1.49011612e-8, n=2, lwa=19):
    xx = np.zeros(max(n, 2))
    xx[:2] = x0
    fvec = np.zeros(max(n, 2))
    info = lib().orc_hybrd1_kat(which, n, _ptr(xx), _ptr(fvec), tol, lwa)
    return info, xx[:2], fvec[:2]


def srmhd_c2p_cells(cons, guess, gamma, tol=1.49011612e-7):
    """Per-cell SRMHD hybrd1 solves; cons (n, 9), guess (n, 2) -> (sol, info, nfev).
    tol 1.49011612e-7 is the grid C2P's (srmhd.cc:380), 1.4e-8 the single-cell one."""
    cons = np.ascontiguousarray(cons, dtype=np.float64)
    guess = np.ascontiguousarray(guess, dtype=np.float64)
    n = cons.shape[0]
    sol = np.zeros((n, 2))
    info = np.zeros(n, dtype=np.int32)
    nfev = np.zeros(n, dtype=np.int32)
    lib().orc_srmhd_c2p_cells(n, gamma, tol, _ptr(cons), _ptr(guess), _ptr(sol),
                              info.ctypes.data_as(C.POINTER(C.c_int)),
                              nfev.ctypes.data_as(C.POINTER(C.c_int)))
    return sol, info, nfev
