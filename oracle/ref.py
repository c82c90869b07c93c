"""ctypes access to the reference METHOD CPU build (oracle/_ref/libmethod_ref*.so).

Test infrastructure only.  `oracle/Makefile` compiles the unmodified reference
sources (Project/CPU/Src/*.cc and the vendored cminpack) together with
`oracle/ref_driver.cc`; this module loads that library.  Only `tests/`,
`__graft_entry__.smoke()` and `bench.py`'s CPU-baseline / reference arms use it.

Arrays use the reference layout ID(var, i, j, k) (Project/CPU/Include/simData.h:10),
exposed here as numpy arrays of shape (nvars, Nx, Ny, Nz).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

MODELS = {"srmhd": 0, "srrmhd": 1, "hybrid": 2}
BCS = {"outflow": 0, "periodic": 1, "flow": 2}
INTEGRATORS = {"rk2": 0, "rksplit": 1, "ssp2": 2, "ssp3": 3, "ssp2322": 4, "rksplit2": 5}
INITS = {"array": 0, "ot": 1, "kh": 2, "khrandom": 3, "briowu": 4, "currentsheet": 5}


class RefConfig(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("endTime", C.c_double), ("cfl", C.c_double), ("Ng", C.c_int),
        ("gamma", C.c_double), ("sigma", C.c_double), ("cp", C.c_double),
        ("weno", C.c_int), ("bcs", C.c_int), ("integrator", C.c_int),
        ("init", C.c_int), ("init_arg0", C.c_int), ("init_arg1", C.c_int),
        ("functional_sigma", C.c_int), ("sigma_exp", C.c_double), ("extension", C.c_int),
        ("sigma_crossover", C.c_double), ("sigma_span", C.c_double), ("use_regime", C.c_int),
    ]


_LIBS: dict = {}


def available(omp: bool = False) -> bool:
    name = "libmethod_ref_omp.so" if omp else "libmethod_ref.so"
    return os.path.exists(os.path.join(REF_DIR, name))


def lib(omp: bool = False):
    name = "libmethod_ref_omp.so" if omp else "libmethod_ref.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: build it with `make -C oracle`")
    L = C.CDLL(path)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    L.mref_create.restype = P
    L.mref_create.argtypes = [C.POINTER(RefConfig), D]
    L.mref_destroy.argtypes = [P]
    L.mref_update_time.argtypes = [P, C.c_int]
    L.mref_step_dt.argtypes = [P, C.c_double]
    L.mref_info.argtypes = [P, C.POINTER(C.c_int), D]
    L.mref_get_state.argtypes = [P, D, D, D]
    L.mref_set_state.argtypes = [P, D, D, D]
    L.mref_flux_F.argtypes = [P, D, D, D, D]
    L.mref_flux_vector.argtypes = [P, D, D, D, D, C.c_int]
    L.mref_c2p.argtypes = [P, D, D, D]
    L.mref_c2p_single.argtypes = [P, D, D, D]
    L.mref_prims_to_all.argtypes = [P, D, D, D]
    L.mref_source.argtypes = [P, D, D, D, D]
    L.mref_apply_bcs.argtypes = [P, D, D, D]
    L.mref_weno3_upwind.restype = C.c_double
    L.mref_weno3_upwind.argtypes = [C.c_double] * 3
    L.mref_weno5_upwind.restype = C.c_double
    L.mref_weno5_upwind.argtypes = [C.c_double] * 5
    L.mref_hybrd1_kat.argtypes = [C.c_int, C.c_int, D, D, C.c_double, C.c_int]
    L.mref_save_text.argtypes = [P, C.c_char_p, C.c_char_p]
    L.mref_save_text.restype = C.c_int
    _LIBS[name] = L
    return L


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_config(**kw) -> RefConfig:
    c = RefConfig()
    c.model = MODELS[kw.get("model", "srmhd")]
    c.nx, c.ny, c.nz = kw["nx"], kw["ny"], kw.get("nz", 0)
    c.xmin, c.xmax = kw.get("xmin", 0.0), kw.get("xmax", 1.0)
    c.ymin, c.ymax = kw.get("ymin", 0.0), kw.get("ymax", 1.0)
    c.zmin, c.zmax = kw.get("zmin", 0.0), kw.get("zmax", 1.0)
    c.endTime = kw.get("endTime", 1.0)
    c.cfl = kw.get("cfl", 0.5)
    c.Ng = kw.get("Ng", 4)
    c.gamma = kw.get("gamma", 5.0 / 3.0)
    c.sigma = kw.get("sigma", 1e3)
    c.cp = kw.get("cp", 0.1)
    c.weno = kw.get("weno", 3)
    c.bcs = BCS[kw.get("bcs", "periodic")]
    c.integrator = INTEGRATORS[kw.get("integrator", "rk2")]
    c.init = INITS[kw.get("init", "array")]
    c.init_arg0 = kw.get("init_arg0", 0)
    c.init_arg1 = kw.get("init_arg1", 0)
    c.functional_sigma = 1 if kw.get("functionalSigma", False) else 0
    c.sigma_exp = kw.get("gam", 12.0)
    c.extension = 1 if kw.get("regime", False) else 0
    c.sigma_crossover = kw.get("sigmaCrossOver", 150.0)
    c.sigma_span = kw.get("sigmaSpan", 50.0)
    c.use_regime = 1 if kw.get("useREGIME", True) else 0
    return c


class RefSim:
    """One reference simulation (Data + Model + FVS + Bcs + Simulation + integrator)."""

    def __init__(self, prims=None, omp: bool = False, **kw):
        self.L = lib(omp)
        self.cfg = make_config(**kw)
        p = None
        if prims is not None:
            prims = np.ascontiguousarray(prims, dtype=np.float64)
            p = _ptr(prims)
        self.h = self.L.mref_create(C.byref(self.cfg), p)
        if not self.h:
            raise RuntimeError("reference rejected the configuration")
        self._refresh()

    def _refresh(self):
        ints = (C.c_int * 8)()
        dbl = (C.c_double * 5)()
        self.L.mref_info(self.h, ints, dbl)
        self.Nx, self.Ny, self.Nz, self.Ncons, self.Nprims, self.Naux, self.iters, self.dims = list(ints)
        self.t, self.dt, self.dx, self.dy, self.dz = list(dbl)

    def close(self):
        if self.h:
            self.L.mref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, nv):
        return (nv, self.Nx, self.Ny, self.Nz)

    def zeros(self, nv):
        return np.zeros(self.shape(nv), dtype=np.float64)

    def update_time(self, n: int = 1) -> int:
        rc = self.L.mref_update_time(self.h, n)
        self._refresh()
        return rc

    def save_text(self, dir: str, app: str = "") -> int:
        """SerialSaveData cons/prims/aux/domain/constants files into dir."""
        return self.L.mref_save_text(self.h, str(dir).encode(), str(app).encode())

    def step_dt(self, dt: float) -> int:
        rc = self.L.mref_step_dt(self.h, dt)
        self._refresh()
        return rc

    def state(self):
        c, p, a = self.zeros(self.Ncons), self.zeros(self.Nprims), self.zeros(self.Naux)
        self.L.mref_get_state(self.h, _ptr(c), _ptr(p), _ptr(a))
        return c, p, a

    def set_state(self, cons=None, prims=None, aux=None):
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        cons, prims, aux = f(cons), f(prims), f(aux)
        self.L.mref_set_state(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def flux_F(self, cons, prims, aux):
        fnet = self.zeros(self.Ncons)
        rc = self.L.mref_flux_F(self.h, _ptr(cons), _ptr(prims), _ptr(aux), _ptr(fnet))
        if rc:
            raise RuntimeError("FVS::F raised")
        return fnet

    def flux_vector(self, cons, prims, aux, d):
        f = self.zeros(self.Ncons)
        self.L.mref_flux_vector(self.h, _ptr(cons), _ptr(prims), _ptr(aux), _ptr(f), d)
        return f

    def c2p(self, cons, prims, aux) -> int:
        return self.L.mref_c2p(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def c2p_single(self, cons, prims, aux) -> int:
        return self.L.mref_c2p_single(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def prims_to_all(self, cons, prims, aux):
        self.L.mref_prims_to_all(self.h, _ptr(cons), _ptr(prims), _ptr(aux))

    def source(self, cons, prims, aux):
        s = self.zeros(self.Ncons)
        self.L.mref_source(self.h, _ptr(cons), _ptr(prims), _ptr(aux), _ptr(s))
        return s

    def apply_bcs(self, cons, prims, aux):
        self.L.mref_apply_bcs(self.h, _ptr(cons), _ptr(prims), _ptr(aux))


def weno3_upwind(a, b, c):
    return lib().mref_weno3_upwind(a, b, c)


def weno5_upwind(a, b, c, d, e):
    return lib().mref_weno5_upwind(a, b, c, d, e)


def hybrd1_kat(which: int, x0, tol=1.49011612e-8, n=2, lwa=19):
    x = np.array(x0, dtype=np.float64)
    fvec = np.zeros(max(n, 2), dtype=np.float64)
    xx = np.zeros(max(n, 2), dtype=np.float64)
    xx[: len(x)] = x
    info = lib().mref_hybrd1_kat(which, n, _ptr(xx), _ptr(fvec), tol, lwa)
    return info, xx[:2], fvec[:2]
