"""METHOD-B200: METHOD's per-timestep hot path on B200 behind METHOD's own API.

Python mirror of the reference's Simulation interface
(Project/CPU/Include/simulation.h:23-118) over the C ABI of
``include/method_b200.h``.  The model, flux method, boundary conditions and
time integrator are chosen by name exactly as a reference ``main.cc`` wires
the corresponding classes together (Examples/KelvinHelmholtz/
SingleFluidIdealSerial/main.cc:18-79).

Errors follow the reference's exceptions: non-convergence raises
RuntimeError (srrmhd.cc:578, SSP2.cc:92-137), bad configuration raises
ValueError (std::invalid_argument in simData.cc:100-106, weno.cc:18).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

MODELS = {"srmhd": 0, "srrmhd": 1, "hybrid": 2}
BCS = {"outflow": 0, "periodic": 1, "flow": 2}
INTEGRATORS = {"rk2": 0, "rksplit": 1, "ssp2": 2, "ssp3": 3, "ssp2322": 4, "rksplit2": 5}
PRECISIONS = {"fp64": 0, "mixed": 1}
GUESSES = {"previous": 0, "mlp": 1}

__all__ = ["Simulation", "Ensemble", "train_guess", "MODELS", "BCS", "INTEGRATORS", "pin_host", "unpin_host"]


def pin_host(arr):
    """Page-locks a numpy array's memory for DMA copies."""
    L = _lib.load()
    if L.mth_pin_host(arr.ctypes.data, arr.nbytes) != 0:
        raise RuntimeError("cudaHostRegister failed")


def unpin_host(arr):
    _lib.load().mth_unpin_host(arr.ctypes.data)


def _dptr(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _config(nx, ny, nz=0, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
            endTime=1.0, cfl=0.5, Ng=4, gamma=5.0 / 3.0, sigma=1e3, cp=0.1, model="srmhd",
            weno=3, bcs="periodic", integrator="rk2", precision="fp64", guess="previous",
            device=0, functionalSigma=False, gam=12.0, x_slab=None, regime=False,
            sigmaCrossOver=150.0, sigmaSpan=50.0, useREGIME=True):
    """mth_config from the reference Data constructor's arguments plus the
    class choices of a reference main.cc (``regime=True``: the REGIME model
    extension with RKSplit; ``model="hybrid"``: Hybrid(data, sigmaCrossOver,
    sigmaSpan, useREGIME))."""
    c = _lib.Config()
    c.model = MODELS[model]
    c.nx, c.ny, c.nz = nx, ny, nz
    c.xmin, c.xmax, c.ymin, c.ymax, c.zmin, c.zmax = xmin, xmax, ymin, ymax, zmin, zmax
    c.endTime, c.cfl, c.Ng = endTime, cfl, Ng
    c.gamma, c.sigma, c.cp = gamma, sigma, cp
    c.weno_order = weno
    c.bcs = BCS[bcs]
    c.integrator = INTEGRATORS[integrator]
    c.precision = PRECISIONS[precision]
    c.guess = GUESSES[guess]
    c.device = device
    c.functional_sigma = 1 if functionalSigma else 0
    c.sigma_exp = gam
    c.regime = 1 if regime else 0
    c.sigma_crossover, c.sigma_span = sigmaCrossOver, sigmaSpan
    if model == "hybrid":
        c.regime = 1 if useREGIME else 0
    if x_slab is not None:  # (offset, global nx): columns [offset, offset + nx) of the domain
        c.x_slab = 1
        c.x_offset, c.x_global_nx = x_slab
    return c


class Simulation:
    """One device-resident simulation (Data + Model + FVS + Bcs + integrator).

    Keyword arguments are the reference Data constructor's (nx, ny, nz, xmin ..
    zmax, endTime, cfl, Ng, gamma, sigma, cp) plus ``model``, ``weno``,
    ``bcs``, ``integrator``, ``precision``, ``guess`` and ``regime`` (the
    REGIME resistive extension of SRMHD under RKSplit, REGIME.cc).  The Hybrid
    model (``model="hybrid"``, hybrid.cc) takes ``sigmaCrossOver``,
    ``sigmaSpan`` and ``useREGIME`` and runs with ``integrator="rk2"`` or
    ``"rksplit2"`` (rkSplit2ndOrder.cc), plain or mixed.
    """

    def __init__(self, nx, ny, nz=0, **kw):
        self.L = _lib.load()
        c = _config(nx, ny, nz, **kw)
        self.cfg = c
        h = C.c_void_p()
        rc = self.L.mth_create(C.byref(c), C.byref(h))
        if rc == 3:
            raise ValueError("invalid simulation configuration")
        if rc != 0:
            raise RuntimeError(f"mth_create failed: {_lib.STATUS.get(rc, rc)}")
        self.h = h
        d = (C.c_int * 7)()
        self.L.mth_get_dims(self.h, d)
        self.Nx, self.Ny, self.Nz, self.Ncons, self.Nprims, self.Naux, self.dims = list(d)

    # -- lifetime ---------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.mth_destroy(self.h)
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

    # -- helpers ----------------------------------------------------------------
    def _check(self, rc, what):
        if rc == 0:
            return
        msg = self.L.mth_last_error(self.h).decode()
        if rc in (1, 2):
            raise RuntimeError(f"{what}: {msg}")
        if rc == 3:
            raise ValueError(f"{what}: {msg}")
        raise RuntimeError(f"{what}: CUDA error: {msg}")

    def shape(self, nv):
        return (nv, self.Nx, self.Ny, self.Nz)

    def zeros(self, nv):
        return np.zeros(self.shape(nv), dtype=np.float64)

    # -- reference API ----------------------------------------------------------
    def set_prims(self, prims):
        """InitialFunc + Simulation::set: primitive state of every cell."""
        prims = np.ascontiguousarray(prims, dtype=np.float64)
        if prims.shape != self.shape(self.Nprims):
            raise ValueError(f"prims must have shape {self.shape(self.Nprims)}")
        self._check(self.L.mth_set_prims(self.h, _dptr(prims)), "set")

    def upload(self, cons=None, prims=None, aux=None):
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        cons, prims, aux = f(cons), f(prims), f(aux)
        self._check(self.L.mth_upload(self.h, _dptr(cons), _dptr(prims), _dptr(aux)), "upload")

    def state(self):
        """(cons, prims, aux) in the reference layout, ghosts included."""
        c, p, a = self.zeros(self.Ncons), self.zeros(self.Nprims), self.zeros(self.Naux)
        self._check(self.L.mth_download(self.h, _dptr(c), _dptr(p), _dptr(a)), "download")
        return c, p, a

    def apply_bcs(self):
        self._check(self.L.mth_apply_bcs(self.h), "Bcs::apply")

    def prims_to_all(self):
        self._check(self.L.mth_prims_to_all(self.h), "primsToAll")

    def c2p(self):
        self._check(self.L.mth_c2p(self.h), "getPrimitiveVars")

    def flux_F(self):
        f = self.zeros(self.Ncons)
        self._check(self.L.mth_flux_F(self.h, _dptr(f)), "FVS::F")
        return f

    def source(self):
        s = self.zeros(self.Ncons)
        self._check(self.L.mth_source(self.h, _dptr(s)), "sourceTerm")
        return s

    def flux_vector(self, dir):
        """Model::fluxVector of the current state along dir (0, 1, 2), every cell."""
        f = self.zeros(self.Ncons)
        self._check(self.L.mth_flux_vector(self.h, int(dir), _dptr(f)), "fluxVector")
        return f

    def step(self, dt, sync=True):
        """TimeIntegrator::step with an explicit dt."""
        self._check(self.L.mth_step(self.h, float(dt)), "step")
        if sync:
            self.sync()

    def update_time(self, n=1, sync=True):
        """Simulation::updateTime, n times."""
        self._check(self.L.mth_update_time(self.h, int(n)), "updateTime")
        if sync:
            self.sync()

    def evolve(self):
        self._check(self.L.mth_evolve(self.h), "evolve")

    def sync(self):
        self._check(self.L.mth_sync(self.h), "step")

    def stats(self):
        s = _lib.Stats()
        rc = self.L.mth_get_stats(self.h, C.byref(s))
        d = {k: getattr(s, k) for k, _ in _lib.Stats._fields_}
        d["status"] = rc
        return d

    def reset_stats(self):
        self._check(self.L.mth_reset_stats(self.h), "reset_stats")

    def step_host(self, cons, prims, aux, dt):
        """TimeIntegrator::step(cons, prims, aux, dt) on host arrays (in place)."""
        for a in (cons, prims, aux):
            if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
                raise ValueError("arrays must be C-contiguous float64")
        self._check(self.L.mth_step_host(self.h, _dptr(cons), _dptr(prims), _dptr(aux),
                                         float(dt)), "step")

    def set_mlp(self, params, stats):
        """Installs a trained C2P guess network (mixed form with guess='mlp')."""
        params = np.ascontiguousarray(params, dtype=np.float32)
        stats = np.ascontiguousarray(stats, dtype=np.float32)
        F = C.POINTER(C.c_float)
        self._check(self.L.mth_set_mlp(self.h, params.ctypes.data_as(F), stats.ctypes.data_as(F)),
                    "set_mlp")

    def set_stream(self, stream_ptr):
        """Orders this simulation's work on an external cudaStream_t (int / None)."""
        self._check(self.L.mth_set_stream(self.h, stream_ptr), "set_stream")

    def profile_step(self, dt, reps=3):
        """Per-kernel event timing of `reps` eager steps: list of dicts."""
        out = (_lib.KernelTime * 32)()
        n = C.c_int()
        self._check(self.L.mth_profile_step(self.h, float(dt), int(reps), out, 32, C.byref(n)),
                    "profile")
        return [dict(name=out[i].name.decode(), launches=out[i].launches,
                     total_ms=out[i].total_ms, bytes_per_launch=out[i].bytes_per_launch)
                for i in range(min(n.value, 32))]

    def save_text(self, dir, app="", which=31):
        """SerialSaveData output: dir/Conserved/cons<app>.dat, Primitive, Auxiliary,
        Domain and Constants files (which: mask cons 1, prims 2, aux 4, domain 8,
        constants 16); the directories must exist."""
        self._check(self.L.mth_save_text(self.h, str(dir).encode(), str(app).encode(),
                                         int(which)), "save")

    def device_state(self):
        """Raw device pointers (cons, prims, aux) for zero-copy interop."""
        c, p, a = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
        self._check(self.L.mth_device_state(self.h, C.byref(c), C.byref(p), C.byref(a)), "state")
        return (C.cast(c, C.c_void_p).value, C.cast(p, C.c_void_p).value,
                C.cast(a, C.c_void_p).value)

    @property
    def t(self):
        return self.stats()["t"]


def train_guess(seed=7, n_samples=1 << 19, iterations=4000, batch=8192, lr=3e-3,
                gamma=4.0 / 3.0, device=0, model="srmhd"):
    """Trains the C2P guess network of `model` on the GPU on (conserved ->
    primitive) pairs the solver generates (mth_mlp_train).  Returns (params,
    stats, final loss) for Simulation.set_mlp / Ensemble.set_mlp."""
    L = _lib.load()
    cfg = _lib.MlpTrainConfig(seed=seed, n_samples=n_samples, iterations=iterations, batch=batch,
                              lr=lr, gamma=gamma, model=MODELS[model])
    P = np.zeros(_lib.MLP_NPARAM, dtype=np.float32)
    S = np.zeros(_lib.MLP_NSTAT, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    F = C.POINTER(C.c_float)
    rc = L.mth_mlp_train(C.byref(cfg), P.ctypes.data_as(F), S.ctypes.data_as(F),
                         loss.ctypes.data_as(F), device)
    if rc != 0:
        raise RuntimeError(f"mth_mlp_train failed: {_lib.STATUS.get(rc, rc)}")
    return P, S, float(loss[0])


class Ensemble:
    """Independent 2D simulations of uneven sizes advanced together on one GPU.

    ``members`` is a list of keyword dicts, each what ``Simulation`` takes.
    One ``step()`` advances every member by one of its own time steps
    (Simulation::updateTime per member: dt from each member's CFL condition,
    clipped to its endTime).  Supported members: SRMHD + RK2 (fp64 or mixed)
    and SRRMHD + SSP2 (mixed); all share precision, WENO order and device.
    """

    _NV = {0: (9, 8, 13), 1: (14, 11, 17)}

    def __init__(self, members):
        self.L = _lib.load()
        cfgs = (_lib.Config * len(members))()
        for i, kw in enumerate(members):
            kw = dict(kw)
            cfgs[i] = _config(kw.pop("nx"), kw.pop("ny"), kw.pop("nz", 0), **kw)
        self.cfgs = cfgs
        e = C.c_void_p()
        rc = self.L.mth_ensemble_create(cfgs, len(members), C.byref(e))
        if rc == 3:
            raise ValueError("invalid ensemble configuration")
        if rc != 0:
            raise RuntimeError(f"mth_ensemble_create failed: {_lib.STATUS.get(rc, rc)}")
        self.e = e
        self.n = len(members)

    def close(self):
        if getattr(self, "e", None):
            self.L.mth_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return self.n

    def _check(self, rc, what):
        if rc == 0:
            return
        msg = self.L.mth_ensemble_last_error(self.e).decode()
        if rc in (1, 2):
            raise RuntimeError(f"{what}: {msg}")
        if rc == 3:
            raise ValueError(f"{what}: {msg}")
        raise RuntimeError(f"{what}: CUDA error: {msg}")

    def shape(self, m, which):
        c = self.cfgs[m]
        ng = 2 * c.Ng
        nv = self._NV[c.model][which]
        return (nv, c.nx + ng, c.ny + ng, 1)

    def set_prims(self, m, prims):
        prims = np.ascontiguousarray(prims, dtype=np.float64)
        if prims.shape != self.shape(m, 1):
            raise ValueError(f"prims of member {m} must have shape {self.shape(m, 1)}")
        self._check(self.L.mth_ensemble_set_prims(self.e, m, _dptr(prims)), "set")

    def state(self, m):
        c, p, a = (np.zeros(self.shape(m, w)) for w in range(3))
        self._check(self.L.mth_ensemble_download(self.e, m, _dptr(c), _dptr(p), _dptr(a)),
                    "download")
        return c, p, a

    def autotune(self, reps=3):
        """Tunes the flux tile height and grid per member size class and the
        cell phases' grid; returns the three tile heights."""
        ti = (C.c_int * 3)()
        self._check(self.L.mth_ensemble_autotune(self.e, int(reps), ti), "autotune")
        return list(ti)

    def tuning(self):
        """The autotuner's choice and its measured gain (dict)."""
        t = _lib.EnsembleTuning()
        self._check(self.L.mth_ensemble_tuning(self.e, C.byref(t)), "tuning")
        return {"tile_height": list(t.tile_height), "flux_ctas": list(t.flux_ctas),
                "cell_ctas": t.cell_ctas, "default_ms": t.default_ms, "tuned_ms": t.tuned_ms}

    def step(self, n=1, sync=True):
        self._check(self.L.mth_ensemble_step(self.e, int(n)), "step")
        if sync:
            self.sync()

    def sync(self):
        self._check(self.L.mth_ensemble_sync(self.e), "step")

    def profile(self, reps=2):
        """Per-phase timing of `reps` eager steps (they advance the members)."""
        out = (_lib.KernelTime * 64)()
        n = C.c_int()
        self._check(self.L.mth_ensemble_profile(self.e, int(reps), out, 64, C.byref(n)),
                    "profile")
        return [dict(name=out[i].name.decode(), launches=out[i].launches,
                     total_ms=out[i].total_ms) for i in range(min(n.value, 64))]

    def set_mlp(self, params, stats, model="srmhd"):
        """Installs a trained C2P guess network for the members of `model`
        (members created with guess='mlp')."""
        params = np.ascontiguousarray(params, dtype=np.float32)
        stats = np.ascontiguousarray(stats, dtype=np.float32)
        F = C.POINTER(C.c_float)
        fn = self.L.mth_ensemble_set_mlp if model == "srmhd" else self.L.mth_ensemble_set_mlp_srrmhd
        self._check(fn(self.e, params.ctypes.data_as(F), stats.ctypes.data_as(F)), "set_mlp")

    def set_stream(self, stream_ptr):
        self._check(self.L.mth_ensemble_set_stream(self.e, stream_ptr), "set_stream")

    def stats(self, m):
        s = _lib.Stats()
        self._check(self.L.mth_ensemble_stats(self.e, m, C.byref(s)), "stats")
        return {k: getattr(s, k) for k, _ in _lib.Stats._fields_}

    def info(self):
        n = C.c_longlong()
        ti = (C.c_int * 3)()
        self._check(self.L.mth_ensemble_info(self.e, C.byref(n), ti), "info")
        return dict(interior_cells=n.value, tile_heights=list(ti))
