#!/usr/bin/env python
"""Benchmark: zone-updates/s of METHOD's RK2 time step on B200.

Workload: SRMHD relativistic Orszag-Tang 2D, periodic [0,1]^2 at 1024x1024,
rho = 1, p = 1, v = (-0.5 sin 2pi y, 0.5 sin 2pi x), B = (-sin 2pi y,
sin 4pi x), gamma = 4/3, FVS + WENO5, RK2, CFL 0.4 (synthetic data built on
the host, method_b200.initial.orszag_tang).  A step is one full RK2 step
(two fused flux stages and two primitive recoveries) over the 1024^2 grid.

Three forms run on the same initial data with the same dt sequence:
  plain     : all-FP64, bit-identical to the reference CPU build
  mixed     : FP32 flux/WENO, FP64 primitive recovery (Newton) and state
  mixed_mlp : mixed, Newton started from the learned guess (trained on the
              GPU at the start of the run, its loss and time reported)
The headline `value` is the mixed form; the other forms and their L1 error
against the plain FP64 result are on the same line, beside the ensemble
workload (256 uneven Kelvin-Helmholtz simulations, `ensemble`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: one process per GPU under torchrun.  The single-domain workload
runs an independent replica per rank (its path has no exchange step); the
ensemble's members are split over the ranks by cost.  Scaling is weak;
timing is the max over ranks of device time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 1024
WORKLOAD = ("SRMHD relativistic Orszag-Tang 2D 1024x1024 periodic, FVS+WENO5, RK2, CFL 0.4, "
            "gamma 4/3")
CFG = dict(model="srmhd", xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1e9, cfl=0.4, Ng=4,
           gamma=4.0 / 3.0, weno=5, bcs="periodic", integrator="rk2")


def steady_dt(n):
    # Simulation::updateTime's dt after the slow start (simulation.cc:113-117)
    dx = 1.0 / n
    return 0.4 * dx / (1.0 * np.sqrt(2.0))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class quiet_stdout:
    """Silences the process's C-level stdout (the reference build prints its
    per-cell diagnostics there) for the duration of a CPU baseline."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def interior(a, Ng=4):
    return a[:, Ng:-Ng, Ng:-Ng, :]


def run_form(mb, torch, prims0, n, form, steps, warmup, dt, device, guess=None):
    sim = mb.Simulation(nx=n, ny=n, precision=form, device=device,
                        guess="mlp" if guess else "previous", **CFG)
    if guess:
        sim.set_mlp(guess[0], guess[1])
    sim.set_prims(prims0)
    stream = torch.cuda.Stream(device=device)
    sim.set_stream(stream.cuda_stream)
    for _ in range(warmup):
        sim.step(dt, sync=False)
    sim.sync()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return sim, stream, start, end


ENS_MEMBERS = 256
ENS_WORKLOAD = ("256 independent 2D Kelvin-Helmholtz simulations (ideal SRMHD + RK2 and resistive "
                "SRRMHD + IMEX SSP2, 1/2 each by seed), nx uniform in [64, 512], ny = 2 nx, shear "
                "U(0.2, 0.8), sigma 10^U(2, 5), FVS+WENO3, CFL 0.4, flow boundaries; mixed form; "
                "one persistent launch per phase, step graph-captured, autotuned tile heights")


def cpu_ensemble(initial):
    """Reference-build (serial) estimate for one ensemble step: each member's
    cells divided by its model's measured reference rate on a KH member of the
    family (64x128: SRMHD RK2 for 20 steps, SRRMHD SSP2 for 2 steps)."""
    from oracle import ref
    if not ref.available():
        return None
    mem = initial.kh_ensemble(ENS_MEMBERS, seed=2024)
    rates = {}
    for model in ("srmhd", "srrmhd"):
        c, ic = next((c, ic) for c, ic in mem if c["model"] == model)
        c = dict(c, nx=64, ny=128, endTime=1e9)
        c.pop("precision", None)
        c.pop("guess", None)
        ic = dict(ic, nx=64, ny=128)
        sim = ref.RefSim(prims=initial.kelvin_helmholtz(**ic), **c)
        steps = 20 if model == "srmhd" else 2
        t0 = time.perf_counter()
        sim.update_time(steps)
        rates[model] = 64 * 128 * steps / (time.perf_counter() - t0)
    cells = sum(c["nx"] * c["ny"] for c, _ in mem)
    secs = sum(c["nx"] * c["ny"] / rates[c["model"]] for c, _ in mem)
    return {"value": cells / secs, "unit": "zone-updates/s", "cores": 1, "kind": "reference",
            "sample": "estimate: member cells / the reference build's serial rate per model "
                      f"(SRMHD RK2 {rates['srmhd']:.3g}, SRRMHD SSP2 {rates['srrmhd']:.3g} "
                      "zone-updates/s on a 64x128 member)"}


def run_ensemble(mb, initial, torch, ranks, K, W, guess, guess_r=None):
    """The ensemble workload, members split over ranks by cost (LPT)."""
    from method_b200.ranks import lpt_partition
    mem = initial.kh_ensemble(ENS_MEMBERS, seed=2024)
    costs = [c["nx"] * c["ny"] * (2 if c["model"] == "srrmhd" else 1) for c, _ in mem]
    mine = lpt_partition(costs, ranks.world)[ranks.rank]
    cfgs = []
    for i in mine:
        c = dict(mem[i][0], device=ranks.local)
        if guess:
            c["guess"] = "mlp"
        cfgs.append(c)
    ens = mb.Ensemble(cfgs)
    if guess:
        ens.set_mlp(guess[0], guess[1])
        if guess_r:
            ens.set_mlp(guess_r[0], guess_r[1], model="srrmhd")
    for k, i in enumerate(mine):
        ens.set_prims(k, initial.kelvin_helmholtz(**mem[i][1]))
    ti = ens.autotune(reps=2)
    tuning = ens.tuning()
    stream = torch.cuda.Stream(device=ranks.local)
    ens.set_stream(stream.cuda_stream)
    ens.step(W, sync=False)
    ens.sync()
    cells = ens.info()["interior_cells"]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ranks.barrier()
    ev0.record(stream)
    ens.step(K, sync=False)
    ev1.record(stream)
    ranks.barrier()
    ens.sync()
    ms = ranks.max(ev0.elapsed_time(ev1))
    total = ranks.sum(cells)
    st = [ens.stats(k) for k in range(len(mine))]
    agg = {k: sum(x[k] for x in st) for k in ("c2p_cells", "c2p_evals", "c2p_unconverged",
                                              "c2p_fallbacks", "implicit_cells", "implicit_evals",
                                              "implicit_fallbacks", "implicit_failed")}
    ens.close()
    n_res = sum(1 for c, _ in mem if c["model"] == "srrmhd")
    bytes_step = sum(mem[i][0]["nx"] * mem[i][0]["ny"] *
                     (SHEET_BYTES if mem[i][0]["model"] == "srrmhd" else 616) for i in mine)
    peak = measured_peaks()[0]
    ach = ranks.sum(bytes_step) / (ms / K * 1e-3) / 1e9
    return {"value": total * K / (ms * 1e-3), "unit": "zone-updates/s", "ms_per_step": ms / K,
            "steps": K, "warmup": W, "members": ENS_MEMBERS, "resistive_members": n_res,
            "members_this_rank": len(mine), "interior_cells_total": int(total),
            "tile_heights_by_class": ti, "autotune": tuning,
            "guess": "mlp" if guess else "previous",
            "c2p_newton_iters_per_cell": agg["c2p_evals"] / max(agg["c2p_cells"], 1),
            "implicit_iters_per_cell": agg["implicit_evals"] / max(agg["implicit_cells"], 1),
            **{k: agg[k] for k in ("c2p_unconverged", "c2p_fallbacks", "implicit_fallbacks",
                                   "implicit_failed")},
            "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(ach / peak, 4),
                         "bytes": "sum over members of cells x (616 B SRMHD RK2, 1624 B SRRMHD "
                                  "SSP2) per step"},
            "workload": ENS_WORKLOAD}


C2P_CELLS = 256 ** 3
C2P_WORKLOAD = ("SRMHD primitive recovery of 256^3 independent random states (W 10^U(0,1), rho "
                "10^U(-3,0), p/rho 10^U(-3,1), b^2/rho 10^U(-2,2), isotropic v and B directions), "
                "gamma 4/3; previous-step guess = generating rho and h 1% high, speed 1% low")


C2P_BYTES = 152  # cons 9 + guess 2 doubles in, prims 8 out, per cell


def cpu_c2p(cons, prims, aux, gamma, n=64):
    """SRMHD::getPrimitiveVars of the reference build (serial) on an n^3 grid
    holding the first n^3 of the same random states and guesses."""
    from oracle import ref
    if not ref.available():
        return None
    Ng = 4
    cfg = dict(model="srmhd", nx=n, ny=n, nz=n, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
               zmin=0.0, zmax=1.0, endTime=1.0, cfl=0.4, Ng=Ng, gamma=gamma, weno=3,
               bcs="outflow", integrator="rk2")
    N = n + 2 * Ng
    sl = (slice(None), slice(Ng, -Ng), slice(Ng, -Ng), slice(Ng, -Ng))

    def grid(vals, nv):
        a = np.zeros((nv, N, N, N))
        a[sl] = vals.reshape(nv, n, n, n)
        return a
    # ghost cells hold the first state: getPrimitiveVars recovers the interior only
    p0 = np.zeros((8, N, N, N))
    p0[:] = prims[:, :1, None, None]
    p0[sl] = prims.reshape(8, n, n, n)
    sim = ref.RefSim(prims=p0, **cfg)
    c, p, a = grid(cons, 9), p0, grid(aux, 13)
    t0 = time.perf_counter()
    sim.c2p(c, p, a)
    el = time.perf_counter() - t0
    return {"value": n ** 3 / el, "unit": "cells/s", "cores": 1, "kind": "reference",
            "sample": f"SRMHD::getPrimitiveVars on a {n}^3 grid of the same states and "
                      f"previous-step guesses, serial build (-O3), {el:.2f} s on the host"}


def run_c2p_batch(mb, torch, ranks, guess, reps=3, cpu=False):
    """Batched primitive recovery: the reference method (Powell hybrid) and
    Newton from the previous-step, cold and learned guesses, each timed with
    CUDA events on its stream, iterations and error against the generating
    state reported."""
    import ctypes as C
    from method_b200 import _lib
    L = _lib.load()
    n = C2P_CELLS
    gamma = 4.0 / 3.0
    dev = torch.device("cuda", ranks.local)
    F, D = C.POINTER(C.c_float), C.POINTER(C.c_double)
    feat = torch.empty((n, 8), dtype=torch.float32, device=dev)
    tgt = torch.empty((n, 2), dtype=torch.float32, device=dev)
    cons = torch.empty((9, n), dtype=torch.float64, device=dev)
    truth = torch.empty((8, n), dtype=torch.float64, device=dev)
    rc = L.mth_mlp_make_pairs(n, 4242 + ranks.rank, gamma, C.cast(feat.data_ptr(), F),
                              C.cast(tgt.data_ptr(), F), C.cast(cons.data_ptr(), D),
                              C.cast(truth.data_ptr(), D), ranks.local)
    if rc != 0:
        raise RuntimeError(f"mth_mlp_make_pairs: {rc}")
    del feat, tgt
    pg0 = truth.clone()
    pg0[0] *= 1.01
    pg0[1:4] *= 0.99
    ag0 = torch.zeros((13, n), dtype=torch.float64, device=dev)
    ag0[0] = (1.0 + truth[4] / truth[0] * (gamma / (gamma - 1.0))) * 1.01
    ctx = C.c_void_p()
    if L.mth_c2p_ctx_create(n, ranks.local, C.byref(ctx)) != 0:
        raise RuntimeError("mth_c2p_ctx_create failed")
    if guess:
        L.mth_c2p_ctx_set_mlp(ctx, guess[0].ctypes.data_as(F), guess[1].ctypes.data_as(F))
    stream = torch.cuda.Stream(device=dev)
    prims = torch.empty_like(pg0)
    aux = torch.empty_like(ag0)
    out = {}
    methods = [("hybrd_previous", 0, 0), ("newton_previous", 1, 0), ("newton_cold", 1, 2)]
    if guess:
        methods.append(("newton_mlp", 1, 1))
    for name, method, g in methods:
        ms = 0.0
        with torch.cuda.stream(stream):
            for rep in range(reps + 1):
                prims.copy_(pg0)
                aux.copy_(ag0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = L.mth_c2p_ctx_run(ctx, gamma, n, cons.data_ptr(), prims.data_ptr(),
                                      aux.data_ptr(), method, g, stream.cuda_stream)
                e1.record(stream)
                if r != 0:
                    raise RuntimeError(f"mth_c2p_ctx_run {name}: {r}")
                st = _lib.C2PBatchStats()
                L.mth_c2p_ctx_stats(ctx, stream.cuda_stream, C.byref(st))
                if rep > 0:
                    ms += e0.elapsed_time(e1)
            rel = ((prims[0] - truth[0]).abs() / truth[0])
            torch.cuda.synchronize(dev)
        ms = ranks.max(ms / reps)
        out[name] = {"cells_per_s": ranks.world * n / (ms * 1e-3), "ms": round(ms, 3),
                     "iters_per_cell": st.iterations / max(st.cells, 1),
                     "unconverged": int(st.unconverged), "fallbacks": int(st.fallbacks),
                     "median_rel_err_rho": float(rel.nan_to_num(1.0).median()),
                     "max_rel_err_rho": float(rel.nan_to_num(1.0).max())}
    L.mth_c2p_ctx_destroy(ctx)
    peak = measured_peaks()[0]
    for name, rec in out.items():
        ach = C2P_BYTES * n / (rec["ms"] * 1e-3) / 1e9
        rec["roofline"] = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                           "unit": "GB/s", "frac": round(ach / peak, 4),
                           "bytes_per_cell": C2P_BYTES}
    res = {"workload": C2P_WORKLOAD, "cells": n, "unit": "cells/s", "methods": out,
           "iterations": "hybrd: residual evaluations; newton: Newton steps (incl. fallbacks)",
           "roofline": out["newton_previous"]["roofline"],
           "hybrd_unconverged_fraction": out["hybrd_previous"]["unconverged"] / n}
    if cpu:
        m = 64 ** 3
        with quiet_stdout():
            res["cpu_baseline"] = cpu_c2p(cons[:, :m].cpu().numpy(), pg0[:, :m].cpu().numpy(),
                                          ag0[:, :m].cpu().numpy(), gamma)
    if "newton_mlp" in out:
        res["mlp_iters_saved_vs_cold"] = (out["newton_cold"]["iters_per_cell"]
                                          - out["newton_mlp"]["iters_per_cell"])
    return res


SHEET_SEED = 0
SHEET_N = (512, 1024)
SHEET_WORKLOAD = ("SRRMHD resistive current sheet 2D 512x1024 on [-0.5,0.5]x[-1,1], outflow, "
                  "rho 1, p 50, By tanh(x/0.01), E = -v x B, seeded velocity noise 1e-3, "
                  "gamma 4/3, sigma 10^U(1,5) per run from the seed, FVS+WENO3, IMEX SSP2, "
                  "CFL 0.4")
SHEET_BYTES = 1624  # algorithmic bytes per SSP2 zone-update (three passes over the state)


def sheet_cfg(sigma):
    nx, ny = SHEET_N
    return dict(model="srrmhd", nx=nx, ny=ny, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
                endTime=1e9, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=sigma, weno=3,
                bcs="outflow", integrator="ssp2")


def timed_steps(sim, torch, device, dt, K, W, barrier, max_over_ranks):
    """W warm-up steps, then K graph-launched steps timed with CUDA
    events on the simulation's stream; returns ms (max over ranks)."""
    stream = torch.cuda.Stream(device=device)
    sim.set_stream(stream.cuda_stream)
    for _ in range(W):
        sim.step(dt, sync=False)
    sim.sync()
    sim.reset_stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(K):
        sim.step(dt, sync=False)
    e1.record(stream)
    barrier()
    sim.sync()
    return max_over_ranks(e0.elapsed_time(e1))


def run_sheet(mb, initial, torch, ranks, K, W, peak, cpu, guess_r=None):
    """Config 3: SSP2 on the resistive current sheet, plain and mixed forms
    (and the mixed form seeded by the SRRMHD guess network when given), the
    reference CPU build's SSP2::step beside them (rank 0, N = 1)."""
    sigma = initial.sigma_for_seed(SHEET_SEED)
    cfg = sheet_cfg(sigma)
    nx, ny = SHEET_N
    cells = nx * ny
    p0 = initial.current_sheet(nx, ny, seed=SHEET_SEED)
    dt = 0.4 * min(1.0 / nx, 2.0 / ny) / np.sqrt(2.0)  # steady-state CFL dt
    out, states = {}, {}
    forms = [("plain", "fp64"), ("mixed", "mixed")] + ([("mixed_mlp", "mixed")] if guess_r else [])
    for form, prec in forms:
        sim = mb.Simulation(precision=prec, device=ranks.local,
                            guess="mlp" if form == "mixed_mlp" else "previous", **cfg)
        if form == "mixed_mlp":
            sim.set_mlp(*guess_r)
        sim.set_prims(p0)
        kk = max(2, K // 5) if form == "plain" else K
        ms = timed_steps(sim, torch, ranks.local, dt, kk, W, ranks.barrier, ranks.max)
        st = sim.stats()
        c, p, _ = sim.state()  # before the profiled steps below advance it
        states[form] = (interior(c), interior(p))
        ks, top, roof = roofline_of(sim, dt, peak)
        roof["peak_kind"] = "measured (burst copy bandwidth, kernel timed alone)"
        out[form] = {
            "value": ranks.world * cells * kk / (ms * 1e-3), "ms_per_step": ms / kk,
            "steps": kk, "implicit_failed": st["implicit_failed"],
            "implicit_iters_per_cell": st["implicit_evals"] / max(st["implicit_cells"], 1),
            "implicit_fallbacks": st["implicit_fallbacks"], "c2p_unconverged":
                st["c2p_unconverged"],
            "c2p_newton_iters_per_cell": st["c2p_evals"] / max(st["c2p_cells"], 1),
            "c2p_fallbacks": st["c2p_fallbacks"], "roofline": roof,
            "step_roofline": {"bytes_per_zone_update": SHEET_BYTES, "achieved_gbs": round(
                SHEET_BYTES * cells / (ms / kk * 1e-3) / 1e9, 1), "peak": peak,
                "frac": round(SHEET_BYTES * cells / (ms / kk * 1e-3) / 1e9 / peak, 4)},
            "kernels": [{"name": k["name"], "launches_per_step": k["launches"] / 3.0,
                         "ms_per_launch": round(k["total_ms"] / k["launches"], 4)} for k in ks],
        }
        sim.close()
    l1 = {}
    # both forms ran W + K(form) steps of the same dt; compare after equal step counts
    # by re-running the plain form's count in the mixed form
    sim = mb.Simulation(precision="mixed", device=ranks.local, **cfg)
    sim.set_prims(p0)
    for _ in range(W + out["plain"]["steps"]):
        sim.step(dt, sync=False)
    sim.sync()
    c, p, _ = sim.state()
    sim.close()
    for k, name in enumerate(("cons", "prims")):
        a, b = (interior(c), interior(p))[k], states["plain"][k]
        d = np.abs(a - b)
        l1[name] = {"l1_rel": float(d.sum() / np.abs(b).sum()), "max_abs": float(d.max())}
    res = {"workload": SHEET_WORKLOAD, "seed": SHEET_SEED, "sigma": sigma, "dt": dt,
           "unit": "zone-updates/s", "plain": out["plain"], "mixed": out["mixed"],
           "mixed_mlp": out.get("mixed_mlp"),
           "speedup_mixed_vs_plain": out["mixed"]["value"] / out["plain"]["value"],
           "l1_mixed_vs_fp64": {"steps": W + out["plain"]["steps"], **l1}}
    if cpu:
        res["cpu_baseline"] = cpu_sheet(cfg, p0, dt)
    return res


def cpu_sheet(cfg, p0, dt, steps=1):
    """The reference build's serial SSP2::step on the full grid (bounded sample)."""
    try:
        from oracle import ref
        if not ref.available():
            raise FileNotFoundError
        sim = ref.RefSim(prims=p0, **cfg)
        kind = "reference"
    except (FileNotFoundError, OSError):
        from oracle import port
        sim = port.PortSim(p0, **cfg)
        kind = "port"
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step_dt(dt)
    el = time.perf_counter() - t0
    n = cfg["nx"] * cfg["ny"]
    return {"value": n * steps / el, "unit": "zone-updates/s", "cores": 1, "kind": kind,
            "sample": f"{steps} SSP2 step(s) of the {cfg['nx']}x{cfg['ny']} sheet, serial build "
                      f"(-O3), {el:.1f} s on the host"}


KH_WORKLOAD = ("SRMHD Kelvin-Helmholtz 2D 64x128 on [-0.5,0.5]x[-1,1], Flow boundaries "
               "(periodic x, outflow y), rho 1, p 1, vx +-0.5 tanh shear layers at y = +-0.5 "
               "(width 0.01), seeded vy noise 0.01, B 0, gamma 4/3, FVS+WENO3, RK2, CFL 0.4, "
               "Simulation::evolve to t = 3")


def run_kh_full(mb, initial, torch, ranks, peak, cpu):
    """Config 1: the whole Kelvin-Helmholtz run (updateTime until t = 3), device
    time with CUDA events on the simulation's stream, both forms."""
    cfg = dict(model="srmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="flow",
               integrator="rk2")
    p0 = initial.kelvin_helmholtz(64, 128, seed=1234)
    cells = 64 * 128
    res = {"workload": KH_WORKLOAD, "unit": "zone-updates/s"}
    for form, prec in (("plain", "fp64"), ("mixed", "mixed")):
        # one untimed run builds the per-dt step graphs; the timed run replays them
        for rep in range(2):
            sim = mb.Simulation(precision=prec, device=ranks.local, **cfg)
            sim.set_prims(p0)
            stream = torch.cuda.Stream(device=ranks.local)
            sim.set_stream(stream.cuda_stream)
            if rep == 0:
                sim.evolve()
                sim.close()
                continue
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ranks.barrier()
            e0.record(stream)
            sim.evolve()
            e1.record(stream)
            ranks.barrier()
            ms = ranks.max(e0.elapsed_time(e1))
            st = sim.stats()
            ks = sim.profile_step(0.4 * (1.0 / 64) / np.sqrt(2.0), reps=3)  # steady dt
            top = max(ks, key=lambda k: k["total_ms"])
            avg = top["total_ms"] / top["launches"]
            ach = top["bytes_per_launch"] / (avg * 1e-3) / 1e9
            sim.close()
        res[form] = {"value": ranks.world * cells * st["iters"] / (ms * 1e-3),
                     "ms_total": ms, "iters": st["iters"], "t": st["t"],
                     "ms_per_step": ms / st["iters"],
                     "roofline": {"kernel": top["name"], "bound": "hbm", "achieved": round(ach, 1),
                                  "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
                                  "note": "state (0.7 MB cons) lives in L2: launch/latency bound"}}
    if cpu:
        res["cpu_baseline"] = cpu_kh(cfg, p0)
    return res


def cpu_kh(cfg, p0, steps=100):
    """The reference build's serial updateTime on the KH run's first `steps` calls."""
    try:
        from oracle import ref
        if not ref.available():
            raise FileNotFoundError
        sim = ref.RefSim(prims=p0, **cfg)
        kind = "reference"
    except (FileNotFoundError, OSError):
        from oracle import port
        sim = port.PortSim(p0, **cfg)
        kind = "port"
    t0 = time.perf_counter()
    sim.update_time(steps)
    el = time.perf_counter() - t0
    return {"value": cfg["nx"] * cfg["ny"] * steps / el, "unit": "zone-updates/s", "cores": 1,
            "kind": kind, "sample": f"the first {steps} updateTime calls of the 64x128 run, "
                                    f"serial build (-O3), {el:.1f} s on the host"}


REGIME_WORKLOAD = ("SRMHD relativistic Orszag-Tang 2D 1024x1024 periodic, FVS+WENO5, RKSplit "
                   "with the REGIME resistive extension, sigma 1e4, CFL 0.4, gamma 4/3")


def regime_cfg():
    return dict(CFG, integrator="rksplit", regime=True, sigma=1e4)


def run_regime(mb, initial, torch, ranks, n, K, W, peak):
    """REGIME (the resistive extension of SRMHD, REGIME.cc) as RKSplit's model
    extension on the Orszag-Tang grid, plain and mixed forms; the extension's
    launches are timed as one group (`regime_source_add`)."""
    cfg = regime_cfg()
    p0 = initial.orszag_tang(n, Ng=4)
    dt = steady_dt(n)
    cells = n * n
    res = {"workload": REGIME_WORKLOAD, "unit": "zone-updates/s", "n": n}
    for form, prec in (("plain", "fp64"), ("mixed", "mixed")):
        sim = mb.Simulation(nx=n, ny=n, precision=prec, device=ranks.local, **cfg)
        sim.set_prims(p0)
        kk = max(2, K // 5) if form == "plain" else K
        ms = timed_steps(sim, torch, ranks.local, dt, kk, W, ranks.barrier, ranks.max)
        st = sim.stats()
        ks = sim.profile_step(dt, reps=3)
        step_ms = sum(k["total_ms"] for k in ks) / 3.0
        reg = next(k for k in ks if k["name"] == "regime_source_add")
        reg_ms = reg["total_ms"] / reg["launches"]
        res[form] = {
            "value": ranks.world * cells * kk / (ms * 1e-3), "ms_per_step": ms / kk,
            "steps": kk, "c2p_unconverged": st["c2p_unconverged"],
            "regime": {"ms_per_launch": round(reg_ms, 4),
                       "share_of_profiled_step": round(reg_ms / step_ms, 4),
                       "bytes_per_launch": reg["bytes_per_launch"],
                       "achieved_gbs": round(reg["bytes_per_launch"] / (reg_ms * 1e-3) / 1e9, 1),
                       "peak": peak},
            "kernels": [{"name": k["name"], "launches_per_step": k["launches"] / 3.0,
                         "ms_per_launch": round(k["total_ms"] / k["launches"], 4)} for k in ks],
        }
        sim.close()
    return res


def cpu_regime(n=512, steps=2):
    """The reference build's serial RKSplit + REGIME step on an n^2 Orszag-Tang
    grid (bounded sample of the REGIME workload)."""
    from method_b200 import initial
    cfg = regime_cfg()
    p0 = initial.orszag_tang(n, Ng=4)
    try:
        from oracle import ref
        if not ref.available():
            raise FileNotFoundError
        sim = ref.RefSim(prims=p0, nx=n, ny=n, **cfg)
    except (FileNotFoundError, OSError):
        return None  # the oracle port has no REGIME
    dt = steady_dt(n)
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step_dt(dt)
    el = time.perf_counter() - t0
    sim.close()
    return {"value": n * n * steps / el, "unit": "zone-updates/s", "cores": 1,
            "kind": "reference", "sample": f"{steps} RKSplit + REGIME steps of a {n}x{n} grid, "
                                           f"serial build (-O3), {el:.1f} s on the host"}


HYBRID_WORKLOAD = ("Hybrid SRMHD/SRRMHD model, Orszag-Tang 2D 1024x1024 periodic, FVS+WENO3, "
                   "RKSplit2, sigma 170 (blend weight 0.92), sigmaCrossOver 150, sigmaSpan 50, "
                   "REGIME on the ideal part, CFL 0.3, gamma 2")


def hybrid_cfg():
    return dict(model="hybrid", integrator="rksplit2", xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
                endTime=1e9, cfl=0.3, Ng=4, gamma=2.0, sigma=170.0, cp=1.0, weno=3,
                bcs="periodic", sigmaCrossOver=150.0, sigmaSpan=50.0, useREGIME=True)


def hybrid_prims(initial, n):
    p = np.zeros((11, n + 8, n + 8, 1))
    p[:8] = initial.orszag_tang(n, Ng=4)
    return p


def run_hybrid(mb, initial, torch, ranks, n, K, W):
    """The Hybrid model (hybrid.cc) under RKSplit2 (rkSplit2ndOrder.cc), plain
    and mixed forms: device time per step and the per-kernel split of one
    profiled step."""
    cfg = hybrid_cfg()
    dt = 0.3 / n / np.sqrt(2.0)
    res = {"workload": HYBRID_WORKLOAD, "unit": "zone-updates/s", "n": n}
    for form, prec in (("plain", "fp64"), ("mixed", "mixed")):
        sim = mb.Simulation(nx=n, ny=n, device=ranks.local, precision=prec, **cfg)
        sim.set_prims(hybrid_prims(initial, n))
        ms = timed_steps(sim, torch, ranks.local, dt, K, W, ranks.barrier, ranks.max)
        st = sim.stats()
        ks = sim.profile_step(dt, reps=2)
        sim.close()
        res[form] = {
            "value": ranks.world * n * n * K / (ms * 1e-3), "ms_per_step": ms / K, "steps": K,
            "c2p_unconverged": st["c2p_unconverged"],
            "kernels": [{"name": k["name"], "launches_per_step": k["launches"] / 2.0,
                         "ms_per_launch": round(k["total_ms"] / k["launches"], 4)} for k in ks]}
    return res


def cpu_hybrid(n=256, steps=2):
    """The reference build's serial Hybrid + RKSplit2 step on an n^2 grid."""
    from method_b200 import initial
    try:
        from oracle import ref
        if not ref.available():
            raise FileNotFoundError
        sim = ref.RefSim(prims=hybrid_prims(initial, n), nx=n, ny=n, **hybrid_cfg())
    except (FileNotFoundError, OSError):
        return None  # the oracle port has no Hybrid model
    dt = 0.3 / n / np.sqrt(2.0)
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step_dt(dt)
    el = time.perf_counter() - t0
    sim.close()
    return {"value": n * n * steps / el, "unit": "zone-updates/s", "cores": 1,
            "kind": "reference", "sample": f"{steps} RKSplit2 steps of the Hybrid model on a "
                                           f"{n}x{n} grid, serial build (-O3), {el:.1f} s"}


def cpu_legs(initial, sheet, kh, ensemble, regime=None, hybrid=None):
    """The reference build's CPU baselines of the side workloads."""
    if regime is not None:
        regime["cpu_baseline"] = cpu_regime()
    if hybrid is not None:
        hybrid["cpu_baseline"] = cpu_hybrid()
    if sheet is not None:
        sheet["cpu_baseline"] = cpu_sheet(sheet_cfg(sheet["sigma"]),
                                          initial.current_sheet(*SHEET_N, seed=SHEET_SEED),
                                          sheet["dt"])
    if kh is not None:
        kh["cpu_baseline"] = cpu_kh(
            dict(model="srmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
                 endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="flow",
                 integrator="rk2"), initial.kelvin_helmholtz(64, 128, seed=1234))
    if ensemble is not None:
        ensemble["cpu_baseline"] = cpu_ensemble(initial)


def long_run_l1(mb, initial, ranks, n, steps=500):
    """Mixed against plain after the configuration's full 500 updateTime calls."""
    st = {}
    for prec in ("fp64", "mixed"):
        sim = mb.Simulation(nx=n, ny=n, precision=prec, device=ranks.local, **CFG)
        sim.set_prims(initial.orszag_tang(n, Ng=4))
        sim.update_time(steps)
        c, p, _ = sim.state()
        s = sim.stats()
        st[prec] = (interior(c), interior(p), s)
        sim.close()
    out = {"steps": steps, "t": st["fp64"][2]["t"]}
    for k, name in enumerate(("cons", "prims")):
        a, b = st["mixed"][k], st["fp64"][k]
        d = np.abs(a - b)
        out[name] = {"l1_rel": float(d.sum() / np.abs(b).sum()), "max_abs": float(d.max())}
    return out


def roofline_of(sim, dt, peak, reps=3):
    ks = sim.profile_step(dt, reps=reps)
    top = max(ks, key=lambda k: k["total_ms"])
    avg_ms = top["total_ms"] / top["launches"]
    achieved = top["bytes_per_launch"] / (avg_ms * 1e-3) / 1e9
    return ks, top, {"kernel": top["name"], "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "avg_launch_ms": round(avg_ms, 4),
                     "bytes_per_launch": top["bytes_per_launch"]}


def ncu_record(kernel):
    """The committed ncu figures of `kernel` (profiles/ncu_traffic.json), or {}."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return {}
    with open(p) as f:
        return json.load(f).get(kernel) or {}


def fp64_pipe_roofline(inst_per_cell, cells, launch_ms, clk):
    """The FP64 pipe's roofline of a kernel whose FP64 work bounds it: thread
    instructions (DADD + DMUL + DFMA, counted by ncu per interior cell) per
    launch over the CUDA-event launch time, against 64 FP64 thread
    instructions per SM per clock (ncu's peak_sustained of
    sm__sass_thread_inst_executed_op_dfma_pred_on on B200) x SMs x the median
    SM clock sampled during the timed region."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz")
    if not mhz:
        return None
    achieved = inst_per_cell * cells / (launch_ms * 1e-3) / 1e9
    peak = 64 * sms * mhz * 1e6 / 1e9
    return {"unit": "G thread-inst/s", "inst_per_cell": inst_per_cell,
            "achieved": round(achieved, 1), "peak": round(peak, 1),
            "frac": round(achieved / peak, 4), "sm_mhz": mhz}


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    return ncu_record(kernel).get("dram_bytes_per_launch_full_size")


def cpu_baseline(n, steps=2):
    """The reference CPU build (serial) on the same workload, bounded sample."""
    from method_b200 import initial
    prims = initial.orszag_tang(n, Ng=4)
    try:
        from oracle import ref
        if not ref.available():
            raise FileNotFoundError
        sim = ref.RefSim(prims=prims, nx=n, ny=n, **CFG)
        kind = "reference"
    except (FileNotFoundError, OSError):
        from oracle import port
        sim = port.PortSim(prims, nx=n, ny=n, **CFG)
        kind = "port"
    dt = steady_dt(n)
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step_dt(dt)
    el = time.perf_counter() - t0
    return {"value": n * n * steps / el, "unit": "zone-updates/s", "cores": 1, "kind": kind,
            "sample": f"{steps} RK2 steps of the {n}x{n} grid, serial build (-O3), "
                      f"{el:.1f} s on the host"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    n = args.n
    out = {"metric": "zone-updates/s", "impl": "reference", "unit": "zone-updates/s",
           "n_gpus": args.gpus, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "n": n}}
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from method_b200 import initial
    from oracle import ref
    prims = initial.orszag_tang(n, Ng=4)
    dt = steady_dt(n)
    if ref.available(omp=True):
        sim = ref.RefSim(prims=prims, omp=True, nx=n, ny=n, **CFG)
        kind = "reference"
    else:
        from oracle import port
        sim = port.PortSim(prims, nx=n, ny=n, **CFG)
        kind, threads = "port", 1
    warm = min(args.warmup, 1)
    timed = max(1, min(args.steps, 3))
    for _ in range(warm):
        sim.step_dt(dt)
    t0 = time.perf_counter()
    for _ in range(timed):
        sim.step_dt(dt)
    el = time.perf_counter() - t0
    v = n * n * timed / el
    out.update({"value": v, "steps": timed, "warmup": warm, "ms_per_step": el / timed * 1e3,
                "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": threads,
                                 "kind": kind,
                                 "sample": f"{timed} RK2 steps of the {n}x{n} grid after {warm} "
                                           f"warm-up, OpenMP build, {threads} threads"},
                "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}})
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--forms", default="plain,mixed,mixed_mlp",
                    help="forms to run (profiling runs one at a time)")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-c2p-batch", action="store_true")
    ap.add_argument("--no-sheet", action="store_true", help="skip the SSP2 current sheet")
    ap.add_argument("--no-kh", action="store_true", help="skip the whole KH 64x128 run")
    ap.add_argument("--no-long-l1", action="store_true", help="skip the 500-step L1 check")
    ap.add_argument("--no-regime", action="store_true", help="skip the REGIME RKSplit workload")
    ap.add_argument("--no-hybrid", action="store_true", help="skip the Hybrid RKSplit2 workload")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import method_b200 as mb
    from method_b200 import initial
    from method_b200.ranks import Ranks

    ranks = Ranks("nccl", timeout_s=120)
    world, rank, local = ranks.world, ranks.rank, ranks.local
    barrier, max_over_ranks = ranks.barrier, ranks.max

    n = args.n
    dt = steady_dt(n)
    prims0 = initial.orszag_tang(n, Ng=4)
    peak, peak_kind = measured_peaks()
    K, W = args.steps, args.warmup
    results = {}
    clocks = Clocks(local)
    forms = [f for f in ("plain", "mixed", "mixed_mlp") if f in args.forms.split(",")]
    guess = None
    train = None
    if "mixed_mlp" in forms or not args.no_ensemble or not args.no_c2p_batch:
        t0 = time.perf_counter()
        P, S, loss = mb.train_guess(device=local)
        train = {"loss": loss, "seconds": round(time.perf_counter() - t0, 2),
                 "samples": 1 << 19, "iterations": 4000, "batch": 8192}
        guess = (P, S)
    guess_r = None
    if not args.no_ensemble or not args.no_sheet:
        t0 = time.perf_counter()
        Pr, Sr, loss_r = mb.train_guess(device=local, model="srrmhd")
        guess_r = (Pr, Sr)
        if train is not None:
            train["srrmhd"] = {"loss": loss_r, "seconds": round(time.perf_counter() - t0, 2)}
    ensemble = None
    with clocks:
        for form in forms:
            prec = "fp64" if form == "plain" else "mixed"
            sim, stream, ev0, ev1 = run_form(mb, torch, prims0, n, prec, K, W, dt, local,
                                             guess if form == "mixed_mlp" else None)
            sim.reset_stats()
            barrier()
            ev0.record(stream)
            for _ in range(K):
                sim.step(dt, sync=False)
            ev1.record(stream)
            barrier()
            sim.sync()
            ms = ev0.elapsed_time(ev1)
            ms = max_over_ranks(ms)
            st = sim.stats()
            c, p, a = sim.state()
            results[form] = dict(sim=sim, ms=ms, stats=st, cons=interior(c), prims=interior(p))
        if not args.no_ensemble:
            ke, we = max(1, min(K, 20)), max(W, 3)
            ensemble = run_ensemble(mb, initial, torch, ranks, ke, we, None)
            if guess:
                e_mlp = run_ensemble(mb, initial, torch, ranks, ke, we, guess, guess_r)
                ensemble["with_learned_guess"] = {
                    k: e_mlp[k] for k in ("value", "ms_per_step", "c2p_newton_iters_per_cell",
                                          "implicit_iters_per_cell", "c2p_unconverged",
                                          "c2p_fallbacks", "implicit_fallbacks",
                                          "implicit_failed")}
                ensemble["with_learned_guess"]["networks"] = "SRMHD and SRRMHD members" \
                    if guess_r else "SRMHD members"
        c2p_batch = None
        want_cpu = rank == 0 and world == 1 and not args.no_cpu
        if not args.no_c2p_batch:
            c2p_batch = run_c2p_batch(mb, torch, ranks, guess, cpu=want_cpu)
        sheet = None
        if not args.no_sheet:
            sheet = run_sheet(mb, initial, torch, ranks, max(K // 5, 5), max(W, 3), peak,
                              cpu=False, guess_r=guess_r)
        kh = None
        if not args.no_kh:
            kh = run_kh_full(mb, initial, torch, ranks, peak, cpu=False)
        regime = None
        if not args.no_regime:
            regime = run_regime(mb, initial, torch, ranks, n, max(K // 5, 5), max(W, 3), peak)
        hybrid = None
        if not args.no_hybrid:
            hybrid = run_hybrid(mb, initial, torch, ranks, n, max(K // 20, 3), 3)
    clk = clocks.summary()
    if regime is not None:  # what bounds the tile (ncu figures of a 768^2 capture)
        for form, key in (("plain", "regime_tile_fp64"), ("mixed", "regime_tile_mixed")):
            rec, rg = ncu_record(key), regime[form]["regime"]
            rg["ncu"] = {k: rec[k] for k in ("fp64_pipe_active_pct", "fma_pipe_active_pct",
                                             "issue_active_pct", "warps_active_pct")
                         if k in rec} or None
            if rec.get("fp64_thread_inst_per_cell"):
                rg["fp64_pipe"] = fp64_pipe_roofline(rec["fp64_thread_inst_per_cell"],
                                                     regime["n"] ** 2, rg["ms_per_launch"], clk)
    long_l1 = None if args.no_long_l1 else long_run_l1(mb, initial, ranks, n)
    if want_cpu:  # reference-build baselines on the host, after the timed GPU work
        with quiet_stdout():
            cpu_legs(initial, sheet, kh, ensemble, regime, hybrid)

    cells = n * n
    for form in forms:
        r = results[form]
        ks, top, roof = roofline_of(r["sim"], dt, peak)
        roof["peak_kind"] = peak_kind + " (burst copy bandwidth, kernel timed alone)"
        roof["traffic"] = ncu_traffic(top["name"])
        # what bounds the kernel instead (ncu, small case of the same workload)
        rec = ncu_record(top["name"])
        roof["ncu_pipes"] = {k: rec[k] for k in ("fp64_pipe_active_pct", "fma_pipe_active_pct",
                                                 "issue_active_pct", "warps_active_pct")
                             if k in rec} or None
        if rec.get("fp64_thread_inst_per_cell"):
            roof["fp64_pipe"] = fp64_pipe_roofline(rec["fp64_thread_inst_per_cell"], cells,
                                                   roof["avg_launch_ms"], clk)
        launches_per_step = sum(k["launches"] for k in ks) / 3.0
        r.update(roof=roof, kernels=ks, launches_per_step=launches_per_step)
        st = r["stats"]
        r["summary"] = {
            "value": world * cells * K / (r["ms"] * 1e-3),
            "ms_per_step": r["ms"] / K,
            "c2p_evals_per_cell": st["c2p_evals"] / max(st["c2p_cells"], 1),
            "c2p_unconverged": st["c2p_unconverged"],
            "roofline": roof,
            "step_roofline": {"bytes_per_zone_update": 616, "achieved_gbs": round(
                616 * cells / (r["ms"] / K * 1e-3) / 1e9, 1), "peak": peak},
            "kernels": [{"name": k["name"], "launches_per_step": k["launches"] / 3.0,
                         "ms_per_launch": round(k["total_ms"] / k["launches"], 4)} for k in ks],
        }
    if not {"plain", "mixed"} <= set(forms):
        if rank == 0:
            print(json.dumps({f: results[f]["summary"] for f in forms}), flush=True)
        for r in results.values():
            r["sim"].close()
        ranks.close()
        return
    # L1 of the mixed form against the FP64 result (bit-identical to the reference)
    l1 = {}
    for form in [f for f in forms if f != "plain"]:
        for name in ("cons", "prims"):
            ref_, mix = results["plain"][name], results[form][name]
            d = np.abs(mix - ref_)
            key = name if form == "mixed" else f"{form}_{name}"
            l1[key] = {"l1_abs": float(d.mean()), "l1_rel": float(d.sum() / np.abs(ref_).sum()),
                       "max_abs": float(d.max())}

    # end to end through the reference-facing call on host arrays (mixed form)
    e2e = None
    if args.e2e_steps > 0:
        sim = mb.Simulation(nx=n, ny=n, precision="mixed", device=local, **CFG)
        sim.set_prims(prims0)
        hc, hp, ha = sim.state()
        for arr in (hc, hp, ha):
            mb.pin_host(arr)
        sim.step_host(hc, hp, ha, dt)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            sim.step_host(hc, hp, ha, dt)
        el = max_over_ranks(time.perf_counter() - t0)
        for arr in (hc, hp, ha):
            mb.unpin_host(arr)
        # the library reports what one call copies: the variables the step reads
        # in, all of cons / prims / aux out
        h2d, d2h = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        if sim.L.mth_step_host_bytes(sim.h, ctypes.byref(h2d), ctypes.byref(d2h)) != 0:
            raise RuntimeError("mth_step_host_bytes failed")
        e2e = {"value": world * cells * args.e2e_steps / el, "unit": "zone-updates/s",
               "h2d_bytes_per_step": int(h2d.value), "d2h_bytes_per_step": int(d2h.value),
               "call": "mth_step_host (TimeIntegrator::step on host arrays), mixed form",
               "steps": args.e2e_steps}
        sim.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        with quiet_stdout():
            cpu = cpu_baseline(n)

    if rank == 0:
        m = results["mixed"]["summary"]
        line = {
            "metric": "zone-updates/s", "value": m["value"], "unit": "zone-updates/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": m["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 flux / f64 c2p+state", "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": "mixed (FP32 flux, FP64 Newton C2P, "
                                                      "previous-step guess)",
                       "n": n, "cells_per_gpu": cells, "dt": "fixed steady-state CFL dt",
                       "l2": "inputs larger than L2 (device state 0.5 GB per form)",
                       "parallelism": f"replicas x{world}"},
            "roofline": results["mixed"]["roof"],
            "plain": {**results["plain"]["summary"], "dtype": "f64"},
            "mixed": results["mixed"]["summary"],
            "mixed_mlp": results["mixed_mlp"]["summary"] if "mixed_mlp" in results else None,
            "guess_training": train,
            "l1_mixed_vs_fp64": l1,
            "l1_mixed_vs_fp64_500_steps": long_l1,
            "kh64x128_full_run": kh,
            "regime_rksplit": regime,
            "hybrid_rksplit2": hybrid,
            "sheet_ssp2": sheet,
            "ensemble": ensemble,
            "c2p_batch": c2p_batch,
            "speedup_mixed_vs_plain": results["plain"]["ms"] / results["mixed"]["ms"],
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "gpu_launches": int(round(results["mixed"]["launches_per_step"] * K)),
        }
        print(json.dumps(line), flush=True)
    for r in results.values():
        r["sim"].close()
    ranks.close()


if __name__ == "__main__":
    main()
