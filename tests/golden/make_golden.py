"""Generates the golden fixtures of tests/golden/ from the reference CPU build.

    make -C oracle REF=/path/to/METHOD      # builds oracle/_ref/libmethod_ref.so
    python tests/golden/make_golden.py

Each fixture runs one small workload through the UNMODIFIED reference
classes (Simulation::updateTime, Project/CPU/Src/simulation.cc:104-133) and
stores the initial primitive array and the final interior state.  The cases
restate the reference's own consistency tests (Tests/CPU/Src/test_rk2.cc,
test_rkSplit.cc, test_imex.cc) and the measured workloads at reduced size.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from method_b200 import initial  # noqa: E402
from oracle import ref  # noqa: E402

CASES = {
    # name: (config, init, builtin-init kwargs, steps)
    "ot16_rk2_weno3_periodic": (
        dict(model="srmhd", nx=16, ny=16, xmin=0, xmax=1, ymin=0, ymax=1, endTime=0.004, cfl=0.6,
             Ng=4, gamma=2.0, weno=3, bcs="periodic", integrator="rk2"),
        None, dict(init="ot"), 2),
    "ot16_rk2_weno5_outflow": (
        dict(model="srmhd", nx=16, ny=16, xmin=0, xmax=1, ymin=0, ymax=1, endTime=1.0, cfl=0.4,
             Ng=4, gamma=4.0 / 3.0, weno=5, bcs="outflow", integrator="rk2"),
        lambda: initial.orszag_tang(16, Ng=4), {}, 3),
    "kh16x32_rk2_weno3_flow": (
        dict(model="srmhd", nx=16, ny=32, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0, endTime=3.0,
             cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="flow", integrator="rk2"),
        lambda: initial.kelvin_helmholtz(16, 32, Ng=4, seed=11), {}, 5),
    "khrandom16_rksplit_flow": (
        dict(model="srmhd", nx=16, ny=16, xmin=0, xmax=1, ymin=0, ymax=1, endTime=0.004, cfl=0.6,
             Ng=4, gamma=4.0 / 3.0, sigma=10.0, cp=1.0, weno=3, bcs="flow",
             integrator="rksplit"),
        None, dict(init="khrandom", init_arg0=1, init_arg1=10), 1),
    "sheet16x32_ssp2_outflow": (
        dict(model="srrmhd", nx=16, ny=32, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0, endTime=3.0,
             cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=100.0, weno=3, bcs="outflow",
             integrator="ssp2"),
        lambda: initial.current_sheet(16, 32, Ng=4, seed=5), {}, 2),
    "kh16x32_srrmhd_rk2_flow": (
        dict(model="srrmhd", nx=16, ny=32, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0, endTime=3.0,
             cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=10.0, weno=3, bcs="flow", integrator="rk2"),
        lambda: initial.kelvin_helmholtz(16, 32, Ng=4, seed=3, model="srrmhd"), {}, 3),
    "briowu64_rk2_outflow_1d": (
        dict(model="srmhd", nx=64, ny=0, xmin=0, xmax=1, ymin=0, ymax=1, endTime=0.4, cfl=0.4,
             Ng=4, gamma=2.0, weno=3, bcs="outflow", integrator="rk2"),
        None, dict(init="briowu", init_arg0=0), 4),
}


def interior(a, Ng, dims):
    sl = [slice(None), slice(Ng, -Ng)]
    sl.append(slice(Ng, -Ng) if dims > 1 else slice(None))
    sl.append(slice(Ng, -Ng) if dims > 2 else slice(None))
    return a[tuple(sl)]


def main():
    if not ref.available():
        sys.exit("oracle/_ref/libmethod_ref.so is missing; run `make -C oracle` first")
    for name, (cfg, mk, binit, steps) in CASES.items():
        prims0 = mk() if mk else None
        r = ref.RefSim(prims=prims0, **cfg, **binit)
        if prims0 is None:
            _, prims0, _ = r.state()
        r.update_time(steps)
        c, p, a = r.state()
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, prims0=prims0, cons=interior(c, cfg["Ng"], r.dims),
                            prims=interior(p, cfg["Ng"], r.dims),
                            aux=interior(a, cfg["Ng"], r.dims), steps=steps, t=r.t,
                            config=repr(cfg))
        print(f"{name}: {os.path.getsize(out)} bytes, t = {r.t}")


if __name__ == "__main__":
    main()
