"""Initial data of the benchmark workloads (project InitialFunc subclasses).

METHOD sets initial data by filling ``d->prims`` for every cell, ghosts
included, in an InitialFunc subclass (Project/CPU/Src/initFunc.cc:10-40); the
simulation then derives cons/aux with Model::primsToAll.  These functions
return that primitive array (shape (Nprims, Nx, Ny, Nz), reference layout)
for the workloads measured here, which differ from the reference's own
InitialFunc classes:

* ``kelvin_helmholtz``: SRMHD / SRRMHD shear layers at y = +-0.5 of width
  0.01, rho = 1, p = 1, seeded uniform random vy of amplitude 0.01;
* ``orszag_tang``: rho = 1, p = 1, v = (-0.5 sin 2pi y, 0.5 sin 2pi x),
  B = (-sin 2pi y, sin 4pi x);
* ``current_sheet``: SRRMHD Harris-like sheet By = tanh(x / 0.01), rho = 1,
  p = 50, seeded velocity noise 1e-3 and ideal E = -v x B;
* ``random_c2p_states``: per-cell random SRMHD states for the primitive
  recovery workload (W, rho, p/rho, b^2/rho log-uniform, isotropic
  directions).

Cell centres follow Simulation's axes, x_i = xmin + (i + 0.5 - Ng) dx
(simulation.cc:48-61).  Transcendental functions are evaluated on the host
once, so every consumer of the array sees identical bits.
"""
from __future__ import annotations

import numpy as np

NPRIMS = {"srmhd": 8, "srrmhd": 11}


def axes(nx, ny, nz, Ng, xmin, xmax, ymin, ymax, zmin=0.0, zmax=1.0):
    Nx = nx + 2 * Ng
    Ny = ny + 2 * Ng if ny > 0 else 1
    Nz = nz + 2 * Ng if nz > 0 else 1
    dx = (xmax - xmin) / nx
    x = xmin + (np.arange(Nx) + 0.5 - Ng) * dx
    y = ymin + (np.arange(Ny) + 0.5 - Ng) * ((ymax - ymin) / ny) if ny > 0 else np.zeros(1)
    z = zmin + (np.arange(Nz) + 0.5 - Ng) * ((zmax - zmin) / nz) if nz > 0 else np.zeros(1)
    return x, y, z


def _ideal_E(p):
    # E = -v x B (initFunc.cc:553-558)
    p[8] = -(p[2] * p[7] - p[3] * p[6])
    p[9] = -(p[3] * p[5] - p[1] * p[7])
    p[10] = -(p[1] * p[6] - p[2] * p[5])


def kelvin_helmholtz(nx=64, ny=128, Ng=4, seed=1234, model="srmhd", shear=0.5, width=0.01,
                     amp=0.01):
    x, y, _ = axes(nx, ny, 0, Ng, -0.5, 0.5, -1.0, 1.0)
    Nx, Ny = len(x), len(y)
    p = np.zeros((NPRIMS[model], Nx, Ny, 1))
    Y = np.broadcast_to(y[None, :], (Nx, Ny))
    p[0] = 1.0
    p[4] = 1.0
    vx = np.where(Y > 0, shear * np.tanh((Y - 0.5) / width), -shear * np.tanh((Y + 0.5) / width))
    p[1, :, :, 0] = vx
    rng = np.random.default_rng(seed)
    p[2, :, :, 0] = amp * rng.uniform(-1.0, 1.0, size=(Nx, Ny))
    if model == "srrmhd":
        _ideal_E(p)
    return p


def orszag_tang(n=1024, Ng=4, model="srmhd"):
    x, y, _ = axes(n, n, 0, Ng, 0.0, 1.0, 0.0, 1.0)
    X, Y = np.meshgrid(x, y, indexing="ij")
    p = np.zeros((NPRIMS[model], len(x), len(y), 1))
    p[0] = 1.0
    p[4] = 1.0
    p[1, :, :, 0] = -0.5 * np.sin(2 * np.pi * Y)
    p[2, :, :, 0] = 0.5 * np.sin(2 * np.pi * X)
    p[5, :, :, 0] = -np.sin(2 * np.pi * Y)
    p[6, :, :, 0] = np.sin(4 * np.pi * X)
    if model == "srrmhd":
        _ideal_E(p)
    return p


def current_sheet(nx=512, ny=1024, Ng=4, seed=1234, width=0.01, noise=1e-3, pressure=50.0):
    x, y, _ = axes(nx, ny, 0, Ng, -0.5, 0.5, -1.0, 1.0)
    Nx, Ny = len(x), len(y)
    p = np.zeros((11, Nx, Ny, 1))
    X = np.broadcast_to(x[:, None], (Nx, Ny))
    rng = np.random.default_rng(seed)
    p[0] = 1.0
    p[4] = pressure
    p[6, :, :, 0] = np.tanh(X / width)
    for v in (1, 2, 3):
        p[v, :, :, 0] = noise * rng.uniform(-1.0, 1.0, size=(Nx, Ny))
    _ideal_E(p)
    return p


def sigma_for_seed(seed, lo=1.0, hi=5.0):
    """Conductivity 10^U(lo, hi) of one resistive run."""
    return float(10.0 ** np.random.default_rng(seed).uniform(lo, hi))


def random_c2p_states(n, seed=1234, gamma=4.0 / 3.0):
    """Random SRMHD primitive states, shape (8, n): W log-uniform in [1, 10],
    rho in [1e-3, 1], p/rho in [1e-3, 10], comoving b^2/rho in [1e-2, 1e2],
    isotropic velocity and field directions."""
    rng = np.random.default_rng(seed)
    W = 10.0 ** rng.uniform(0.0, 1.0, n)
    rho = 10.0 ** rng.uniform(-3.0, 0.0, n)
    prs = rho * 10.0 ** rng.uniform(-3.0, 1.0, n)
    sig = 10.0 ** rng.uniform(-2.0, 2.0, n)

    def unit(k):
        v = rng.normal(size=(3, k))
        return v / np.linalg.norm(v, axis=0)

    vhat, bhat = unit(n), unit(n)
    vmag = np.sqrt(1.0 - 1.0 / (W * W))
    v = vhat * vmag
    # choose |B| so that the comoving b^2 = (B^2 + W^2 (v.B)^2) / W^2 matches sig * rho
    vb = np.sum(vhat * bhat, axis=0) * vmag
    Bmag = np.sqrt(sig * rho * W * W / (1.0 + W * W * vb * vb))
    B = bhat * Bmag
    p = np.zeros((8, n))
    p[0], p[1:4], p[4], p[5:8] = rho, v, prs, B
    return p


def kh_ensemble(n=256, seed=2024, nx_lo=64, nx_hi=512, weno=3, precision="mixed"):
    """Members of a Kelvin-Helmholtz parameter study: per member nx uniform
    in [nx_lo, nx_hi], ny = 2 nx, shear speed uniform in [0.2, 0.8], and with
    probability 1/2 a resistive (SRRMHD, IMEX SSP2) member with sigma
    log-uniform in [1e2, 1e5], else ideal (SRMHD, RK2).  Returns a list of
    (config dict for Simulation / Ensemble, kelvin_helmholtz keyword dict)."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        nx = int(rng.integers(nx_lo, nx_hi + 1))
        shear = float(rng.uniform(0.2, 0.8))
        resistive = bool(rng.random() < 0.5)
        sigma = float(10.0 ** rng.uniform(2.0, 5.0)) if resistive else 0.0
        cfg = dict(model="srrmhd" if resistive else "srmhd",
                   integrator="ssp2" if resistive else "rk2", nx=nx, ny=2 * nx, xmin=-0.5,
                   xmax=0.5, ymin=-1.0, ymax=1.0, endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0,
                   sigma=sigma, weno=weno, bcs="flow", precision=precision)
        ic = dict(nx=nx, ny=2 * nx, Ng=4, seed=int(seed) * 1000 + m,
                  model=cfg["model"], shear=shear)
        out.append((cfg, ic))
    return out
