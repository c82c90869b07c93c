"""CPU tests of the oracle (oracle/oracle.c): pinned to the reference.

1. Known answers restated from the reference's own unit tests
   (Tests/CPU/Src/test_weno.cc, test_cminpack.cc, test_srmhd.cc,
   test_simulation.cc).
2. The committed golden fixtures (tests/golden/*.npz, made from the reference
   build by tests/golden/make_golden.py) reproduced exactly.
3. Live bit-for-bit comparison with the reference build when oracle/_ref was
   built in this checkout.
"""
import glob
import os

import numpy as np
import pytest

from method_b200 import initial
from oracle import port

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def interior(a, Ng, dims):
    sl = [slice(None), slice(Ng, -Ng)]
    sl.append(slice(Ng, -Ng) if dims > 1 else slice(None))
    sl.append(slice(Ng, -Ng) if dims > 2 else slice(None))
    return a[tuple(sl)]


# --------------------------------------------------------------------- KATs
def test_weno3_known_answers():
    # test_weno.cc:36-79: upwind of (0, 1, 2) at the face -> 1.5; downwind -> 0.5
    assert abs(port.weno3_upwind(0.0, 1.0, 2.0) - 1.5) < 1e-15
    assert abs(port.weno3_upwind(2.0, 1.0, 0.0) - 0.5) < 1e-15


def test_weno5_known_answer():
    # test_weno.cc:161-180: linear data is reconstructed exactly
    assert abs(port.weno5_upwind(0.0, 1.0, 2.0, 3.0, 4.0) - 2.5) < 1e-15


def test_hybrd1_known_answers():
    # test_cminpack.cc:33-79
    info, x, _ = port.hybrd1_kat(0, [0.0, 0.0])
    assert info == 1
    assert abs(x[0] + 4.0) < 1.49011612e-8 and abs(x[1] - 2.5) < 1.49011612e-8
    info, _, _ = port.hybrd1_kat(0, [0.0, 0.0], n=6, lwa=19)
    assert info == 0
    info, _, _ = port.hybrd1_kat(1, list(x))
    assert info == 4
    info, _, f = port.hybrd1_kat(2, [0.0, 1.0])
    assert info == 1 and abs(f[0]) < 1.49011612e-8 and abs(f[1]) < 1.49011612e-8


def test_srmhd_prims_to_all_known_answer():
    # test_srmhd.cc:228-282: all prims 1e-16 -> cons ~ 0, h = 3.5, W = 1, e = 1.5, c = sqrt(10/21)
    cfg = dict(model="srmhd", nx=10, ny=10, nz=10, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1,
               endTime=1.0, bcs="periodic")
    p = np.full((8, 18, 18, 18), 1e-16)
    s = port.PortSim(p, **cfg)
    c, _, a = s.state()
    assert np.all(np.abs(c) < 1e-15)
    assert np.all(a[0] == 3.5)
    assert np.all(np.abs(a[1] - 1.0) < 1e-15)
    assert np.all(a[2] == 1.5)
    assert np.all(a[3] == np.sqrt(10.0 / 21.0))
    assert np.all(np.abs(a[4:]) < 1e-15)


def test_dt_known_answer():
    # test_simulation.cc:40-62: Data(100, 10, 2, 0, 1, -0.5, 0.5, -0.1, 0.1, 0.8), cfl 0.5
    cfg = dict(model="srmhd", nx=100, ny=10, nz=2, xmin=0, xmax=1, ymin=-0.5, ymax=0.5,
               zmin=-0.1, zmax=0.1, endTime=0.8, cfl=0.5, Ng=4, bcs="outflow")
    p = np.zeros((8, 108, 18, 10))
    p[0] = 1.0
    p[4] = 1.0
    s = port.PortSim(p, **cfg)
    assert abs(s.dt - 0.002886751346) < 1e-11
    assert s.dx == 0.01 and s.dy == 0.1


def ot_vortex_prims(n=10, Ng=4):
    """Orszag-Tang data of the reference's OTVortexSingleFluid (initFunc.cc:229-272)."""
    PI = 3.14159265358979323
    x = 0.0 + (np.arange(n + 2 * Ng) + 0.5 - Ng) * (1.0 / n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    p = np.zeros((8, n + 2 * Ng, n + 2 * Ng, 1))
    p[0] = 25.0 / 36.0 / PI
    p[4] = 5.0 / 12.0 / PI
    p[5, :, :, 0] = -np.sin(2.0 * PI * Y) / np.sqrt(4.0 * PI)
    p[6, :, :, 0] = np.sin(4.0 * PI * X) / np.sqrt(4.0 * PI)
    p[1, :, :, 0] = -0.5 * np.sin(2.0 * PI * Y)
    p[2, :, :, 0] = 0.5 * np.sin(2.0 * PI * X)
    return p


def test_srmhd_c2p_round_trip():
    # test_srmhd.cc:134-220: OT vortex prims -> cons -> prims to 1.49e-8, then
    # again from a guess scaled by 0.9
    tol = 1.49011612e-8
    s = port.PortSim(ot_vortex_prims(), model="srmhd", nx=10, ny=10, bcs="periodic")
    c, p0, a0 = s.state()
    p, a = p0.copy(), a0.copy()
    assert s.c2p(c, p, a) == 0
    assert np.max(np.abs(p - p0)) < tol and np.max(np.abs(a - a0)) < tol
    p, a = p0 * 0.9, a0 * 0.9
    assert s.c2p(c, p, a) == 0
    sl = (slice(None), slice(4, -4), slice(4, -4))
    assert np.max(np.abs(p[sl] - p0[sl])) < tol
    assert np.max(np.abs(a[sl] - a0[sl])) < tol


# ---------------------------------------------------------- golden fixtures
GOLDEN_FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


@pytest.mark.parametrize("path", GOLDEN_FILES, ids=[os.path.basename(p)[:-4] for p in GOLDEN_FILES])
def test_oracle_reproduces_golden(path):
    g = np.load(path, allow_pickle=False)
    cfg = eval(str(g["config"]))
    s = port.PortSim(g["prims0"], **cfg)
    assert s.update_time(int(g["steps"])) == 0
    c, p, a = s.state()
    assert s.t == float(g["t"])
    for name, mine in (("cons", c), ("prims", p), ("aux", a)):
        ref = g[name]
        got = interior(mine, cfg["Ng"], s.dims)
        assert np.array_equal(got, ref), f"{name}: max diff {np.max(np.abs(got - ref))}"


# ---------------------------------------------------- live reference check
LIVE = {
    "kh_weno3": (dict(model="srmhd", nx=32, ny=64, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
                      endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="flow",
                      integrator="rk2"), lambda: initial.kelvin_helmholtz(32, 64, seed=2), 20),
    "ot_weno5": (dict(model="srmhd", nx=48, ny=48, xmin=0, xmax=1, ymin=0, ymax=1, endTime=3.0,
                      cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=5, bcs="periodic", integrator="rk2"),
                 lambda: initial.orszag_tang(48), 10),
    "sheet_ssp2": (dict(model="srrmhd", nx=24, ny=48, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
                        endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3, weno=3,
                        bcs="outflow", integrator="ssp2"),
                   lambda: initial.current_sheet(24, 48, seed=9), 3),
    "sheet_ssp3": (dict(model="srrmhd", nx=16, ny=32, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
                        endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3, weno=3,
                        bcs="outflow", integrator="ssp3"),
                   lambda: initial.current_sheet(16, 32, seed=10), 2),
    "sheet_ssp2322": (dict(model="srrmhd", nx=16, ny=32, xmin=-0.5, xmax=0.5, ymin=-1.0,
                           ymax=1.0, endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3,
                           weno=3, bcs="periodic", integrator="ssp2322"),
                      lambda: initial.current_sheet(16, 32, seed=11), 2),
    # WENO7 / WENO9 / WENO11 (weno.cc:239-482), Ng = shift + 1
    "kh_weno7": (dict(model="srmhd", nx=32, ny=64, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
                      endTime=3.0, cfl=0.4, Ng=5, gamma=4.0 / 3.0, weno=7, bcs="flow",
                      integrator="rk2"), lambda: initial.kelvin_helmholtz(32, 64, Ng=5, seed=4), 6),
    "ot_weno9": (dict(model="srmhd", nx=32, ny=32, xmin=0, xmax=1, ymin=0, ymax=1, endTime=3.0,
                      cfl=0.4, Ng=6, gamma=4.0 / 3.0, weno=9, bcs="periodic", integrator="rk2"),
                 lambda: initial.orszag_tang(32, Ng=6), 4),
    "sheet_weno11_ssp2": (dict(model="srrmhd", nx=24, ny=48, xmin=-0.5, xmax=0.5, ymin=-1.0,
                               ymax=1.0, endTime=3.0, cfl=0.4, Ng=7, gamma=4.0 / 3.0, sigma=1e3,
                               weno=11, bcs="outflow", integrator="ssp2"),
                          lambda: initial.current_sheet(24, 48, Ng=7, seed=14), 2),
    # Data::functionalSigma: conductivity sigma * D^gam per cell (simData.cc:114-127)
    "sheet_ssp2_functional_sigma": (dict(model="srrmhd", nx=24, ny=48, xmin=-0.5, xmax=0.5,
                                         ymin=-1.0, ymax=1.0, endTime=3.0, cfl=0.4, Ng=4,
                                         gamma=4.0 / 3.0, sigma=1e3, weno=3, bcs="outflow",
                                         integrator="ssp2", functionalSigma=True, gam=12.0),
                                    lambda: _dense_sheet(24, 48, seed=12), 3),
    "kh_srrmhd_rk2_functional_sigma": (dict(model="srrmhd", nx=24, ny=48, xmin=-0.5, xmax=0.5,
                                            ymin=-1.0, ymax=1.0, endTime=3.0, cfl=0.4, Ng=4,
                                            gamma=4.0 / 3.0, sigma=10.0, weno=3, bcs="flow",
                                            integrator="rk2", functionalSigma=True, gam=3.0),
                                       lambda: _dense_kh(24, 48, seed=13), 4),
}


def _dense_sheet(nx, ny, seed):
    """Current sheet with a density that varies over the grid, so that a
    functional conductivity sigma * D^gam differs from cell to cell."""
    p = initial.current_sheet(nx, ny, seed=seed)
    p[0] *= 1.0 + 0.3 * np.sin(np.linspace(0, 3.0, p.shape[2]))[None, :, None]
    return p


def _dense_kh(nx, ny, seed):
    p = initial.kelvin_helmholtz(nx, ny, seed=seed, model="srrmhd")
    p[0] *= 1.0 + 0.2 * np.cos(np.linspace(0, 2.0, p.shape[1]))[:, None, None]
    return p


@pytest.mark.parametrize("case", list(LIVE))
def test_oracle_matches_reference_live(ref, case):
    cfg, mk, steps = LIVE[case]
    p = mk()
    r = ref.RefSim(prims=p, **cfg)
    o = port.PortSim(p, **cfg)
    r.update_time(steps)
    o.update_time(steps)
    for a, b in zip(r.state(), o.state()):
        assert np.array_equal(a, b)
