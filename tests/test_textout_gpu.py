"""SerialSaveData text output (mth_save_text) against the reference's own
SerialSaveData files, byte for byte, and the device "%.16f" formatter against
correctly rounded formatting on values chosen to stress it (ties, carries into
the integer part, subnormals, huge integers, infinities, NaNs, signed zero)."""
import math
import os
import tempfile

import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu

SUBDIRS = ("Conserved", "Primitive", "Auxiliary", "Domain", "Constants")
FILES = ("Conserved/cons{}.dat", "Primitive/prims{}.dat", "Auxiliary/aux{}.dat",
         "Domain/domain{}.dat", "Constants/constants{}.dat")


def _outdir():
    d = tempfile.mkdtemp(prefix="mt", dir="/tmp")  # the reference keeps dir in char[50]
    for s in SUBDIRS:
        os.makedirs(os.path.join(d, s))
    return d


CASES = {
    "ot2d_rk2": (dict(model="srmhd", nx=24, ny=20, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
                      endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="periodic",
                      integrator="rk2"),
                 lambda: np.ascontiguousarray(initial.orszag_tang(24)[:, :32, :28]), 4),
    "sheet_ssp2": (dict(model="srrmhd", nx=16, ny=24, xmin=-0.5, xmax=0.5, ymin=-1.0,
                        ymax=1.0, endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3,
                        weno=3, bcs="outflow", integrator="ssp2"),
                   lambda: initial.current_sheet(16, 24, seed=5), 2),
}


@pytest.mark.parametrize("case", list(CASES))
def test_files_match_reference(ref, case):
    import method_b200 as mb
    cfg, mk, steps = CASES[case]
    p = mk()
    r = ref.RefSim(prims=p, **cfg)
    g = mb.Simulation(**cfg)
    g.set_prims(p)
    for n in (0, steps):
        if n:
            assert r.update_time(n) == 0
            g.update_time(n)
        dr, dg = _outdir(), _outdir()
        assert r.save_text(dr, str(n)) == 0
        g.save_text(dg, str(n))
        for f in FILES:
            a = open(os.path.join(dr, f.format(n)), "rb").read()
            b = open(os.path.join(dg, f.format(n)), "rb").read()
            assert a == b, (case, n, f)


def test_3d_and_1d_layouts_match_reference(ref):
    """3D rows (one line per (var, i, j)) and 1D lines, plus collapsed-axis
    domain and constants lines."""
    import method_b200 as mb
    n = 6
    x = (np.arange(n + 8) + 0.5 - 4) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    p = np.zeros((8, n + 8, n + 8, n + 8))
    p[0] = 1.0 + 0.1 * np.sin(2 * np.pi * X)
    p[4] = 1.0
    p[1] = 0.2 * np.sin(2 * np.pi * Y)
    p[3] = 0.1 * np.sin(2 * np.pi * Z)
    cfg3 = dict(model="srmhd", nx=n, ny=n, nz=n, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0,
                zmax=1, endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="periodic",
                integrator="rk2")
    cfg1 = dict(model="srmhd", nx=40, ny=0, xmin=0, xmax=1, ymin=0, ymax=1, endTime=0.4,
                cfl=0.4, Ng=4, gamma=2.0, weno=3, bcs="outflow", integrator="rk2")
    for cfg, init in ((cfg3, None), (cfg1, "briowu")):
        if init:
            r = ref.RefSim(init=init, init_arg0=0, **cfg)
            _, prims, _ = r.state()
        else:
            prims = p
            r = ref.RefSim(prims=prims, **cfg)
        g = mb.Simulation(**cfg)
        g.set_prims(prims)
        r.update_time(1)
        g.update_time(1)
        dr, dg = _outdir(), _outdir()
        assert r.save_text(dr, "") == 0
        g.save_text(dg, "")
        for f in FILES:
            a = open(os.path.join(dr, f.format("")), "rb").read()
            b = open(os.path.join(dg, f.format("")), "rb").read()
            assert a == b, (cfg["nx"], cfg["ny"], f)


def _expected(v):
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    if math.isinf(v):
        return "-inf" if v < 0 else "inf"
    return "%.16f" % v  # correctly rounded, ties to even


def test_formatter_edge_values():
    import method_b200 as mb
    specials = [0.0, -0.0, 1.0, -1.0, 0.5, 2.0 ** -17, 3 * 2.0 ** -17, 2.0 ** -18,
                -5 * 2.0 ** -18, 0.99999999999999995, 0.99999999999999994, 9.99999999999999995,
                123456789.123456789, 2.0 ** 53, 2.0 ** 53 + 2, 2.0 ** 63, 2.0 ** 64, 1e20, 1e22,
                1.7976931348623157e308, -1e300, 5e-324, 2.2250738585072014e-308, 1e-17, 5e-17,
                4.9999999999999996e-17, 1.5e-16, float("inf"), float("-inf"), float("nan"),
                -float("nan"), math.pi, -math.e, 1.0 / 3.0]
    rng = np.random.default_rng(7)
    rand = list(rng.standard_normal(200) * 10.0 ** rng.integers(-20, 20, 200))
    rand += list(rng.integers(-2 ** 62, 2 ** 62, 50).astype(np.float64))
    vals = np.array(specials + rand, dtype=np.float64)
    nx = len(vals)
    cfg = dict(model="srmhd", nx=nx, ny=0, xmin=0, xmax=1, ymin=0, ymax=1, endTime=1.0,
               cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="outflow", integrator="rk2")
    g = mb.Simulation(**cfg)
    cons = np.zeros((9, nx + 8, 1, 1))
    for v in range(9):
        cons[v, 4:-4, 0, 0] = vals * (1 if v % 2 == 0 else -1)
    g.upload(cons=cons)
    d = _outdir()
    g.save_text(d, "e", which=1)
    lines = open(os.path.join(d, "Conserved/conse.dat")).read().split("\n")
    assert lines[0] == "cons = D, Sx, Sy, Sz, tau, Bx, By, Bz, phi"
    body = lines[1:-1]
    assert len(body) == 9 * nx and lines[-1] == ""
    for v in range(9):
        for q in range(nx):
            x = cons[v, 4 + q, 0, 0]
            assert body[v * nx + q] == _expected(x) + " ", (v, q, x, body[v * nx + q])
