"""Ensembles of uneven 2D simulations against the same simulations run alone.

Every member of an ensemble must end bit-identical to a single Simulation of
its configuration after the same number of updateTime steps (plain FP64
members therefore match the reference bit for bit, which the single-simulation
parity tests establish), whatever tile heights the autotuner picked.  Member
sizes cover the three size classes (nx <= 96, <= 192, larger), interiors
that are not multiples of the 32-cell tile width, every boundary type, and a
member whose endTime clips dt.
"""
import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu

NSTEPS = 12


def _prims(kind, nx, ny, model, Ng):
    if kind == "ot":
        p = initial.orszag_tang(max(nx, ny), Ng=Ng, model=model)
        return np.ascontiguousarray(p[:, :nx + 2 * Ng, :ny + 2 * Ng])
    if kind == "kh":
        return initial.kelvin_helmholtz(nx, ny, Ng=Ng, model=model, seed=nx + ny)
    return initial.current_sheet(nx, ny, Ng=Ng, seed=nx * 7 + ny)


def _members(precision, weno):
    Ng = 4
    srmhd = [
        ("ot", dict(nx=64, ny=64, cfl=0.4, bcs="periodic")),
        ("kh", dict(nx=40, ny=72, cfl=0.3, bcs="flow", xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0)),
        ("ot", dict(nx=130, ny=50, cfl=0.4, bcs="outflow", endTime=0.004)),
        ("ot", dict(nx=200, ny=36, cfl=0.5, bcs="periodic")),
    ]
    out = []
    for kind, kw in srmhd:
        cfg = dict(model="srmhd", integrator="rk2", Ng=Ng, gamma=4.0 / 3.0, weno=weno,
                   precision=precision, endTime=kw.pop("endTime", 1.0), **kw)
        out.append((kind, cfg))
    if precision == "mixed":
        for nx, ny, sigma, bcs in ((48, 96, 1e3, "outflow"), (100, 40, 1e5, "periodic")):
            out.append(("cs", dict(model="srrmhd", integrator="ssp2", nx=nx, ny=ny, xmin=-0.5,
                                   xmax=0.5, ymin=-1.0, ymax=1.0, endTime=3.0, cfl=0.4, Ng=Ng,
                                   gamma=4.0 / 3.0, sigma=sigma, weno=weno, bcs=bcs,
                                   precision=precision)))
    return out


def _run_single(kind, cfg, n):
    import method_b200 as mb
    s = mb.Simulation(**cfg)
    s.set_prims(_prims(kind, cfg["nx"], cfg["ny"], cfg["model"], cfg["Ng"]))
    s.update_time(n)
    st = s.stats()
    out = s.state(), st
    s.close()
    return out


def _check_ensemble(precision, weno, autotune):
    import method_b200 as mb
    members = _members(precision, weno)
    ens = mb.Ensemble([cfg for _, cfg in members])
    for m, (kind, cfg) in enumerate(members):
        ens.set_prims(m, _prims(kind, cfg["nx"], cfg["ny"], cfg["model"], cfg["Ng"]))
    if autotune:
        ti = ens.autotune(reps=2)
        assert all(t in (4, 8, 16) for t in ti), ti
    ens.step(NSTEPS)
    for m, (kind, cfg) in enumerate(members):
        got = ens.state(m)
        want, st = _run_single(kind, cfg, NSTEPS)
        est = ens.stats(m)
        assert est["iters"] == NSTEPS == st["iters"], (m, est)
        assert est["t"] == st["t"], (m, est["t"], st["t"])
        assert est["c2p_unconverged"] == st["c2p_unconverged"] == 0, (m, est)
        for name, a, b in zip(("cons", "prims", "aux"), got, want):
            assert a.shape == b.shape, (m, name)
            diff = np.argwhere(a != b)
            assert diff.size == 0, (m, cfg, name, diff[:5])
    info = ens.info()
    assert info["interior_cells"] == sum(c["nx"] * c["ny"] for _, c in members)
    ens.close()


@pytest.mark.parametrize("weno", [3, 5])
def test_plain_ensemble_matches_single_runs(weno):
    _check_ensemble("fp64", weno, autotune=False)


def test_plain_ensemble_autotuned():
    _check_ensemble("fp64", 3, autotune=True)


@pytest.mark.parametrize("weno", [3, 5])
def test_mixed_ensemble_matches_single_runs(weno):
    _check_ensemble("mixed", weno, autotune=True)


def test_plain_member_matches_reference(ref):
    """One plain member against the reference CPU build directly."""
    import method_b200 as mb
    members = _members("fp64", 3)
    ens = mb.Ensemble([c for _, c in members])
    for m, (kind, cfg) in enumerate(members):
        ens.set_prims(m, _prims(kind, cfg["nx"], cfg["ny"], "srmhd", cfg["Ng"]))
    kind, cfg = members[2]  # clipped endTime, outflow, nx in the middle class
    p0 = _prims(kind, cfg["nx"], cfg["ny"], "srmhd", cfg["Ng"])
    ens.step(NSTEPS)
    got = ens.state(2)
    r = ref.RefSim(prims=p0, model="srmhd", nx=cfg["nx"], ny=cfg["ny"], nz=0, xmin=0.0,
                   xmax=1.0, ymin=0.0, ymax=1.0, endTime=cfg["endTime"], cfl=cfg["cfl"],
                   Ng=cfg["Ng"], gamma=cfg["gamma"], weno=3, bcs=cfg["bcs"], integrator="rk2")
    assert r.update_time(NSTEPS) == 0
    want = r.state()
    sl = (slice(None), slice(4, -4), slice(4, -4))
    for name, a, b in zip(("cons", "prims"), got, want):
        assert np.array_equal(a[sl], b[sl]), name
