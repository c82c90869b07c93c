"""Failure paths: solver non-convergence reported as the reference reports it.

Failures are made on the host, as ordinary inputs: conserved states with
v^2 >= 1 (momentum beyond the energy), tau < 0, or a NaN, and guesses a solver
cannot leave.  Every device loop is capped (Powell hybrid maxfev, secant 50,
Newton 60), so these inputs end in a status, never a trap or a hang.

The reference's behaviour is the spec:
  * SRRMHD::getPrimitiveVars throws std::runtime_error when the secant fails
    (srrmhd.cc:576-579) -> MTH_ERR_C2P, RuntimeError, std::runtime_error;
  * SRMHD::getPrimitiveVars only prints when the neighbour-average retry fails
    (srmhd.cc:495-498) -> MTH_OK, with the count in mth_stats.c2p_unconverged;
  * SRMHD::getPrimitiveVarsSingleCell throws (srmhd.cc:345) -> MTH_ERR_C2P;
  * SSP2::step throws when a stage's hybrd1 fails (SSP2.cc:89-98, 134-143)
    -> MTH_ERR_IMPLICIT.
Each device status is compared with the reference build's return code on the
same input (oracle/_ref, which catches the exception and returns 1).  The
error words are sticky until read: the next mth_sync after a failure reports
MTH_OK while the failure counts stay in the statistics.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SHEET = dict(model="srrmhd", nx=16, ny=32, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
             endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3, weno=3, bcs="outflow",
             integrator="ssp2")


def _inject(cons, kind, cell):
    """One unphysical conserved state at `cell` (i, j) of a ghost-inclusive array."""
    i, j = cell
    c = cons.copy()
    if kind == "nan":
        c[0, i, j, 0] = np.nan
    elif kind == "tau_negative":
        c[4, i, j, 0] = -5.0 * abs(c[0, i, j, 0])
    elif kind == "v2_ge_1":  # |S| far beyond tau + D: no physical velocity
        c[1, i, j, 0] = 50.0 * (abs(c[4, i, j, 0]) + abs(c[0, i, j, 0]))
    else:
        raise ValueError(kind)
    return c


def _sheet_state(ref):
    prims = initial.current_sheet(SHEET["nx"], SHEET["ny"], Ng=4, seed=5)
    r = ref.RefSim(prims=prims, init="array", **SHEET)
    return r, r.state()


@pytest.mark.parametrize("kind", ["nan", "tau_negative", "v2_ge_1"])
def test_srrmhd_grid_c2p_failure_matches_reference(ref, kind):
    import method_b200 as mb
    from method_b200 import _lib

    r, (cons, prims, aux) = _sheet_state(ref)
    bad = _inject(cons, kind, (9, 20))
    rc_ref = r.c2p(bad.copy(), prims.copy(), aux.copy())
    assert rc_ref == 1, "the reference's secant fails on this state"

    g = mb.Simulation(**SHEET)
    g.set_prims(prims)
    g.upload(bad, prims, aux)
    L = _lib.load()
    assert L.mth_c2p(g.h) == 1  # MTH_ERR_C2P
    assert "C2P could not converge" in L.mth_last_error(g.h).decode()
    assert g.stats()["c2p_unconverged"] >= 1
    assert L.mth_sync(g.h) == 0  # the error word cleared when it was read
    # the Python mirror raises the reference's exception type
    g.upload(bad, prims, aux)
    with pytest.raises(RuntimeError, match="C2P could not converge"):
        g.c2p()
    # a clean state recovers again on the same handle
    g.upload(cons, prims, aux)
    g.c2p()
    assert r.c2p(cons.copy(), prims.copy(), aux.copy()) == 0
    g.close()


@pytest.mark.parametrize("kind", ["nan", "tau_negative", "v2_ge_1"])
def test_srmhd_grid_c2p_failure_only_counts(ref, kind):
    """SRMHD's grid recovery prints and continues when the retry fails: the
    device returns MTH_OK and counts the cells, as many as the oracle counts."""
    import method_b200 as mb
    from oracle import port

    n = 32
    cfg = dict(model="srmhd", nx=n, ny=n, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1.0,
               cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="periodic", integrator="rk2")
    p0 = initial.orszag_tang(n, Ng=4)
    r = ref.RefSim(prims=p0, init="array", **cfg)
    cons, prims, aux = r.state()
    bad = _inject(cons, kind, (12, 7))
    rp, ra = prims.copy(), aux.copy()
    assert r.c2p(bad.copy(), rp, ra) == 0

    o = port.PortSim(p0, **cfg)
    o.c2p(bad.copy(), prims.copy(), aux.copy())
    _, still = o.solution()

    g = mb.Simulation(**cfg)
    g.set_prims(p0)
    g.reset_stats()
    g.upload(bad, prims, aux)
    g.c2p()  # no exception
    s = g.stats()
    assert s["status"] == 0
    assert s["c2p_unconverged"] == still
    # every interior value equals the reference's, the failed cell included
    _, gp, ga = g.state()
    core = (slice(None), slice(4, -4), slice(4, -4))
    np.testing.assert_array_equal(gp[core], rp[core])
    np.testing.assert_array_equal(ga[core], ra[core])
    g.close()


@pytest.mark.parametrize("kind", ["nan", "tau_negative", "v2_ge_1"])
def test_srmhd_single_cell_failure_matches_reference(ref, kind):
    from method_b200 import _lib

    L = _lib.load()
    n = 32
    cfg = dict(model="srmhd", nx=n, ny=n, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1.0,
               cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="periodic", integrator="rk2")
    r = ref.RefSim(prims=initial.orszag_tang(n, Ng=4), init="array", **cfg)
    cons, prims, aux = r.state()
    bad = _inject(cons, kind, (12, 7))
    c1 = np.ascontiguousarray(bad[:, 12, 7, 0])
    p1 = np.ascontiguousarray(prims[:, 12, 7, 0])
    a1 = np.ascontiguousarray(aux[:, 12, 7, 0])
    rc_ref = r.c2p_single(c1.copy(), p1.copy(), a1.copy())
    D = C.POINTER(C.c_double)
    pc, ac = p1.copy(), a1.copy()
    rc = L.mth_c2p_cells(0, 4.0 / 3.0, 0.0, 1, c1.ctypes.data_as(D), pc.ctypes.data_as(D),
                         ac.ctypes.data_as(D), 1.4e-8, 0)
    assert rc == (1 if rc_ref else 0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ssp2_step_failure_matches_reference(ref, precision):
    import method_b200 as mb
    from method_b200 import _lib

    r, (cons, prims, aux) = _sheet_state(ref)
    bad = _inject(cons, "nan", (10, 12))
    dt = 1e-4
    r.set_state(bad, prims, aux)
    assert r.step_dt(dt) == 1  # the reference throws out of SSP2::step

    g = mb.Simulation(precision=precision, **SHEET)
    g.set_prims(prims)
    g.upload(bad, prims, aux)
    L = _lib.load()
    assert L.mth_step(g.h, dt) == 0  # enqueued
    assert L.mth_sync(g.h) == 2  # MTH_ERR_IMPLICIT
    assert g.stats()["implicit_failed"] >= 1
    assert L.mth_sync(g.h) == 0
    g.upload(bad, prims, aux)
    with pytest.raises(RuntimeError, match="could not converge"):
        g.step(dt)
    # the same step from the clean state succeeds on both
    g.upload(cons, prims, aux)
    g.step(dt)
    r.set_state(cons, prims, aux)
    assert r.step_dt(dt) == 0
    g.close()


def test_ensemble_failure_is_reported_and_cleared():
    """A member whose state holds a NaN makes the ensemble's sync return
    MTH_ERR_C2P or MTH_ERR_IMPLICIT (as the single simulation would); the next
    sync after the failure was read returns MTH_OK."""
    import method_b200 as mb
    from method_b200 import _lib

    members = []
    for m, model in enumerate(("srmhd", "srrmhd")):
        members.append(dict(model=model, nx=32, ny=64, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
                            endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3, weno=3,
                            bcs="flow", integrator="rk2" if model == "srmhd" else "ssp2",
                            precision="mixed"))
    e = mb.Ensemble(members)
    for m, cfg in enumerate(members):
        p = initial.kelvin_helmholtz(cfg["nx"], cfg["ny"], Ng=4, seed=3 + m, model=cfg["model"])
        if m == 1:
            p[0, 10, 20, 0] = np.nan
        e.set_prims(m, p)
    L = _lib.load()
    assert L.mth_ensemble_step(e.e, 1) == 0
    assert L.mth_ensemble_sync(e.e) in (1, 2)
    assert L.mth_ensemble_sync(e.e) == 0
    e.close()


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_cpp_dropin_throws_reference_exceptions(tmp_path):
    exe = tmp_path / "fail_main"
    r = subprocess.run(["g++", "-std=c++11", "-O2", "-I",
                        os.path.join(ROOT, "include", "method_b200"),
                        os.path.join(ROOT, "tests", "cpp", "fail_main.cc"), "-o", str(exe),
                        "-L", os.path.join(ROOT, "method_b200"), "-lmethod_b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "method_b200")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = dict(line.split() for line in r.stdout.splitlines() if line.count(" ") == 1)
    assert got == {"srrmhd_c2p_nan": "runtime_error", "srrmhd_c2p_clean": "ok",
                   "ssp2_step_nan": "runtime_error", "srmhd_single_cell_bad": "runtime_error",
                   "negative_sigma": "invalid_argument"}, r.stdout
