"""The Hybrid model (hybrid.cc: SRRMHD's variables, ideal and resistive
fluxes, sources and recoveries blended by a conductivity weight, optionally
with the REGIME term on the ideal part) and the second-order split integrator
RKSplit2 (rkSplit2ndOrder.cc), against the reference CPU build running the
same configuration (`Hybrid model(&data, sigmaCrossOver, sigmaSpan,
useREGIME); model.setupREGIME(&fvs); RKSplit2 ti(...)`).

Both sides start from the same raw primitives (Simulation::set then runs the
Hybrid primsToAll blend on each side).  The bar for the plain form is 1e-12
relative.
"""
import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel_err(a, b):
    scale = np.maximum(np.abs(b), 1e-300)
    d = np.abs(a - b)
    return float(np.max(np.where(np.abs(b) > 1e-12, d / scale, d)))


def assert_state_equal(gpu_state, ref_state, what, tol=RTOL):
    for name, g, r in zip(("cons", "prims", "aux"), gpu_state, ref_state):
        assert g.shape == r.shape, (what, name)
        assert np.all(np.isfinite(g)), (what, name)
        e = rel_err(g, r)
        assert e <= tol, f"{what}: {name} differs from the reference, max rel err {e:.3e}"


def raw_prims(ref, init, **cfg):
    """The initial data of a reference InitialFunc on SRRMHD's variables
    (SRRMHD's primsToAll leaves prims as set)."""
    r = ref.RefSim(init=init, **dict(cfg, model="srrmhd", integrator="rk2"))
    p = r.state()[1]
    r.close()
    return p


def run_pair(ref, steps, prims, **cfg):
    import method_b200 as mb
    r = ref.RefSim(prims=prims, init="array", **cfg)
    g = mb.Simulation(**cfg)
    g.set_prims(prims)
    set_state = g.state(), r.state()
    r.update_time(steps)
    g.update_time(steps)
    out = g.state(), r.state()
    g.close()
    r.close()
    return set_state, out


BRIOWU = dict(model="hybrid", integrator="rksplit2", nx=400, ny=0, xmin=-3.0, xmax=3.0,
              ymin=-1.0, ymax=1.0, zmin=-1.0, zmax=1.0, endTime=0.4, cfl=0.2, Ng=4, gamma=2.0,
              sigma=1e56, cp=1.0, weno=3, bcs="outflow", functionalSigma=True, gam=112.0,
              sigmaCrossOver=150.0, sigmaSpan=50.0)


@pytest.mark.parametrize("use_regime", [True, False])
def test_briowu_functional_conductivity(ref, use_regime):
    """Examples/Hybrid/BrioWuFunctionalConductivity: sigma = 1e56 D^112 makes
    the dense side ideal and the light side resistive, with a blended layer
    between; 40 of its ~133 steps."""
    cfg = dict(BRIOWU, useREGIME=use_regime)
    p0 = raw_prims(ref, "briowu", **cfg)
    (g0, r0), (g, r) = run_pair(ref, 40, p0, **cfg)
    assert_state_equal(g0, r0, "Hybrid Brio-Wu after Simulation::set")
    assert_state_equal(g, r, f"Hybrid Brio-Wu (REGIME {use_regime})")


@pytest.mark.parametrize("integrator", ["rk2", "rksplit2"])
@pytest.mark.parametrize("use_regime", [True, False])
def test_orszag_tang_2d_blend(ref, integrator, use_regime):
    """2D, constant sigma inside the blend band (weight 0.5 + tanh ramp), the
    REGIME mask's neighbourhood over a third, unused dimension."""
    cfg = dict(model="hybrid", integrator=integrator, nx=32, ny=32, xmin=0.0, xmax=1.0,
               ymin=0.0, ymax=1.0, endTime=1.0, cfl=0.3, Ng=4, gamma=2.0, sigma=170.0, cp=1.0,
               weno=3, bcs="periodic", sigmaCrossOver=150.0, sigmaSpan=50.0,
               useREGIME=use_regime)
    p0 = np.zeros((11, 40, 40, 1))
    p0[:8] = initial.orszag_tang(32, Ng=4)
    (g0, r0), (g, r) = run_pair(ref, 8, p0, **cfg)
    assert_state_equal(g0, r0, "Hybrid OT after Simulation::set")
    assert_state_equal(g, r, f"Hybrid OT {integrator} REGIME {use_regime}")


@pytest.mark.parametrize("model", ["srmhd", "srrmhd"])
def test_rksplit2_single_models(ref, model):
    """RKSplit2 with the SRMHD and SRRMHD models (no extension)."""
    import method_b200 as mb
    cfg = dict(model=model, integrator="rksplit2", nx=40, ny=40, xmin=0.0, xmax=1.0, ymin=0.0,
               ymax=1.0, endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=10.0, cp=1.0,
               weno=3, bcs="periodic")
    n = 11 if model == "srrmhd" else 8
    p0 = initial.orszag_tang(40, Ng=4, model=model)[:n]
    r = ref.RefSim(prims=p0, init="array", **cfg)
    g = mb.Simulation(**cfg)
    g.set_prims(p0)
    r.update_time(6)
    g.update_time(6)
    assert_state_equal(g.state(), r.state(), f"RKSplit2 {model}")
    g.close()
    r.close()


def test_current_sheet_recovery_failure_matches(ref):
    """Examples/Hybrid/CurrentSheet: the reference's first step throws
    ("C2P could not converge") from the ideal recovery; the device reports the
    same failure as MTH_ERR_C2P."""
    import method_b200 as mb
    cfg = dict(BRIOWU, sigma=150.0, functionalSigma=False, endTime=7.0)
    p0 = raw_prims(ref, "currentsheet", **cfg)
    r = ref.RefSim(prims=p0, init="array", **cfg)
    ref_rc = r.update_time(1)
    r.close()
    g = mb.Simulation(**cfg)
    g.set_prims(p0)
    if ref_rc != 0:
        with pytest.raises(RuntimeError):
            g.update_time(1)
    else:
        g.update_time(1)
    g.close()


@pytest.mark.parametrize("case", ["ot2d", "briowu1d"])
def test_mixed_form_against_plain(case):
    """The mixed form (FP32 flux tile in 2D; Newton recoveries in both
    branches) stays within 1e-6 (L1, relative) of the plain form."""
    import method_b200 as mb
    if case == "ot2d":
        cfg = dict(model="hybrid", integrator="rksplit2", nx=64, ny=64, xmin=0.0, xmax=1.0,
                   ymin=0.0, ymax=1.0, endTime=1.0, cfl=0.3, Ng=4, gamma=2.0, sigma=170.0,
                   cp=1.0, weno=5, bcs="periodic", sigmaCrossOver=150.0, sigmaSpan=50.0)
        p0 = np.zeros((11, 72, 72, 1))
        p0[:8] = initial.orszag_tang(64, Ng=4)
    else:
        cfg = dict(BRIOWU)
        p0 = np.zeros((11, 408, 1, 1))
        p0[0] = np.where(np.arange(408) < 204, 1.0, 0.125)[:, None, None]
        p0[4] = np.where(np.arange(408) < 204, 1.0, 0.1)[:, None, None]
        p0[5] = 0.75
        p0[6] = np.where(np.arange(408) < 204, 1.0, -1.0)[:, None, None]
    out = {}
    for prec in ("fp64", "mixed"):
        s = mb.Simulation(precision=prec, **cfg)
        s.set_prims(p0)
        s.update_time(20)
        out[prec] = s.state()[0][:, 4:-4]
        s.close()
    l1 = np.abs(out["mixed"] - out["fp64"]).sum() / np.abs(out["fp64"]).sum()
    assert np.all(np.isfinite(out["mixed"]))
    assert l1 < 1e-6, l1
