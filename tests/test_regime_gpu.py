"""REGIME, the resistive extension of SRMHD (REGIME.cc; Wright & Hawke 2019),
as RKSplit's model extension, against the reference CPU build running the
same configuration (`REGIME ext(&data, &fvs); RKSplit ti(..., &ext)`).

Workloads: the reference's own REGIME examples (Examples/REGIME: the 1D
current sheet and Brio-Wu shock tube, WENO3, outflow) at their sizes for a
number of steps, and two-dimensional runs (Kelvin-Helmholtz and Orszag-Tang,
WENO3 and WENO5, periodic, outflow and flow boundaries) that exercise the y
diffusion vectors.  The plain FP64 form must match bit for bit (the bar
written here is 1e-12 relative); the mixed form keeps the REGIME source in
FP64 and is compared with the plain form.
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


def run_pair(ref, steps, init=None, prims=None, init_arg0=0, init_arg1=0, **cfg):
    import method_b200 as mb
    cfg = dict(cfg, model="srmhd", integrator="rksplit", regime=True)
    r = ref.RefSim(prims=prims, init=init or "array", init_arg0=init_arg0, init_arg1=init_arg1,
                   **cfg)
    _, p0, _ = r.state()
    g = mb.Simulation(**cfg)
    g.set_prims(p0)
    r.update_time(steps)
    g.update_time(steps)
    out = g.state(), r.state()
    g.close()
    r.close()
    return out


def test_current_sheet_1d(ref):
    """Examples/REGIME/CurrentSheetSerial/main.cc: nx 128, [-3, 3], cfl 0.2,
    gamma 2, sigma 1e4, WENO3, outflow."""
    cfg = dict(nx=128, ny=0, xmin=-3.0, xmax=3.0, ymin=-1.0, ymax=1.0, endTime=7.0, cfl=0.2,
               Ng=4, gamma=2.0, sigma=1e4, weno=3, bcs="outflow")
    g, r = run_pair(ref, 40, init="currentsheet", **cfg)
    assert_state_equal(g, r, "REGIME 1D current sheet")


@pytest.mark.parametrize("sigma", [100.0, 1e4])
def test_brio_wu_1d(ref, sigma):
    """Examples/REGIME/BrioWuSerial shape: Brio-Wu shock tube, WENO3, outflow."""
    cfg = dict(nx=100, ny=0, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=0.4, cfl=0.4,
               Ng=4, gamma=2.0, sigma=sigma, weno=3, bcs="outflow")
    g, r = run_pair(ref, 30, init="briowu", **cfg)
    assert_state_equal(g, r, f"REGIME 1D Brio-Wu sigma {sigma}")


@pytest.mark.parametrize("bcs", ["periodic", "outflow", "flow"])
def test_kh_2d(ref, bcs):
    """KHRandomInstabilitySingleFluid(mag=1, seed=10) on its unit square."""
    cfg = dict(nx=32, ny=64, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=3.0, cfl=0.4,
               Ng=4, gamma=4.0 / 3.0, sigma=300.0, weno=3, bcs=bcs)
    g, r = run_pair(ref, 6, init="khrandom", init_arg0=1, init_arg1=10, **cfg)
    assert_state_equal(g, r, f"REGIME KH {bcs}")


def test_ot_2d_weno5(ref):
    """WENO5 (halo 3): the stiff face fluxes are zero on the reference's
    outermost reconstructed ring, which K then reads."""
    cfg = dict(nx=40, ny=40, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1.0, cfl=0.4,
               Ng=4, gamma=2.0, sigma=1e3, weno=5, bcs="periodic")
    g, r = run_pair(ref, 5, init="ot", **cfg)
    assert_state_equal(g, r, "REGIME OT WENO5")


def test_functional_sigma_2d(ref):
    """sigma * D^gam per cell in the diffusion prefactor and dwdsb, on
    KHInstabilitySingleFluid(mag=1)."""
    cfg = dict(nx=32, ny=32, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0, endTime=3.0, cfl=0.4,
               Ng=4, gamma=4.0 / 3.0, sigma=500.0, weno=3, bcs="flow", functionalSigma=True,
               gam=2.0)
    g, r = run_pair(ref, 4, init="kh", init_arg0=1, **cfg)
    assert_state_equal(g, r, "REGIME functional sigma")


def test_regime_changes_the_step():
    """The extension is on the path: the same run without it differs, and the
    mixed form (FP32 flux, FP64 REGIME source) stays within 1e-6 of the plain
    form.  Orszag-Tang: the field is non-zero, so E = -v x B and the
    extension's source are too."""
    import method_b200 as mb
    cfg = dict(model="srmhd", nx=64, ny=64, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
               endTime=1.0, cfl=0.4, Ng=4, gamma=2.0, sigma=100.0, weno=3, bcs="periodic",
               integrator="rksplit")
    p0 = initial.orszag_tang(64, Ng=4)
    out = {}
    for name, kw in (("ideal", dict()), ("regime", dict(regime=True)),
                     ("regime_mixed", dict(regime=True, precision="mixed"))):
        s = mb.Simulation(**cfg, **kw)
        s.set_prims(p0)
        s.update_time(20)
        out[name] = s.state()[0][:, 4:-4, 4:-4]
        s.close()
    d = np.abs(out["regime"] - out["ideal"]).sum() / np.abs(out["ideal"]).sum()
    assert d > 1e-10, d
    l1 = np.abs(out["regime_mixed"] - out["regime"]).sum() / np.abs(out["regime"]).sum()
    assert l1 < 1e-6, l1
