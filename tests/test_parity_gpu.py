"""GPU parity against the reference CPU build (oracle/_ref).

The plain FP64 form is expected to reproduce the reference bit for bit; the
acceptance bar written here is the one the workload states, 1e-12 relative
in every conserved, primitive and auxiliary variable (aux where the reference
defines it for interior and ghost cells alike).  Workloads restate the
reference's own consistency tests (Tests/CPU/Src/test_rk2.cc, test_rkSplit.cc,
test_imex.cc, test_fvs.cc) plus the measured configurations at reduced size.
"""
import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel_err(a, b):
    scale = np.maximum(np.abs(b), 1e-300)
    d = np.abs(a - b)
    # absolute floor for values that are zero in the reference
    return float(np.max(np.where(np.abs(b) > 1e-12, d / scale, d)))


def assert_state_equal(gpu_state, ref_state, what, tol=RTOL):
    for name, g, r in zip(("cons", "prims", "aux"), gpu_state, ref_state):
        assert g.shape == r.shape, (what, name)
        assert np.all(np.isfinite(g)) == np.all(np.isfinite(r)), (what, name)
        e = rel_err(g, r)
        assert e <= tol, f"{what}: {name} differs from the reference, max rel err {e:.3e}"


def make_pair(ref, prims=None, init=None, **cfg):
    import method_b200 as mb
    rkw = dict(cfg)
    rkw["weno"] = cfg.get("weno", 3)
    r = ref.RefSim(prims=prims, init=init or "array", **rkw)
    if prims is None:
        _, prims, _ = r.state()
    g = mb.Simulation(**cfg)
    g.set_prims(prims)
    return g, r


OT40 = dict(model="srmhd", nx=40, ny=40, xmin=0, xmax=1, ymin=0, ymax=1, endTime=0.004,
            cfl=0.6, Ng=4, gamma=2.0, weno=3, integrator="rk2")


@pytest.mark.parametrize("bcs", ["periodic", "outflow", "flow"])
def test_set_matches_reference(ref, bcs):
    g, r = make_pair(ref, init="ot", bcs=bcs, **OT40)
    assert_state_equal(g.state(), r.state(), f"Simulation::set ({bcs})", tol=0.0)


@pytest.mark.parametrize("bcs", ["periodic", "outflow", "flow"])
def test_rk2_one_step_ot40(ref, bcs):
    """test_rk2.cc RK2SrmhdPeriodicOTVSF / Outflow / Flow: OT 40x40, one step."""
    g, r = make_pair(ref, init="ot", bcs=bcs, **OT40)
    r.update_time(1)
    g.update_time(1)
    assert_state_equal(g.state(), r.state(), f"RK2 OT40 {bcs}")


def test_flux_F_matches_reference(ref):
    g, r = make_pair(ref, init="ot", bcs="periodic", **OT40)
    c, p, a = r.state()
    fr = r.flux_F(c, p, a)
    fg = g.flux_F()
    sl = (slice(None), slice(4, -4), slice(4, -4))
    assert rel_err(fg[sl], fr[sl]) == 0.0


@pytest.mark.parametrize("weno,steps", [(3, 40), (5, 20)])
def test_kh_steps(ref, weno, steps):
    """Kelvin-Helmholtz 64x128 (the measured SRMHD shear-layer workload)."""
    prims = initial.kelvin_helmholtz(64, 128, Ng=4, seed=7)
    cfg = dict(model="srmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=weno, bcs="flow",
               integrator="rk2")
    g, r = make_pair(ref, prims=prims, **cfg)
    r.update_time(steps)
    g.update_time(steps)
    assert_state_equal(g.state(), r.state(), f"KH weno{weno} {steps} steps")


def test_ot_weno5_periodic(ref):
    prims = initial.orszag_tang(96, Ng=4)
    cfg = dict(model="srmhd", nx=96, ny=96, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
               endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=5, bcs="periodic",
               integrator="rk2")
    g, r = make_pair(ref, prims=prims, **cfg)
    r.update_time(10)
    g.update_time(10)
    assert_state_equal(g.state(), r.state(), "OT96 weno5")


@pytest.mark.parametrize("bcs", ["periodic", "outflow", "flow"])
def test_rksplit_kh_random(ref, bcs):
    """test_rkSplit.cc: KHRandomInstabilitySingleFluid(mag=1, seed=10), RKSplit."""
    cfg = dict(model="srmhd", nx=40, ny=40, xmin=0, xmax=1, ymin=0, ymax=1, endTime=0.004,
               cfl=0.6, Ng=4, gamma=4.0 / 3.0, sigma=10.0, cp=1.0, weno=3, bcs=bcs,
               integrator="rksplit")
    import method_b200 as mb
    r = ref.RefSim(init="khrandom", init_arg0=1, init_arg1=10, **cfg)
    _, prims, _ = r.state()
    g = mb.Simulation(**cfg)
    g.set_prims(prims)
    r.update_time(1)
    g.update_time(1)
    assert_state_equal(g.state(), r.state(), f"RKSplit {bcs}")


def test_srrmhd_rk2(ref):
    prims = initial.kelvin_helmholtz(32, 64, Ng=4, seed=3, model="srrmhd")
    cfg = dict(model="srrmhd", nx=32, ny=64, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=10.0, weno=3, bcs="flow",
               integrator="rk2")
    g, r = make_pair(ref, prims=prims, **cfg)
    assert_state_equal(g.state(), r.state(), "SRRMHD set", tol=0.0)
    r.update_time(5)
    g.update_time(5)
    assert_state_equal(g.state(), r.state(), "SRRMHD RK2")


def test_srrmhd_ssp2(ref):
    """test_imex.cc SSP2FlowKHSingleFluid shape: SRRMHD KH 64x16, SSP2."""
    cfg = dict(model="srrmhd", nx=64, ny=16, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=0.05, cfl=0.5, Ng=4, gamma=4.0 / 3.0, sigma=10.0, weno=3, bcs="flow",
               integrator="ssp2")
    import method_b200 as mb
    r = ref.RefSim(init="kh", init_arg0=0, **cfg)
    _, prims, _ = r.state()
    g = mb.Simulation(**cfg)
    g.set_prims(prims)
    assert_state_equal(g.state(), r.state(), "SSP2 set", tol=0.0)
    r.update_time(3)
    g.update_time(3)
    assert_state_equal(g.state(), r.state(), "SSP2 3 steps")


@pytest.mark.parametrize("integrator", ["ssp3", "ssp2322"])
def test_srrmhd_imex3_brio_wu(ref, integrator):
    """test_imex.cc IMEX3BenchmarkForParallelCode shape: SRRMHD Brio-Wu 64x16,
    sigma 0, outflow, SSP3(332) (and SSP2(322) on the same case)."""
    cfg = dict(model="srrmhd", nx=64, ny=16, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
               endTime=0.05, cfl=0.5, Ng=4, gamma=4.0 / 3.0, sigma=0.0, weno=3, bcs="outflow",
               integrator=integrator)
    import method_b200 as mb
    r = ref.RefSim(init="briowu", init_arg0=0, **cfg)
    _, prims, _ = r.state()
    g = mb.Simulation(**cfg)
    g.set_prims(prims)
    r.update_time(3)
    g.update_time(3)
    assert_state_equal(g.state(), r.state(), f"{integrator} Brio-Wu 3 steps")


@pytest.mark.parametrize("integrator,bcs,sigma",
                         [("ssp3", "outflow", 1e3), ("ssp3", "flow", 1e5),
                          ("ssp2322", "periodic", 1e3), ("ssp2322", "outflow", 1e5)])
def test_srrmhd_imex3_current_sheet(ref, integrator, bcs, sigma):
    """Resistive current sheet 32x64 with stiff conductivity, SSP3 / SSP2322."""
    cfg = dict(model="srrmhd", nx=32, ny=64, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=sigma, weno=3, bcs=bcs,
               integrator=integrator)
    p = initial.current_sheet(32, 64, seed=17)
    g, r = make_pair(ref, prims=p, **cfg)
    r.update_time(3)
    g.update_time(3)
    st = g.stats()
    assert st["implicit_failed"] == 0
    assert_state_equal(g.state(), r.state(), f"{integrator} current sheet")


def test_3d_generic_path(ref):
    """3D (generic per-direction flux path), OT-like data, periodic."""
    n = 12
    x = (np.arange(n + 8) + 0.5 - 4) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    p = np.zeros((8, n + 8, n + 8, n + 8))
    p[0] = 1.0
    p[4] = 1.0
    p[1] = -0.3 * np.sin(2 * np.pi * Y)
    p[2] = 0.3 * np.sin(2 * np.pi * X)
    p[3] = 0.1 * np.sin(2 * np.pi * Z)
    p[5] = -0.5 * np.sin(2 * np.pi * Y)
    p[6] = 0.5 * np.sin(4 * np.pi * X)
    p[7] = 0.2 * np.cos(2 * np.pi * Z)
    cfg = dict(model="srmhd", nx=n, ny=n, nz=n, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0,
               zmax=1, endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="periodic",
               integrator="rk2")
    g, r = make_pair(ref, prims=p, **cfg)
    r.update_time(2)
    g.update_time(2)
    assert_state_equal(g.state(), r.state(), "3D RK2")


def test_1d_brio_wu(ref):
    cfg = dict(model="srmhd", nx=64, ny=0, xmin=0, xmax=1, ymin=0, ymax=1, endTime=0.4,
               cfl=0.4, Ng=4, gamma=2.0, weno=3, bcs="outflow", integrator="rk2")
    import method_b200 as mb
    r = ref.RefSim(init="briowu", init_arg0=0, **cfg)
    _, prims, _ = r.state()
    g = mb.Simulation(**cfg)
    g.set_prims(prims)
    r.update_time(5)
    g.update_time(5)
    assert_state_equal(g.state(), r.state(), "1D Brio-Wu")


@pytest.mark.parametrize("sigma", [10.0, 1e3, 1e5])
def test_srrmhd_ssp2_mixed_vs_fp64(sigma):
    """Mixed form of SSP2 (FP32 flux, closed-form psi/phi + Newton on E, Newton
    C2P) against the plain FP64 form (bit-identical to the reference) on the
    resistive current sheet: L1 relative < 1e-6 after 10 steps, every cell
    converged."""
    import method_b200 as mb
    cfg = dict(model="srrmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=sigma, weno=3, bcs="outflow",
               integrator="ssp2")
    p = initial.current_sheet(64, 128, Ng=4, seed=21)
    a = mb.Simulation(**cfg)
    a.set_prims(p)
    a.update_time(10)
    b = mb.Simulation(precision="mixed", **cfg)
    b.set_prims(p)
    b.update_time(10)
    st = b.stats()
    assert st["status"] == 0 and st["implicit_failed"] == 0
    ca, pa, _ = a.state()
    cb, pb, _ = b.state()
    sl = (slice(None), slice(4, -4), slice(4, -4))
    for name, x, y in (("cons", cb, ca), ("prims", pb, pa)):
        l1 = np.abs(x[sl] - y[sl]).sum() / np.abs(y[sl]).sum()
        assert l1 < 1e-6, (name, l1, st)


@pytest.mark.parametrize("integrator", ["ssp3", "ssp2322"])
@pytest.mark.parametrize("sigma", [1e3, 1e5])
def test_srrmhd_imex3_mixed_vs_fp64(integrator, sigma):
    """Mixed form of SSP3 / SSP2322 (FP32 flux, closed-form psi/phi + Newton on
    E, Newton C2P, exact solve for unconverged cells) against the plain FP64
    form on the current sheet: L1 relative < 1e-6 after 10 steps."""
    import method_b200 as mb
    cfg = dict(model="srrmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=sigma, weno=3, bcs="outflow",
               integrator=integrator)
    p = initial.current_sheet(64, 128, Ng=4, seed=23)
    a = mb.Simulation(**cfg)
    a.set_prims(p)
    a.update_time(10)
    b = mb.Simulation(precision="mixed", **cfg)
    b.set_prims(p)
    b.update_time(10)
    st = b.stats()
    assert st["status"] == 0 and st["implicit_failed"] == 0 and st["c2p_unconverged"] == 0
    ca, pa, _ = a.state()
    cb, pb, _ = b.state()
    sl = (slice(None), slice(4, -4), slice(4, -4))
    for name, x, y in (("cons", cb, ca), ("prims", pb, pa)):
        l1 = np.abs(x[sl] - y[sl]).sum() / np.abs(y[sl]).sum()
        assert l1 < 1e-6, (name, l1, st)


@pytest.mark.parametrize("integrator,sigma,gam", [("ssp2", 1e3, 12.0), ("rk2", 10.0, 3.0),
                                                  ("ssp3", 1e2, 2.0)])
def test_srrmhd_functional_sigma(ref, integrator, sigma, gam):
    """Data::functionalSigma: the conductivity of each cell is sigma * D^gam
    (simData.cc:114-127), in the recovery, primsToAll and the implicit stages.
    The device's pow and the host C library's differ in the last place for
    about 0.1% of arguments (the C library's pow is not correctly rounded:
    it misrounds even x^2 that often), so equality is not the bar.  RK2 keeps
    such differences at rounding level: 1e-12 relative.  The IMEX stages
    solve with the Powell hybrid, whose finite-difference Jacobian turns a
    last-place difference in the residual into a different stopping point
    within its tolerance (xtol 1.49e-7 relative to the cell's state norm), so
    there the bar is each cell's state within 1e-6 of the reference's,
    relative to the cell's norm."""
    import method_b200 as mb
    cfg = dict(model="srrmhd", nx=24, ny=48, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=sigma, weno=3,
               bcs="outflow", integrator=integrator, functionalSigma=True, gam=gam)
    p = initial.current_sheet(24, 48, seed=12)
    p[0] *= 1.0 + 0.3 * np.sin(np.linspace(0, 3.0, p.shape[2]))[None, :, None]
    g, r = make_pair(ref, prims=p, **cfg)
    assert_state_equal(g.state(), r.state(), "functional sigma set")
    r.update_time(3)
    g.update_time(3)
    if integrator == "rk2":
        assert_state_equal(g.state(), r.state(), f"functional sigma {integrator}")
    else:
        for name, a, b in zip(("cons", "prims"), g.state()[:2], r.state()[:2]):
            d = np.linalg.norm(a - b, axis=0) / np.linalg.norm(b, axis=0)
            assert np.max(d) <= 1e-6, (name, float(np.max(d)))
    if integrator == "ssp2":  # the mixed form against the plain one
        m = mb.Simulation(precision="mixed", **cfg)
        m.set_prims(p)
        m.update_time(3)
        for a, b in zip(m.state()[:2], g.state()[:2]):
            core = (slice(None), slice(4, -4), slice(4, -4))
            l1 = np.abs(a[core] - b[core]).sum() / np.abs(b[core]).sum()
            assert l1 < 1e-6, l1


@pytest.mark.parametrize("weno", [7, 9, 11])
def test_high_order_weno_matches_reference(ref, weno):
    """Weno7 / Weno9 / Weno11 (weno.cc:239-482) in the fused 2D tile: KH on
    Flow boundaries, RK2, against the reference build, and the mixed form
    against the plain one."""
    import method_b200 as mb
    Ng = (weno + 1) // 2 + 1
    cfg = dict(model="srmhd", nx=40, ny=80, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=Ng, gamma=4.0 / 3.0, weno=weno, bcs="flow",
               integrator="rk2")
    p = initial.kelvin_helmholtz(40, 80, Ng=Ng, seed=weno)
    g, r = make_pair(ref, prims=p, **cfg)
    r.update_time(6)
    g.update_time(6)
    assert_state_equal(g.state(), r.state(), f"WENO{weno} KH RK2")
    m = mb.Simulation(precision="mixed", **cfg)
    m.set_prims(p)
    m.update_time(6)
    core = (slice(None), slice(Ng, -Ng), slice(Ng, -Ng))
    for a, b in zip(m.state()[:2], g.state()[:2]):
        l1 = np.abs(a[core] - b[core]).sum() / np.abs(b[core]).sum()
        assert l1 < 1e-6, (weno, l1)


@pytest.mark.parametrize("weno,dims", [(7, 3), (9, 1)])
def test_high_order_weno_generic_path(ref, weno, dims):
    """The 1D / 3D (unfused) flux path with WENO7 / WENO9."""
    Ng = (weno + 1) // 2 + 1
    if dims == 3:
        n = 12
        cfg = dict(model="srmhd", nx=n, ny=n, nz=n, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0,
                   zmax=1, endTime=1.0, cfl=0.4, Ng=Ng, gamma=4.0 / 3.0, weno=weno,
                   bcs="periodic", integrator="rk2")
        p = np.zeros((8, n + 2 * Ng, n + 2 * Ng, n + 2 * Ng))
        x = np.linspace(0, 1, n + 2 * Ng)
        p[0] = 1.0 + 0.1 * np.sin(2 * np.pi * x)[:, None, None]
        p[1] = 0.2 * np.sin(2 * np.pi * x)[None, :, None]
        p[2] = 0.1 * np.cos(2 * np.pi * x)[None, None, :]
        p[4] = 1.0
        p[5] = 0.3
    else:
        n = 64
        cfg = dict(model="srmhd", nx=n, ny=0, xmin=0, xmax=1, endTime=1.0, cfl=0.4, Ng=Ng,
                   gamma=2.0, weno=weno, bcs="outflow", integrator="rk2")
        p = np.zeros((8, n + 2 * Ng, 1, 1))
        left = np.arange(n + 2 * Ng) < (n + 2 * Ng) // 2
        p[0, :, 0, 0] = np.where(left, 1.0, 0.125)
        p[4, :, 0, 0] = np.where(left, 1.0, 0.1)
        p[5] = 0.5
        p[6, :, 0, 0] = np.where(left, 1.0, -1.0)
    g, r = make_pair(ref, prims=p, **cfg)
    r.update_time(3)
    g.update_time(3)
    assert_state_equal(g.state(), r.state(), f"WENO{weno} {dims}D")
