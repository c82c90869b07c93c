"""Checks at the measured workloads' full sizes.

Exact comparison with the reference where the reference finishes in seconds
(one RK2 step of Orszag-Tang 1024^2; the whole Kelvin-Helmholtz 64x128 run to
t = 3), and size-independent properties elsewhere: conservation under
periodic boundaries (the flux form telescopes, so interior sums change by
rounding only), the mixed form's L1 distance from the bit-exact FP64 form,
convergence of every primitive recovery and implicit solve, recovery of the
generating states of 256^3 random cells, and ensemble members equal to
their single runs.
"""
import ctypes as C

import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu

OT = dict(model="srmhd", xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1e9, cfl=0.4, Ng=4,
          gamma=4.0 / 3.0, weno=5, bcs="periodic", integrator="rk2")
SL = (slice(None), slice(4, -4), slice(4, -4))


def test_ot1024_first_step_matches_reference(ref):
    import method_b200 as mb
    n = 1024
    p0 = initial.orszag_tang(n, Ng=4)
    g = mb.Simulation(nx=n, ny=n, **OT)
    g.set_prims(p0)
    g.update_time(1)
    r = ref.RefSim(prims=p0, nx=n, ny=n, **OT)
    assert r.update_time(1) == 0
    for name, a, b in zip(("cons", "prims", "aux"), g.state(), r.state()):
        assert np.array_equal(a, b), name


def test_ot1024_conservation_and_mixed_distance():
    import method_b200 as mb
    n, steps = 1024, 20
    p0 = initial.orszag_tang(n, Ng=4)
    out = {}
    for prec in ("fp64", "mixed"):
        s = mb.Simulation(nx=n, ny=n, precision=prec, **OT)
        s.set_prims(p0)
        c0 = s.state()[0][SL].sum(axis=(1, 2, 3))
        s.update_time(steps)
        st = s.stats()
        assert st["c2p_unconverged"] == 0 and st["status"] == 0, (prec, st)
        c, p, _ = s.state()
        c1 = c[SL].sum(axis=(1, 2, 3))
        scale = np.abs(c[SL]).sum(axis=(1, 2, 3)) + 1.0
        # D, S, tau, B, phi: interior totals move by rounding only (of FP64
        # face fluxes in the plain form, of FP32 ones in the mixed form)
        tol = 1e-12 if prec == "fp64" else 1e-8
        assert np.all(np.abs(c1 - c0) <= tol * scale), (prec, (c1 - c0) / scale)
        out[prec] = (c[SL], p[SL])
        s.close()
    for k, name in enumerate(("cons", "prims")):
        a, b = out["mixed"][k], out["fp64"][k]
        l1 = np.abs(a - b).sum() / np.abs(b).sum()
        assert l1 < 1e-6, (name, l1)


def test_kh64x128_full_run_matches_reference(ref):
    """The whole Kelvin-Helmholtz run (t = 0 .. 3, ~700 updateTime calls)."""
    import method_b200 as mb
    cfg = dict(model="srmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3, bcs="flow",
               integrator="rk2")
    p0 = initial.kelvin_helmholtz(64, 128, seed=1234)
    g = mb.Simulation(**cfg)
    g.set_prims(p0)
    g.evolve()
    r = ref.RefSim(prims=p0, **cfg)
    steps = 0
    while r.t < cfg["endTime"]:
        assert r.update_time(1) == 0
        steps += 1
    st = g.stats()
    assert st["iters"] == steps and st["t"] == r.t
    for name, a, b in zip(("cons", "prims", "aux"), g.state(), r.state()):
        assert np.array_equal(a, b), name


def test_sheet512x1024_mixed_vs_plain():
    """SSP2 on the resistive current sheet at 512x1024 (sigma 1e4)."""
    import method_b200 as mb
    cfg = dict(model="srrmhd", nx=512, ny=1024, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e4, weno=3, bcs="outflow",
               integrator="ssp2")
    p0 = initial.current_sheet(512, 1024, seed=3)
    res = {}
    for prec in ("fp64", "mixed"):
        s = mb.Simulation(precision=prec, **cfg)
        s.set_prims(p0)
        s.update_time(4)
        st = s.stats()
        assert st["status"] == 0 and st["implicit_failed"] == 0, (prec, st)
        c, p, _ = s.state()
        res[prec] = (c[SL], p[SL])
        s.close()
    for k, name in enumerate(("cons", "prims")):
        a, b = res["mixed"][k], res["fp64"][k]
        l1 = np.abs(a - b).sum() / np.abs(b).sum()
        assert l1 < 1e-6, (name, l1)


def test_c2p_256cubed_recovers_generating_states():
    import torch

    import method_b200 as mb
    from method_b200 import _lib
    L = _lib.load()
    n, gamma = 256 ** 3, 4.0 / 3.0
    F, D = C.POINTER(C.c_float), C.POINTER(C.c_double)
    feat = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    tgt = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    cons = torch.empty((9, n), dtype=torch.float64, device="cuda")
    truth = torch.empty((8, n), dtype=torch.float64, device="cuda")
    assert L.mth_mlp_make_pairs(n, 99, gamma, C.cast(feat.data_ptr(), F), C.cast(tgt.data_ptr(), F),
                                C.cast(cons.data_ptr(), D), C.cast(truth.data_ptr(), D), 0) == 0
    del feat, tgt
    P, S, _ = mb.train_guess()
    ctx = C.c_void_p()
    assert L.mth_c2p_ctx_create(n, 0, C.byref(ctx)) == 0
    try:
        assert L.mth_c2p_ctx_set_mlp(ctx, P.ctypes.data_as(F), S.ctypes.data_as(F)) == 0
        for guess in (0, 1, 2):
            prims = truth.clone()
            prims[0] *= 1.01
            prims[1:4] *= 0.99
            aux = torch.zeros((13, n), dtype=torch.float64, device="cuda")
            aux[0] = (1.0 + truth[4] / truth[0] * (gamma / (gamma - 1.0))) * 1.01
            assert L.mth_c2p_ctx_run(ctx, gamma, n, cons.data_ptr(), prims.data_ptr(),
                                     aux.data_ptr(), 1, guess, None) == 0
            st = _lib.C2PBatchStats()
            assert L.mth_c2p_ctx_stats(ctx, None, C.byref(st)) == 0
            assert st.cells == n and st.unconverged == 0, guess
            rel = ((prims[0] - truth[0]).abs() / truth[0]).max().item()
            assert rel < 1e-8, (guess, rel)
    finally:
        L.mth_c2p_ctx_destroy(ctx)


def test_ensemble_256_members_sampled_against_single_runs():
    import method_b200 as mb
    mem = initial.kh_ensemble(256, seed=2024)
    ens = mb.Ensemble([c for c, _ in mem])
    for m, (c, ic) in enumerate(mem):
        ens.set_prims(m, initial.kelvin_helmholtz(**ic))
    ens.autotune(reps=1)
    ens.step(4)
    sizes = [c["nx"] for c, _ in mem]
    sample = {int(np.argmin(sizes)), int(np.argmax(sizes))}
    sample |= {next(i for i, (c, _) in enumerate(mem) if c["model"] == "srrmhd"),
               next(i for i, (c, _) in enumerate(mem) if c["model"] == "srmhd")}
    for m in range(len(mem)):
        st = ens.stats(m)
        assert st["iters"] == 4 and st["c2p_unconverged"] == 0 and st["implicit_failed"] == 0
    for m in sample:
        c, ic = mem[m]
        s = mb.Simulation(**c)
        s.set_prims(initial.kelvin_helmholtz(**ic))
        s.update_time(4)
        for name, a, b in zip(("cons", "prims", "aux"), ens.state(m), s.state()):
            assert np.array_equal(a, b), (m, name)
        s.close()
    ens.close()


def test_ot1024_50_steps_match_reference(ref):
    """The measured configuration for its first 50 updateTime calls (slow start
    included), against the reference build's OpenMP form (its threads split
    the WENO/FVS loops only; the arithmetic is the serial build's)."""
    import method_b200 as mb
    if not ref.available(omp=True):
        pytest.skip("OpenMP reference build missing")
    n, steps = 1024, 50
    p0 = initial.orszag_tang(n, Ng=4)
    g = mb.Simulation(nx=n, ny=n, **OT)
    g.set_prims(p0)
    g.update_time(steps)
    r = ref.RefSim(prims=p0, omp=True, nx=n, ny=n, **OT)
    assert r.update_time(steps) == 0
    assert g.stats()["iters"] == r.iters == steps
    for name, a, b in zip(("cons", "prims", "aux"), g.state(), r.state()):
        assert np.array_equal(a, b), name


@pytest.mark.parametrize("seed", [3, 0, 10])
def test_sheet64x128_ssp2_matches_reference_at_seeded_sigma(ref, seed):
    """The resistive current-sheet workload at reduced size (64x128), IMEX
    SSP2, 10 updateTime calls, conductivity drawn per run as 10^U(1, 5) from
    the seed (seeds 3, 0, 10: sigma 22, 3.5e3, 6.7e4)."""
    import method_b200 as mb
    sigma = initial.sigma_for_seed(seed)
    cfg = dict(model="srrmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=sigma, weno=3,
               bcs="outflow", integrator="ssp2")
    p0 = initial.current_sheet(64, 128, seed=seed)
    g = mb.Simulation(**cfg)
    g.set_prims(p0)
    g.update_time(10)
    st = g.stats()
    assert st["status"] == 0 and st["implicit_failed"] == 0
    r = ref.RefSim(prims=p0, **cfg)
    assert r.update_time(10) == 0
    for name, a, b in zip(("cons", "prims", "aux"), g.state(), r.state()):
        assert np.array_equal(a, b), (name, sigma)
