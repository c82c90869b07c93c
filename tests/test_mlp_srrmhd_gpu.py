"""The learned guess for the resistive model (SRRMHD): a network trained by the
project's own kernels on pairs the solver generates (SRRMHD primsToAll of
random states), seeding the recovery's Newton in Z = rho h W^2 and the inner
recoveries of the SSP2 implicit stages.  The previous state's Z stays the
fallback and the judge: every cell must converge to the same tolerance, and
what the network gains is the Newton work on starts that are not already at
the root."""
import ctypes as C

import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu

F = C.POINTER(C.c_float)
D = C.POINTER(C.c_double)

SHEET = dict(model="srrmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
             endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3, weno=3, bcs="outflow",
             integrator="ssp2", precision="mixed")


@pytest.fixture(scope="module")
def net():
    import method_b200 as mb
    P, S, loss = mb.train_guess(model="srrmhd", seed=11)
    assert np.isfinite(loss) and loss < 0.05, loss
    return P, S


def features_srrmhd(c):
    """NumPy restatement of the device's SRRMHD feature map (mlp.cuh)."""
    D_ = c[0]
    sx = c[1] - (c[9] * c[7] - c[10] * c[6])
    sy = c[2] - (c[10] * c[5] - c[8] * c[7])
    sz = c[3] - (c[8] * c[6] - c[9] * c[5])
    S2 = sx * sx + sy * sy + sz * sz
    tb = c[4] - 0.5 * (c[5] ** 2 + c[6] ** 2 + c[7] ** 2 + c[8] ** 2 + c[9] ** 2 + c[10] ** 2)
    E = tb + D_
    return np.stack([np.log10(np.maximum(tb / D_, 1e-30)), np.log10(S2 / D_ ** 2 + 1e-30),
                     np.log10(1 + np.maximum(tb / D_, 0)), np.sqrt(S2) / E,
                     np.log10(S2 / E ** 2 + 1e-30), S2 / E ** 2, D_ / E, 0 * D_], axis=1)


def test_pairs_and_network_predict_z(net):
    """Solver-generated pairs: the device features equal their NumPy
    restatement, the targets are the generating state's log10(Z/D) and v^2,
    and the trained network predicts Z on fresh pairs."""
    from method_b200 import _lib
    L = _lib.load()
    P, S = net
    n = 4096
    feat = np.zeros((n, 8), dtype=np.float32)
    tgt = np.zeros((n, 2), dtype=np.float32)
    cons = np.zeros((14, n))
    prims = np.zeros((11, n))
    assert L.mth_mlp_make_pairs_srrmhd(n, 12345, 4.0 / 3.0, feat.ctypes.data_as(F),
                                       tgt.ctypes.data_as(F), cons.ctypes.data_as(D),
                                       prims.ctypes.data_as(D), 0) == 0
    np.testing.assert_allclose(feat, features_srrmhd(cons), rtol=2e-5, atol=2e-5)
    g = 4.0 / 3.0
    W = 1 / np.sqrt(1 - np.sum(prims[1:4] ** 2, axis=0))
    h = 1 + prims[4] / prims[0] * g / (g - 1)
    Z = prims[0] * h * W * W
    np.testing.assert_allclose(tgt[:, 0], np.log10(Z / cons[0]), rtol=1e-5, atol=1e-5)
    x = ((feat - S[:8]) * S[8:16]).astype(np.float32)
    y = np.zeros((n, 2), dtype=np.float32)
    assert L.mth_mlp_forward(P.ctypes.data_as(F), n, x.ctypes.data_as(F),
                             y.ctypes.data_as(F), 0) == 0
    z_net = cons[0] * 10.0 ** (y[:, 0] * S[18] + S[16])
    rel = np.abs(z_net - Z) / Z
    assert np.median(rel) < 0.1, np.median(rel)


def _sheet_sim(guess, net):
    import method_b200 as mb
    s = mb.Simulation(guess=guess, **SHEET)
    if guess == "mlp":
        s.set_mlp(*net)
    s.set_prims(initial.current_sheet(64, 128, seed=4))
    return s


def test_network_seeded_ssp2_matches_previous_guess(net):
    """SSP2 on the current sheet with the network seeding every recovery and
    implicit stage: every cell converges, and the state equals the run seeded
    by the previous state to the solvers' tolerance."""
    runs = {}
    for guess in ("previous", "mlp"):
        s = _sheet_sim(guess, net)
        s.update_time(6)
        st = s.stats()
        assert st["status"] == 0 and st["c2p_unconverged"] == 0 and st["implicit_failed"] == 0
        runs[guess] = (s.state(), st)
        s.close()
    (a, _), (b, _) = runs["mlp"], runs["previous"]
    for name, x, y in zip(("cons", "prims"), a[:2], b[:2]):
        core = (slice(None), slice(4, -4), slice(4, -4))
        l1 = np.abs(x[core] - y[core]).sum() / np.abs(y[core]).sum()
        assert l1 < 1e-9, (name, l1)


def test_network_gains_on_cold_starts(net):
    """Recovery of 64 x 64 random resistive states (Lorentz factors 1-10, the
    pairs' distributions) from a Z guess 40% off, as after a restart from
    primitive data without aux: the network's start needs fewer Newton steps
    per cell than the stale guess, and both recover the generating state."""
    import method_b200 as mb
    from method_b200 import _lib
    L = _lib.load()
    n, Ng = 64, 4
    feat = np.zeros((n * n, 8), dtype=np.float32)
    tgt = np.zeros((n * n, 2), dtype=np.float32)
    cons1 = np.zeros((14, n * n))
    prims1 = np.zeros((11, n * n))
    assert L.mth_mlp_make_pairs_srrmhd(n * n, 777, 4.0 / 3.0, feat.ctypes.data_as(F),
                                       tgt.ctypes.data_as(F), cons1.ctypes.data_as(D),
                                       prims1.ctypes.data_as(D), 0) == 0
    g = 4.0 / 3.0
    W = 1 / np.sqrt(1 - np.sum(prims1[1:4] ** 2, axis=0))
    Z = prims1[0] * (1 + prims1[4] / prims1[0] * g / (g - 1)) * W * W
    N = n + 2 * Ng
    core = (slice(None), slice(Ng, -Ng), slice(Ng, -Ng), 0)
    cons = np.zeros((14, N, N, 1))
    cons[core] = cons1.reshape(14, n, n)
    out = {}
    for guess in ("previous", "mlp"):
        s = mb.Simulation(model="srrmhd", nx=n, ny=n, Ng=Ng, gamma=g, sigma=1e3, weno=3,
                          bcs="periodic", integrator="ssp2", precision="mixed", guess=guess)
        if guess == "mlp":
            s.set_mlp(*net)
        prims = np.zeros((11, N, N, 1))
        aux = np.zeros((17, N, N, 1))
        aux[10][core[1:]] = (1.4 * Z).reshape(n, n)
        s.upload(cons, prims, aux)
        s.reset_stats()
        s.c2p()
        st = s.stats()
        assert st["status"] == 0 and st["c2p_unconverged"] == 0
        _, p, _ = s.state()
        rel = np.abs(p[0][core[1:]] - prims1[0].reshape(n, n)) / prims1[0].reshape(n, n)
        assert rel.max() < 1e-8, (guess, rel.max())
        out[guess] = st["c2p_evals"] / st["c2p_cells"]
        s.close()
    assert out["mlp"] < out["previous"], out


def test_ensemble_resistive_members_with_network_equal_single_runs(net):
    """The ensemble's resistive members seeded by the network equal single
    runs with the same network, bit for bit."""
    import method_b200 as mb
    mem = []
    for k, (model, nx) in enumerate((("srrmhd", 64), ("srmhd", 64), ("srrmhd", 96))):
        c = dict(model=model, integrator="ssp2" if model == "srrmhd" else "rk2", nx=nx,
                 ny=2 * nx, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0, endTime=3.0, cfl=0.4,
                 Ng=4, gamma=4.0 / 3.0, sigma=3e3 if model == "srrmhd" else 0.0, weno=3,
                 bcs="flow", precision="mixed", guess="mlp")
        mem.append((c, dict(nx=nx, ny=2 * nx, Ng=4, seed=90 + k, model=model, shear=0.4)))
    ens = mb.Ensemble([c for c, _ in mem])
    ens.set_mlp(*net, model="srrmhd")
    for m, (c, ic) in enumerate(mem):
        ens.set_prims(m, initial.kelvin_helmholtz(**ic))
    ens.step(3)
    for m, (c, ic) in enumerate(mem):
        st = ens.stats(m)
        assert st["c2p_unconverged"] == 0 and st["implicit_failed"] == 0
        if c["model"] != "srrmhd":
            continue
        s = mb.Simulation(**c)
        s.set_mlp(*net)
        s.set_prims(initial.kelvin_helmholtz(**ic))
        s.update_time(3)
        for name, a, b in zip(("cons", "prims", "aux"), ens.state(m), s.state()):
            assert np.array_equal(a, b), (m, name)
        s.close()
    ens.close()
