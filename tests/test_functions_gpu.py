"""Model-level functions on the device against the reference build, each on
its own: Model::primsToAll, Bcs::apply, Model::fluxVector in every direction
(including the reference's SRRMHD z-direction flux, srrmhd.cc:159-171),
Model::sourceTerm and Model::getPrimitiveVars from a perturbed guess, for both
models in 2D and 3D.  Plain FP64: bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(model, n, nz, seed):
    """Smooth, physical primitive state on an n x n (x nz) grid with 4 ghosts."""
    rng = np.random.default_rng(seed)
    N = n + 8
    Nz = nz + 8 if nz else 1
    x = (np.arange(N) + 0.5 - 4) / n
    z = (np.arange(Nz) + 0.5 - 4) / max(nz, 1)
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    nv = 8 if model == "srmhd" else 11
    p = np.zeros((nv, N, N, Nz))
    k = rng.uniform(1, 3, 8)
    p[0] = 1.0 + 0.3 * np.sin(2 * np.pi * (k[0] * X + Z))
    p[1] = 0.3 * np.sin(2 * np.pi * k[1] * Y)
    p[2] = 0.2 * np.cos(2 * np.pi * (k[2] * X + Z))
    p[3] = 0.1 * np.sin(2 * np.pi * k[3] * (X + Y))
    p[4] = 1.0 + 0.2 * np.cos(2 * np.pi * k[4] * Y)
    p[5] = 0.5 * np.sin(2 * np.pi * k[5] * Y)
    p[6] = 0.5 * np.cos(2 * np.pi * k[6] * X)
    p[7] = 0.3 * np.sin(2 * np.pi * (k[7] * Z + X))
    if model == "srrmhd":  # E = -v x B plus a small resistive part
        p[8] = -(p[2] * p[7] - p[3] * p[6]) + 0.01 * np.sin(2 * np.pi * Z)
        p[9] = -(p[3] * p[5] - p[1] * p[7])
        p[10] = -(p[1] * p[6] - p[2] * p[5]) + 0.01 * np.cos(2 * np.pi * X)
    return p


CASES = [("srmhd", 24, 0), ("srmhd", 10, 10), ("srrmhd", 24, 0), ("srrmhd", 10, 10)]


@pytest.mark.parametrize("model,n,nz", CASES)
def test_model_functions_match_reference(ref, model, n, nz):
    import method_b200 as mb
    p = _state(model, n, nz, seed=n + nz)
    cfg = dict(model=model, nx=n, ny=n, nz=nz, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1,
               endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3, weno=3, bcs="periodic",
               integrator="rk2")
    g = mb.Simulation(**cfg)
    r = ref.RefSim(prims=p, **cfg)
    # primsToAll + Bcs::apply (Simulation::set)
    g.set_prims(p)
    rc, rp, ra = r.state()
    for name, a, b in zip(("cons", "prims", "aux"), g.state(), (rc, rp, ra)):
        assert np.array_equal(a, b), ("set", name)
    # fluxVector along every direction of the grid
    for d in range(3 if nz else 2):
        assert np.array_equal(g.flux_vector(d), r.flux_vector(rc, rp, ra, d)), ("flux", d)
    # sourceTerm
    assert np.array_equal(g.source(), r.source(rc, rp, ra)), "source"
    # getPrimitiveVars from a perturbed guess, then the boundaries
    pg, ag = rp * 0.98, ra * 0.98
    g.upload(cons=rc, prims=pg, aux=ag)
    g.c2p()
    g.apply_bcs()
    rp2, ra2 = pg.copy(), ag.copy()
    assert r.c2p(rc, rp2, ra2) == 0
    r.apply_bcs(rc, rp2, ra2)
    gc, gp, ga = g.state()
    assert np.array_equal(gp, rp2), "c2p prims"
    assert np.array_equal(ga, ra2), "c2p aux"
