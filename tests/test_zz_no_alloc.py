"""The allocation-free SRMHD primitive recovery, checked against mth_c2p.

mth_c2p_srmhd_noalloc exists for callers that may not allocate device memory
themselves -- an application that owns every device buffer through its own
fixed-budget pool, or a stepping loop that cannot afford cudaMalloc and the
synchronisation it may bring.  Such a caller passes its own device arrays;
the entry point keeps its failure queue and counters in one fixed device
array instead of allocating them.

The first test gives both entry points the same state and the same guesses (a
few isolated cells get an unphysical guess, so that the Powell-hybrid solve
fails there and the neighbour-average retry -- the part that uses the fixed
array -- runs), on two calls in a row, and asks for agreement to 1e-12
relative, the tolerance of the other GPU parity tests.  The second puts failing
cells next to the boundary, where the retry averages ghost-cell solution values
that the caller supplies (one of them absurd, so that the retry fails too), and
checks prims, aux, the solution array and the reported unconverged count
against the oracle given the same solution array.  The device buffers of the
allocation-free calls come from torch: the test is the caller that owns memory.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel_err(a, b):
    """Largest relative difference; a NaN must sit at the same place in both
    (a retry that fails leaves the same NaN state in either entry point)."""
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return float("inf")
    a, b = np.where(na, 0.0, a), np.where(nb, 0.0, b)
    d = np.abs(a - b)
    return float(np.max(np.where(np.abs(b) > 1e-12, d / np.maximum(np.abs(b), 1e-300), d)))


def _ot_state(n, Ng, steps=3):
    import method_b200 as mb
    from method_b200 import initial

    cfg = dict(model="srmhd", nx=n, ny=n, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1.0,
               cfl=0.4, Ng=Ng, gamma=4.0 / 3.0, weno=5, bcs="periodic", integrator="rk2")
    sim = mb.Simulation(**cfg)
    sim.set_prims(initial.orszag_tang(n, Ng=Ng))
    sim.update_time(steps)
    return sim, cfg


def _noalloc(L, n, Ng, gamma, cons, pg, ag, sol):
    """One call on torch-owned device arrays; returns (prims, aux, unconverged)."""
    import torch

    dc = torch.from_numpy(cons).cuda()
    dpg = torch.from_numpy(pg).cuda()
    dag = torch.from_numpy(ag).cuda()
    dp = dpg.clone()
    da = dag.clone()
    still = C.c_longlong(-1)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.mth_c2p_srmhd_noalloc(n, n, 0, Ng, gamma, dc.data_ptr(), dpg.data_ptr(),
                                 dag.data_ptr(), dp.data_ptr(), da.data_ptr(), sol.data_ptr(),
                                 stream, C.byref(still))
    assert rc == 0
    torch.cuda.synchronize()
    return dp.cpu().numpy(), da.cpu().numpy(), still.value


def test_noalloc_c2p_matches_existing_entry_point():
    import torch

    from method_b200 import _lib
    from oracle import port

    n, Ng, gamma = 128, 4, 4.0 / 3.0
    sim, _ = _ot_state(n, Ng)
    cons, prims, aux = sim.state()
    L = _lib.load()
    Ntot = cons.shape[1] * cons.shape[2] * cons.shape[3]
    sol = torch.zeros(2 * Ntot, dtype=torch.float64, device="cuda")
    bad = [(20, 30), (47, 90), (100, 11), (64, 64)]  # isolated interior cells
    for call in range(2):
        rng = np.random.default_rng(call)
        pg = np.ascontiguousarray(prims * (1.0 + 0.02 * (rng.random(prims.shape) - 0.5)))
        ag = np.ascontiguousarray(aux.copy())
        for (i, j) in bad:
            pg[1, Ng + i, Ng + j, 0] = 1.5  # v^2 > 1: the residual is flat, hybrd1 fails
        # the failing cells really take the retry path
        cells = np.array([[cons[v, Ng + i, Ng + j, 0] for v in range(9)] for (i, j) in bad])
        guess = []
        for (i, j) in bad:  # the kernel's guess (srmhd.cc:438-442)
            v2 = sum(pg[v, Ng + i, Ng + j, 0] ** 2 for v in (1, 2, 3))
            guess.append([v2, pg[0, Ng + i, Ng + j, 0] * ag[0, Ng + i, Ng + j, 0] / (1 - v2)])
        guess = np.array(guess)
        _, info, _ = port.srmhd_c2p_cells(cells, guess, gamma)
        assert np.all(info != 1)

        # existing entry point: the handle's own scratch
        sim.reset_stats()
        sim.upload(cons, pg, ag)
        sim.c2p()
        _, p_ref, a_ref = sim.state()
        want_still = sim.stats()["c2p_unconverged"]

        # allocation-free entry point on caller-owned device arrays
        p_got, a_got, still = _noalloc(L, n, Ng, gamma, cons, pg, ag, sol)
        assert rel_err(p_got, p_ref) <= RTOL, f"call {call}: prims"
        assert rel_err(a_got, a_ref) <= RTOL, f"call {call}: aux"
        assert still == want_still, f"call {call}: unconverged {still} vs {want_still}"
    sim.close()


def test_noalloc_retry_at_boundary_matches_oracle():
    import torch

    from method_b200 import _lib
    from oracle import port

    n, Ng, gamma = 64, 4, 4.0 / 3.0
    sim, cfg = _ot_state(n, Ng)
    cons, prims, aux = sim.state()
    sim.close()
    L = _lib.load()
    orc = port.PortSim(prims, **cfg)
    orc.set_state(cons, prims, aux)
    # a converged solution array of this state, ghost cells filled by the caller
    orc.c2p(cons.copy(), prims.copy(), aux.copy())
    sol0, still0 = orc.solution()
    assert still0 == 0
    for g in range(Ng):  # periodic copies: nonzero, plausible ghost solutions
        sol0[:, g, :, :] = sol0[:, n + g, :, :]
        sol0[:, n + Ng + g, :, :] = sol0[:, Ng + g, :, :]
        sol0[:, :, g, :] = sol0[:, :, n + g, :]
        sol0[:, :, n + Ng + g, :] = sol0[:, :, Ng + g, :]
    sol0[:, Ng - 1, Ng + 40, 0] = (50.0, -1.0e3)  # an absurd ghost value: that retry fails
    sol = torch.from_numpy(sol0.reshape(-1).copy()).cuda()
    orc.solution(sol0)

    # failing cells: one interior, two beside the x = 0 face, one beside y = ny-1
    bad = [(30, 30), (0, 17), (0, 40), (25, n - 1)]
    for call in range(2):
        rng = np.random.default_rng(10 + call)
        pg = np.ascontiguousarray(prims * (1.0 + 0.02 * (rng.random(prims.shape) - 0.5)))
        ag = np.ascontiguousarray(aux.copy())
        for (i, j) in bad:
            pg[1, Ng + i, Ng + j, 0] = 1.5
        p_want, a_want = pg.copy(), ag.copy()
        orc.c2p(cons.copy(), p_want, a_want)
        sol_want, still_want = orc.solution()

        p_got, a_got, still = _noalloc(L, n, Ng, gamma, cons, pg, ag, sol)
        assert still_want >= 1, "the absurd ghost solution should defeat one retry"
        assert still == still_want, f"call {call}: unconverged {still} vs {still_want}"
        assert rel_err(p_got, p_want) <= RTOL, f"call {call}: prims"
        assert rel_err(a_got, a_want) <= RTOL, f"call {call}: aux"
        got_sol = sol.cpu().numpy().reshape(sol_want.shape)
        assert rel_err(got_sol, sol_want) <= RTOL, f"call {call}: solution"
    orc.close()


def test_noalloc_rejects_grids_beyond_capacity():
    import torch

    from method_b200 import _lib

    L = _lib.load()
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = x.data_ptr()
    # 2048 x 1024 interior cells exceed MTH_NOALLOC_MAX_CELLS (1 << 20); rejected before any launch
    rc = L.mth_c2p_srmhd_noalloc(2048, 1024, 0, 4, 4.0 / 3.0, p, p, p, p, p, p, None, None)
    assert rc == 3
    # few interior cells but ghost-inclusive cell ids beyond the int range
    rc = L.mth_c2p_srmhd_noalloc(8, 8, 0, 1 << 30, 4.0 / 3.0, p, p, p, p, p, p, None, None)
    assert rc == 3
    rc = L.mth_c2p_srmhd_noalloc(4, 4, 4, 700, 4.0 / 3.0, p, p, p, p, p, p, None, None)
    assert rc == 3
