"""One domain in x-slabs against the same domain on one handle.

Each slab is its own handle; the slabs of one domain are held by this
process and exchange their halos by device copies (LocalTransport), which is
the ordering NCCL ranks follow with one slab each (the transport's message
pairing is tested on CPU ranks in test_slab_cpu.py).  Every interior flux,
recovery and implicit solve sees the values it sees on the whole domain, so
the assembled slabs must equal the single run exactly, in the plain form
(itself bit-identical to the reference) and in the mixed form.
"""
import numpy as np
import pytest

from method_b200 import initial, slab

pytestmark = pytest.mark.gpu

CASES = {
    "ot_rk2_weno5_periodic": (dict(model="srmhd", nx=64, ny=64, xmin=0.0, xmax=1.0, ymin=0.0,
                                   ymax=1.0, endTime=1.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0,
                                   weno=5, bcs="periodic", integrator="rk2"),
                              lambda: initial.orszag_tang(64, Ng=4), 6),
    "kh_rk2_weno3_flow": (dict(model="srmhd", nx=48, ny=96, xmin=-0.5, xmax=0.5, ymin=-1.0,
                               ymax=1.0, endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=3,
                               bcs="flow", integrator="rk2"),
                          lambda: initial.kelvin_helmholtz(48, 96, seed=5), 6),
    "sheet_ssp2_outflow": (dict(model="srrmhd", nx=40, ny=64, xmin=-0.5, xmax=0.5, ymin=-1.0,
                                ymax=1.0, endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0,
                                sigma=1e3, weno=3, bcs="outflow", integrator="ssp2"),
                           lambda: initial.current_sheet(40, 64, seed=6), 4),
    "kh_rksplit_weno3_outflow": (dict(model="srmhd", nx=32, ny=64, xmin=-0.5, xmax=0.5,
                                      ymin=-1.0, ymax=1.0, endTime=3.0, cfl=0.4, Ng=4,
                                      gamma=4.0 / 3.0, weno=3, bcs="outflow",
                                      integrator="rksplit"),
                                 lambda: initial.kelvin_helmholtz(32, 64, seed=8), 4),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n_slabs", [2, 3])
@pytest.mark.parametrize("case", list(CASES))
def test_slabs_equal_single_domain(case, n_slabs, precision):
    import torch

    import method_b200 as mb
    cfg, mk, steps = CASES[case]
    if precision == "fp64" and cfg["integrator"] == "ssp2" and n_slabs == 3:
        pytest.skip("plain SSP2 covered by the 2-slab case")
    cfg = dict(cfg, precision=precision)
    p0 = mk()
    one = mb.Simulation(**cfg)
    one.set_prims(p0)
    one.update_time(steps)
    want = one.state()
    t_want = one.stats()["t"]
    one.close()

    dom = slab.SlabDomain(cfg, n_slabs, range(n_slabs), slab.LocalTransport(n_slabs, cfg["bcs"]),
                          torch)
    dom.set_prims(p0)
    dom.update_time(steps)
    got = slab.assemble(dom.local_states(), dom.extents, cfg["Ng"])
    for s in dom.slabs:
        assert s.sim.stats()["t"] == t_want
    dom.close()
    for name, a, b in zip(("cons", "prims", "aux"), got, want):
        assert a.shape == b.shape, name
        np.testing.assert_array_equal(a, b, err_msg=f"{case}: {name}")


def test_slab_handles_refuse_whole_steps():
    import method_b200 as mb
    cfg = dict(CASES["ot_rk2_weno5_periodic"][0], nx=32, x_slab=(0, 64))
    s = mb.Simulation(**cfg)
    with pytest.raises(ValueError):
        s.step(1e-3)
    s.close()
    with pytest.raises(ValueError):  # SSP3 has no part split
        mb.Simulation(**dict(cfg, model="srrmhd", integrator="ssp3"))
