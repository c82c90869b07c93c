"""TimeIntegrator::step on host arrays (`mth_step_host`, the call the
end-to-end benchmark times) against the same steps on device-resident state.

The handle that runs `step_host` first holds a different state on the device,
so any device array the call needed but did not refresh from the host arrays
would change the result (the mixed form uploads only the variables a step
reads).  The host arrays come back with boundary conditions applied, as the
reference's `finalise` leaves them.
"""
import ctypes as C

import numpy as np
import pytest

from method_b200 import initial

pytestmark = pytest.mark.gpu

OT = dict(model="srmhd", nx=64, ny=64, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1e9,
          cfl=0.4, Ng=4, gamma=4.0 / 3.0, weno=5, bcs="periodic", integrator="rk2")
SHEET = dict(model="srrmhd", nx=32, ny=64, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
             endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=1e3, weno=3, bcs="outflow")
# variables uploaded per call: (cons, prims, aux) counts
UPLOADED = {"srmhd-rk2-mixed": (9, 8, 7), "srrmhd-rk2-mixed": (14, 4, 6),
            "srrmhd-ssp2-mixed": (14, 0, 1)}


def _cases():
    ot0 = lambda: initial.orszag_tang(64, Ng=4)
    ot1 = lambda: initial.kelvin_helmholtz(64, 64, Ng=4, seed=5)
    sh0 = lambda: initial.current_sheet(32, 64, seed=3)
    sh1 = lambda: initial.current_sheet(32, 64, seed=8)
    for prec in ("fp64", "mixed"):
        yield f"srmhd-rk2-{prec}", dict(OT, precision=prec), ot0, ot1, 2e-3
        for integ in ("ssp2", "rk2"):
            yield (f"srrmhd-{integ}-{prec}", dict(SHEET, integrator=integ, precision=prec), sh0,
                   sh1, 2e-3)
    # mixed RK2 grids of 256 interior x-rows and more take the pipelined path
    # (blocks of 64 rows; a partial last block; periodic, flow and outflow x)
    yield ("srmhd-rk2-mixed-pipelined-periodic", dict(OT, nx=320, precision="mixed"),
           lambda: initial.orszag_tang(320, Ng=4)[:, :, :72],
           lambda: initial.kelvin_helmholtz(320, 64, Ng=4, seed=6), 1e-3)
    kh = dict(OT, nx=300, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0, bcs="flow",
              precision="mixed", weno=3)
    yield ("srmhd-rk2-mixed-pipelined-flow", kh,
           lambda: initial.kelvin_helmholtz(300, 64, Ng=4, seed=7),
           lambda: initial.kelvin_helmholtz(300, 64, Ng=4, seed=8), 1e-3)
    yield ("srrmhd-rk2-mixed-pipelined-outflow", dict(SHEET, nx=256, integrator="rk2",
                                                      precision="mixed"),
           lambda: initial.current_sheet(256, 64, seed=9),
           lambda: initial.current_sheet(256, 64, seed=10), 2e-4)


@pytest.mark.parametrize("name,cfg,init,other,dt", [pytest.param(*c, id=c[0]) for c in _cases()])
def test_step_host_matches_device_steps(name, cfg, init, other, dt):
    import method_b200 as mb
    dev = mb.Simulation(**cfg)
    dev.set_prims(init())
    hc, hp, ha = (np.array(a, copy=True) for a in dev.state())
    for _ in range(2):
        dev.step(dt)
    want = dev.state()
    dev.close()

    host = mb.Simulation(**cfg)
    host.set_prims(other())
    h2d, d2h = C.c_ulonglong(), C.c_ulonglong()
    assert host.L.mth_step_host_bytes(host.h, C.byref(h2d), C.byref(d2h)) == 0
    per = hc[0].nbytes
    nc, np_, na = UPLOADED.get(name.replace("-pipelined-periodic", "").replace(
        "-pipelined-flow", "").replace("-pipelined-outflow", ""),
        (hc.shape[0], hp.shape[0], ha.shape[0]))
    assert h2d.value == per * (nc + np_ + na), name
    assert d2h.value == hc.nbytes + hp.nbytes + ha.nbytes, name
    for _ in range(2):
        host.step_host(hc, hp, ha, dt)
    host.close()
    for what, a, b in zip(("cons", "prims", "aux"), (hc, hp, ha), want):
        assert np.array_equal(a, b), (name, what)
