"""GPU checks of the C++ drop-in classes (include/method_b200/method.hpp).

A reference-style driver (tests/cpp/kh_main.cc: Data, SRMHD, Weno3, FVS,
Flow, Simulation, RK2 wired as in the reference's examples) is built against
the drop-in headers, run, and its final state compared with the reference CPU
build run on the same initial data through the reference's own classes.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_reference_style_driver_matches_reference(tmp_path, ref):
    exe = tmp_path / "kh_main"
    r = subprocess.run(["g++", "-std=c++11", "-O2", "-I",
                        os.path.join(ROOT, "include", "method_b200"),
                        os.path.join(ROOT, "tests", "cpp", "kh_main.cc"), "-o", str(exe),
                        "-L", os.path.join(ROOT, "method_b200"), "-lmethod_b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "method_b200")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out, init = tmp_path / "state.bin", tmp_path / "prims0.bin"
    import tempfile
    textdir = tempfile.mkdtemp(prefix="kh", dir="/tmp")  # the reference keeps dir in char[50]
    refdir = tempfile.mkdtemp(prefix="khr", dir="/tmp")
    for d in (textdir, refdir):
        for sub in ("Conserved", "Primitive", "Auxiliary", "Domain", "Constants"):
            os.makedirs(os.path.join(d, sub))
    r = subprocess.run([str(exe), str(out), str(init), textdir], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    Nx, Ny = 72, 136
    data = np.fromfile(out, dtype=np.float64)
    cons = data[:9 * Nx * Ny].reshape(9, Nx, Ny, 1)
    prims = data[9 * Nx * Ny:].reshape(8, Nx, Ny, 1)
    prims0 = np.fromfile(init, dtype=np.float64).reshape(8, Nx, Ny, 1)

    # the reference classes on the driver's initial data, same 20 updateTime calls
    cfg = dict(model="srmhd", nx=64, ny=128, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0,
               endTime=3.0, cfl=0.4, Ng=4, gamma=4.0 / 3.0, sigma=0.0, weno=3, bcs="flow",
               integrator="rk2")
    rs = ref.RefSim(prims=prims0, **cfg)
    rs.update_time(20)
    rc, rp, _ = rs.state()
    assert np.array_equal(cons, rc)
    assert np.array_equal(prims, rp)
    # SerialSaveData files of the drop-in classes == the reference's, byte for byte
    assert rs.save_text(refdir, "") == 0
    for f in ("Conserved/cons.dat", "Primitive/prims.dat", "Auxiliary/aux.dat",
              "Domain/domain.dat", "Constants/constants.dat"):
        a = open(os.path.join(refdir, f), "rb").read()
        b = open(os.path.join(textdir, f), "rb").read()
        assert a == b, f


def test_single_cell_c2p_batch_matches_oracle():
    """mth_c2p_cells (getPrimitiveVarsSingleCell on n cells) vs the oracle's hybrd1."""
    import ctypes as C

    from method_b200 import _lib, initial
    from oracle import port

    L = _lib.load()
    n = 4096
    p = initial.random_c2p_states(n, seed=3)
    # conserved states from the oracle's primsToAll on a 1D strip of n cells
    s = port.PortSim(np.concatenate([np.repeat(p[:, :1], 4, axis=1), p,
                                     np.repeat(p[:, -1:], 4, axis=1)], axis=1)[:, :, None, None],
                     model="srmhd", nx=n, ny=0, gamma=4.0 / 3.0, bcs="outflow")
    c, p0, a0 = s.state()
    cons = np.ascontiguousarray(c[:, 4:-4, 0, 0])
    prims = np.ascontiguousarray(p0[:, 4:-4, 0, 0] * 0.99)
    aux = np.ascontiguousarray(a0[:, 4:-4, 0, 0] * 0.99)
    D = C.POINTER(C.c_double)
    rc = L.mth_c2p_cells(0, 4.0 / 3.0, 0.0, n, cons.ctypes.data_as(D), prims.ctypes.data_as(D),
                         aux.ctypes.data_as(D), 1.4e-8, 0)
    assert rc in (0, 1)
    guess = np.stack([np.sum((p0[1:4, 4:-4, 0, 0] * 0.99) ** 2, axis=0),
                      (p0[0, 4:-4, 0, 0] * 0.99) * (a0[0, 4:-4, 0, 0] * 0.99) /
                      (1 - np.sum((p0[1:4, 4:-4, 0, 0] * 0.99) ** 2, axis=0))], axis=1)
    sol, info, _ = port.srmhd_c2p_cells(cons.T, guess, 4.0 / 3.0, tol=1.4e-8)
    ok = info == 1
    # converged cells: the device's W and rho h W^2 follow the oracle's solution exactly
    W = 1.0 / np.sqrt(1.0 - sol[ok, 0])
    assert np.array_equal(aux[1, ok], W)
    assert (rc == 1) == (not np.all(ok))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_regime_driver_matches_reference(tmp_path, ref):
    """tests/cpp/regime_main.cc: REGIME(&data, &fvs) handed to RKSplit, as the
    reference's REGIME examples wire it, against the reference CPU build."""
    exe = tmp_path / "regime_main"
    r = subprocess.run(["g++", "-std=c++11", "-O2", "-I",
                        os.path.join(ROOT, "include", "method_b200"),
                        os.path.join(ROOT, "tests", "cpp", "regime_main.cc"), "-o", str(exe),
                        "-L", os.path.join(ROOT, "method_b200"), "-lmethod_b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "method_b200")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out, init = tmp_path / "state.bin", tmp_path / "prims0.bin"
    r = subprocess.run([str(exe), str(out), str(init)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    Nx = Ny = 48
    data = np.fromfile(out, dtype=np.float64)
    cons = data[:9 * Nx * Ny].reshape(9, Nx, Ny, 1)
    prims = data[9 * Nx * Ny:].reshape(8, Nx, Ny, 1)
    prims0 = np.fromfile(init, dtype=np.float64).reshape(8, Nx, Ny, 1)
    cfg = dict(model="srmhd", nx=40, ny=40, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, endTime=1.0,
               cfl=0.4, Ng=4, gamma=2.0, sigma=1e3, weno=3, bcs="periodic",
               integrator="rksplit", regime=True)
    rs = ref.RefSim(prims=prims0, **cfg)
    rs.update_time(5)
    rc, rp, _ = rs.state()
    rs.close()
    assert np.array_equal(cons, rc)
    assert np.array_equal(prims, rp)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_hybrid_driver_matches_reference(tmp_path, ref):
    """tests/cpp/hybrid_main.cc: Hybrid(&data, 150, 50, true) with
    setupREGIME and RKSplit2, as the reference's Hybrid examples wire it, on
    the reference's OTVortexSingleFluid, against the reference CPU build."""
    exe = tmp_path / "hybrid_main"
    r = subprocess.run(["g++", "-std=c++11", "-O2", "-I",
                        os.path.join(ROOT, "include", "method_b200"),
                        os.path.join(ROOT, "tests", "cpp", "hybrid_main.cc"), "-o", str(exe),
                        "-L", os.path.join(ROOT, "method_b200"), "-lmethod_b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "method_b200")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out, init = tmp_path / "state.bin", tmp_path / "prims0.bin"
    r = subprocess.run([str(exe), str(out), str(init)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    Nx = Ny = 40
    data = np.fromfile(out, dtype=np.float64)
    cons = data[:14 * Nx * Ny].reshape(14, Nx, Ny, 1)
    prims = data[14 * Nx * Ny:].reshape(11, Nx, Ny, 1)
    prims0 = np.fromfile(init, dtype=np.float64).reshape(11, Nx, Ny, 1)
    cfg = dict(model="hybrid", nx=32, ny=32, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
               endTime=1.0, cfl=0.3, Ng=4, gamma=2.0, sigma=170.0, cp=1.0, weno=3,
               bcs="periodic", integrator="rksplit2", sigmaCrossOver=150.0, sigmaSpan=50.0,
               useREGIME=True)
    rs = ref.RefSim(init="ot", **cfg)
    assert np.array_equal(prims0, rs.state()[1])
    rs.update_time(8)
    rc, rp, _ = rs.state()
    rs.close()
    assert np.array_equal(cons, rc)
    assert np.array_equal(prims, rp)
