"""CPU checks of the boundary: the C-ABI library loads and exports every
symbol include/method_b200.h declares, configuration errors are rejected on
the host, and a reference-style C++ driver builds against the drop-in headers."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "method_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(mth_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from method_b200 import _lib
    L = _lib.load()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, f"symbols declared but not exported: {missing}"
    assert set(declared_symbols()) == set(_lib.SYMBOLS)


def test_invalid_configuration_rejected_on_host():
    import method_b200 as mb
    with pytest.raises(ValueError):  # WENO5 needs Ng >= 4 (weno.cc:13-20)
        mb.Simulation(nx=16, ny=16, Ng=3, weno=5)
    with pytest.raises(ValueError):  # sigma >= 0 (simData.cc:100-102)
        mb.Simulation(nx=16, ny=16, sigma=-1.0)
    with pytest.raises(ValueError):  # SSP2 is provided for SRRMHD
        mb.Simulation(nx=16, ny=16, model="srmhd", integrator="ssp2")
    for integ in ("ssp3", "ssp2322"):  # so are SSP3 and SSP2322
        with pytest.raises(ValueError):
            mb.Simulation(nx=16, ny=16, model="srmhd", integrator=integ)
    with pytest.raises(ValueError):  # a 3D grid needs ny > 0 (simData.cc:66-84)
        mb.Simulation(nx=16, ny=0, nz=8)
    with pytest.raises(ValueError):  # WENO orders 3, 5, 7, 9, 11 (weno.h)
        mb.Simulation(nx=16, ny=16, Ng=8, weno=6)
    with pytest.raises(ValueError):  # WENO7 needs Ng >= 5
        mb.Simulation(nx=16, ny=16, Ng=4, weno=7)
    with pytest.raises(KeyError):  # no such boundary class
        mb.Simulation(nx=16, ny=16, bcs="reflective")


def test_invalid_ensembles_rejected_on_host():
    import method_b200 as mb
    base = dict(nx=32, ny=64, model="srmhd", integrator="rk2", precision="mixed")
    bad = [
        [base, dict(base, nz=8)],                                   # 3D member
        [base, dict(base, precision="fp64")],                       # mixed precisions
        [base, dict(base, weno=5)],                                 # mixed WENO orders
        [dict(base, model="srrmhd", integrator="ssp2", precision="fp64")],  # plain SSP2 member
        [dict(base, model="srrmhd", integrator="rk2")],             # SRRMHD needs SSP2 here
        [dict(base, ny=0)],                                         # 1D member
        [dict(base, guess="mlp", precision="fp64")],                # learned guess needs mixed
    ]
    for members in bad:
        with pytest.raises(ValueError):
            mb.Ensemble(members)
    with pytest.raises(ValueError):  # no members
        mb.Ensemble([])


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_reference_style_driver_builds(tmp_path):
    exe = tmp_path / "kh_main"
    cmd = ["g++", "-std=c++11", "-O2", "-I", os.path.join(ROOT, "include", "method_b200"),
           os.path.join(ROOT, "tests", "cpp", "kh_main.cc"), "-o", str(exe),
           "-L", os.path.join(ROOT, "method_b200"), "-lmethod_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "method_b200")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_regime_configuration_rules():
    """The REGIME extension runs with SRMHD and RKSplit in one or two
    dimensions; other combinations are rejected on the host."""
    import method_b200 as mb
    base = dict(nx=16, ny=16, Ng=4, weno=3, bcs="periodic", regime=True)
    for bad in (dict(model="srrmhd", integrator="rksplit"), dict(model="srmhd", integrator="rk2"),
                dict(model="srmhd", integrator="rksplit", nz=16)):
        with pytest.raises(ValueError):
            mb.Simulation(**dict(base, **bad))


def test_hybrid_configuration_rules():
    """The Hybrid model runs with RK2 or RKSplit2, previous-state guesses and a
    positive blend width; other combinations are rejected on the host."""
    import method_b200 as mb
    base = dict(nx=16, ny=16, Ng=4, weno=3, bcs="periodic", model="hybrid")
    for bad in (dict(integrator="ssp2"),
                dict(integrator="rksplit"), dict(integrator="rk2", sigmaSpan=0.0),
                dict(integrator="rk2", guess="mlp")):
        with pytest.raises(ValueError):
            mb.Simulation(**dict(base, **bad))
