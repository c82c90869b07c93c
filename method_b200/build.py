"""In-tree build of libmethod_b200.so (sm_100a) with nvcc.

    python -m method_b200.build            # incremental
    python -m method_b200.build --force    # rebuild everything

Translation units and their floating-point contracts:
  kernels_fp64.cu   -fmad=false: the plain FP64 form must round every
                    expression like the reference's x86-64 build (no FMA).
  regime.cu         -fmad=false: the REGIME source extension, plain form.
  regime_mixed.cu   FMA allowed: its fused tile with FP32 stiff-flux WENO.
  hybrid.cu         -fmad=false: the Hybrid model (blended SRMHD / SRRMHD).
  kernels_mixed.cu  FMA allowed: FP32 flux path, Newton primitive recovery.
  mlp.cu            FMA allowed: guess-network inference / training kernels.
  api.cu            C-ABI, host logic only.
  ensemble.cu       C-ABI of ensembles (work lists, autotuner, step graph).
  textout.cu        SerialSaveData text output formatted on the device.
  shim.cc           C++ mirror of the reference's class API over the C-ABI.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmethod_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]

UNITS = [
    ("kernels_fp64.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("regime.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("hybrid.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("regime_mixed.cu", []),
    ("kernels_mixed.cu", []),
    ("mlp.cu", []),
    ("mlp_tc.cu", []),
    ("api.cu", []),
    ("noalloc.cu", []),
    ("ensemble.cu", []),
    ("textout.cu", []),
    ("shim.cc", []),
]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
        if f.endswith(".h")]


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _compile(src, flags):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [NVCC] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    if src.endswith(".cc"):
        cmd = [NVCC] + COMMON + flags + ["-x", "cu", "-c", src, "-o", obj] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = _headers()
    jobs = []
    objs = []
    for name, flags in UNITS:
        src = os.path.join(CSRC, name)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append((src, flags))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            futs = [ex.submit(_compile, s, f) for s, f in jobs]
            for fu in futs:
                fu.result()
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    if verbose:
        print(f"built {LIB} ({len(jobs)} unit(s) recompiled)")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(force=a.force)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
