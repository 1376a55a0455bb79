"""Builds the CUDA library of zlatko_b200 for sm_100a, in-tree: zlatko_b200/_lib/libzlatko_b200.so.

    python -m zlatko_b200.build            # compile if any source is newer than the library
    python -m zlatko_b200.build --force

nvcc cross-compiles without a GPU; the library links only against the CUDA runtime.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libzlatko_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["fused_exposure.cu", "basis_revalue.cu", "row_stats.cu", "nested_inner.cu", "amc_fit.cu", "mlp.cu", "surrogate.cu", "capi.cu", "peaks.cu"]
CPP_SOURCES = ["plan_compiler.cpp", "hermite_proxy.cpp", "basis_plan.cpp"]
HEADERS = ["zk_device.cuh", "zk_kernels.h", "plan_compiler.h", "umma.cuh", "surrogate.cuh", "basis.cuh", "basis_plan.h"]


def _sources():
    return [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES]


def _deps():
    deps = _sources() + [os.path.join(CSRC, h) for h in HEADERS if os.path.exists(os.path.join(CSRC, h))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "zlatko_b200.h"))
    return deps


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in _deps())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(os.path.join(OUT_DIR, "obj"), exist_ok=True)
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", "-diag-suppress", "186,128", "-I", os.path.join(os.path.dirname(HERE), "include")]

    def compile_one(src: str) -> str:
        obj = os.path.join(OUT_DIR, "obj", os.path.basename(src) + ".o")
        cmd = [NVCC] + ARCH + common + ["-c", src, "-o", obj]
        if src.endswith(".cu") and ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose or ptxas_info:
            sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=4) as ex:
        objs = list(ex.map(compile_one, _sources()))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "--cudart", "static", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True, ptxas_info=a.ptxas_info))
