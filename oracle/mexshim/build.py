"""Build recipe for the MEX runtime stand-in and the reference's own MEX kernels.

TEST INFRASTRUCTURE ONLY.  Outputs go to ``oracle/_ref/`` (git-ignored; the
built files travel with the tree to the GPU machine, where the reference's
sources are not available):

* ``libmexshim.so``          the stand-in runtime (oracle/mexshim/mexshim.cpp);
* ``ref_decompBlockLU.so``   Runtime/solver/decompBlockLU.cu of the reference,
* ``ref_applyBlockLU.so``    Runtime/solver/applyBlockLU.cu of the reference,
                             each compiled unchanged from the reference tree
                             (its own block_lu_mex_utils.h beside it) against
                             the stand-in's mex.h / gpu/mxGPUArray.h, linked
                             with cuSOLVER and cuBLAS as wust_build_mex.m:7-8
                             links them (mexcuda -lcusolver -lcublas), for
                             sm_100a.

``build_gateway`` compiles one of this repository's MEX gateways
(waveforminversionust_b200/mex/*.c) against the stand-in for the tests.

The reference location is taken from the WUST_REFERENCE_ROOT environment
variable, default ``/root/reference``; without it only the stand-in is built.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
OUT = os.path.join(ORACLE, "_ref")
SHIM = os.path.join(OUT, "libmexshim.so")
REF_SOLVER = os.path.join("Runtime", "solver")
REF_KERNELS = {"decompBlockLU": "ref_decompBlockLU.so", "applyBlockLU": "ref_applyBlockLU.so"}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_lib() -> str:
    return os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(_nvcc()))), "lib64")


def _stale(target: str, deps: list[str]) -> bool:
    return not os.path.exists(target) or any(os.path.getmtime(d) > os.path.getmtime(target) for d in deps)


def _headers() -> list[str]:
    return [os.path.join(HERE, "mex.h"), os.path.join(HERE, "matrix.h"), os.path.join(HERE, "gpu", "mxGPUArray.h")]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_shim(verbose: bool = False) -> str:
    src = os.path.join(HERE, "mexshim.cpp")
    os.makedirs(OUT, exist_ok=True)
    if _stale(SHIM, [src] + _headers()):
        tmp = SHIM + ".tmp"
        _run([_nvcc(), "-std=c++17", "-O2", *ARCH, "-shared", "-Xcompiler", "-fPIC", "-I", HERE, src, "-o", tmp],
             verbose)
        os.replace(tmp, SHIM)
    return SHIM


def reference_root() -> str:
    return os.environ.get("WUST_REFERENCE_ROOT", "/root/reference")


def build_reference(verbose: bool = False) -> dict:
    """Compile the reference's two MEX kernels where its sources are present."""
    build_shim(verbose)
    src_dir = os.path.join(reference_root(), REF_SOLVER)
    built = {}
    if not os.path.isdir(src_dir):
        return built
    for name, lib in REF_KERNELS.items():
        src = os.path.join(src_dir, name + ".cu")
        out = os.path.join(OUT, lib)
        deps = [src, os.path.join(src_dir, "block_lu_mex_utils.h"), SHIM] + _headers()
        if _stale(out, deps):
            tmp = out + ".tmp"
            _run([_nvcc(), "-std=c++17", "-O3", *ARCH, "-shared", "-Xcompiler", "-fPIC", "-I", HERE, src,
                  "-L", OUT, "-lmexshim", "-L", _cuda_lib(), "-lcusolver", "-lcublas",
                  "-Xlinker", "-rpath,$ORIGIN", "-Xlinker", "-rpath," + _cuda_lib(), "-o", tmp], verbose)
            os.replace(tmp, out)
        built[name] = out
    return built


def reference_kernels() -> dict:
    """Paths of the prebuilt reference MEX kernels (empty if not built)."""
    return {n: os.path.join(OUT, lib) for n, lib in REF_KERNELS.items() if os.path.exists(os.path.join(OUT, lib))}


def build_gateway(src: str, out: str, verbose: bool = False) -> str:
    """One of this repository's C MEX gateways against the stand-in and libwust_b200."""
    build_shim(verbose)
    lib_dir = os.path.join(ROOT, "waveforminversionust_b200")
    cc = shutil.which("gcc") or "gcc"
    _run([cc, "-std=c99", "-O2", "-fPIC", "-shared", "-fexceptions", "-Wall", "-Werror", "-I", HERE,
          "-I", os.path.join(ROOT, "include"), src, "-L", OUT, "-lmexshim", "-L", lib_dir, "-lwust_b200",
          "-Wl,-rpath," + OUT, "-Wl,-rpath," + lib_dir, "-o", out], verbose)
    return out


if __name__ == "__main__":
    print(build_reference(verbose="-v" in sys.argv))
