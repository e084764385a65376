"""Build recipe for the native library of the B200 LL MD path.

``python -m classical_mcmc_spin_b200.build`` compiles every CUDA/C++ source
under ``csrc/`` for sm_100a into ``libcmd_b200.so`` next to this file (in the
source tree, so the built library travels with the repository snapshot).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libcmd_b200.so"
BUILD = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]
SOURCES = ["cmd_api.cu", "resident.cu", "stream.cu", "global.cu", "rk45.cu", "adjoint.cu", "noalloc.cu", "mixed_api.cu",
           "spectrum.cu", "lattice_host.cpp"]
DRIVER = PKG / "cmd_spin_solver"          # command-line driver (csrc/spin_solver.cpp) over the C ABI


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libcmd_b200.so")
    return cand


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(Path(d).stat().st_mtime <= t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    """Compiles every source (in parallel, each object only when it is older than
    its source or any header) and links libcmd_b200.so."""
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    deps = [CSRC / s for s in SOURCES] + headers
    if not force and not ptxas_info and _newer(LIB, deps):
        build_driver(verbose, force)
        return LIB
    BUILD.mkdir(exist_ok=True)
    inc = ["-I", str(ROOT / "include"), "-I", str(CSRC)]
    jobs = []
    for src in SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        if not force and not ptxas_info and _newer(obj, [CSRC / src] + headers):
            continue
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *inc, "-c", str(CSRC / src), "-o", str(obj)]
        if ptxas_info and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(run, jobs))
    failed = [r for r in results if r.returncode != 0]
    for r in results:
        if verbose or r.returncode != 0:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
    if failed:
        raise RuntimeError(f"{len(failed)} source(s) failed to compile")
    objs = [str(BUILD / (Path(src).stem + ".o")) for src in SOURCES]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart", "-lcufft", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_driver(verbose, True)
    return LIB


def build_driver(verbose: bool = False, force: bool = False) -> Path:
    """The command-line driver, linked against libcmd_b200.so next to it."""
    deps = [CSRC / "spin_solver.cpp", LIB] + list((ROOT / "include").glob("*.h"))
    if not force and _newer(DRIVER, deps):
        return DRIVER
    cxx = shutil.which("g++") or "g++"
    tmp = DRIVER.with_suffix(".tmp")
    cmd = [cxx, "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(CSRC / "spin_solver.cpp"), "-o", str(tmp),
           "-L", str(PKG), "-lcmd_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, DRIVER)
    return DRIVER


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
