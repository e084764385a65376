"""Builds the call-sequence programs tests/cpp/*.cpp against the header-only drop-ins
include/classical_spin/gpu/{lattice,mixed_lattice}_gpu_api.h and libcmd_b200.so (g++, no GPU needed)."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "classical_mcmc_spin_b200"


def build_shim_program(out: Path, source: str = "shim_calls.cpp") -> Path:
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "cpp" / source), "-o", str(out), "-L", str(PKG), "-lcmd_b200",
           f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    return out
