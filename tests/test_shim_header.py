"""The header-only drop-ins for the reference's gpu:: and mixed_gpu:: APIs compile warning-free as C++17
and link against libcmd_b200.so (every cmd_* call they make resolves)."""
import subprocess

import pytest

from shim_build import PKG, ROOT, build_shim_program


@pytest.mark.parametrize("header", ["lattice_gpu_api.h", "mixed_lattice_gpu_api.h"])
def test_header_alone_compiles(header):
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-I",
                        str(ROOT / "include"), "-x", "c++", str(ROOT / "include" / "classical_spin" / "gpu" / header)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("source", ["shim_calls.cpp", "mixed_shim_calls.cpp"])
def test_call_sequence_links(tmp_path, source):
    if not (PKG / "libcmd_b200.so").exists():
        pytest.skip("libcmd_b200.so not built")
    exe = build_shim_program(tmp_path / "prog", source)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
