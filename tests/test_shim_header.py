"""The header-only drop-in for the reference's gpu:: API compiles warning-free as C++17 and links
against libcmd_b200.so (every cmd_* call it makes resolves)."""
import subprocess

import pytest

from shim_build import PKG, ROOT, build_shim_program


def test_header_alone_compiles():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-I",
                        str(ROOT / "include"), "-x", "c++",
                        str(ROOT / "include" / "classical_spin" / "gpu" / "lattice_gpu_api.h")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_call_sequence_links(tmp_path):
    if not (PKG / "libcmd_b200.so").exists():
        pytest.skip("libcmd_b200.so not built")
    exe = build_shim_program(tmp_path / "shim_calls")
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
