"""The C-ABI library loads and exports every function include/*.h declares (no GPU needed)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(cmd_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(native):
    names = declared_functions()
    assert len(names) >= 25, names
    lib = C.CDLL(str(native.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the whole ABI too
    assert set(names) <= set(native.EXPORTED), set(names) - set(native.EXPORTED)


def test_library_is_sm100a_and_independent_of_the_oracle(native):
    out = subprocess.run(["nm", "-D", "--defined-only", str(native.LIB_PATH)], capture_output=True, text=True)
    assert "ora_" not in out.stdout and "refgpu_" not in out.stdout
    ldd = subprocess.run(["ldd", str(native.LIB_PATH)], capture_output=True, text=True).stdout
    assert "ll_oracle" not in ldd and "libref" not in ldd


def test_status_and_version_without_gpu(native):
    L = native.lib()
    assert b"sm_100a" in L.cmd_version()
    assert L.cmd_batch_rows(10, 5) == 3 and L.cmd_batch_rows(11, 5) == 4 and L.cmd_batch_rows(0, 1) == 1
    assert L.cmd_create(None, None) == native.CMD_ERR_INVALID_ARG
    assert b"NULL" in L.cmd_last_error()


def test_no_cpu_fallback_without_gpu(native):
    """Without a CUDA device cmd_create fails loudly instead of computing on the host."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200._native import CmdError
    with pytest.raises(CmdError) as e:
        Lattice.kitaev(4, 4, 1).to_gpu()
    assert e.value.code == native.CMD_ERR_CUDA
