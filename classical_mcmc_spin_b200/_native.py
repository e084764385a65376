"""Loader and ctypes signatures of libcmd_b200.so (include/cmd.h, include/cmd_lattice.h).

There is no CPU fallback: if the library is missing or cannot be loaded the
import fails loudly, and every GPU entry point reports the CUDA error instead
of computing anything on the host.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcmd_b200.so"

CMD_OK = 0
CMD_ERR_INVALID_ARG = 1
CMD_ERR_UNSUPPORTED = 2
CMD_ERR_CUDA = 3
CMD_ERR_NONFINITE = 4
CMD_ERR_WATCHDOG = 5
CMD_ERR_OOM = 6
CMD_ERR_STATE = 7

CMD_RK4 = 0
CMD_DOPRI5_FIXED = 1
CMD_RK45 = 2
CMD_CASH_KARP_FIXED = 3
CMD_EULER = 4
CMD_MIDPOINT = 5
CMD_SSPRK53 = 6
CMD_RK78 = 7
CMD_BULIRSCH_STOER = 8

STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED", 3: "CUDA_ERROR", 4: "NONFINITE",
                5: "WATCHDOG_TIMEOUT", 6: "OOM", 7: "STATE"}

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_I32 = C.POINTER(C.c_int32)


class LatticeDesc(C.Structure):
    _fields_ = [("lattice_size", C.c_int64), ("spin_dim", C.c_int32), ("n_atoms", C.c_int32),
                ("max_bilinear", C.c_int32), ("reserved", C.c_int32),
                ("field", _D), ("onsite", _D), ("bilinear", _D), ("partners", _I64), ("counts", _I64),
                ("frames", _D), ("afm_signs", _D)]


class BatchDesc(C.Structure):
    _fields_ = [("B", C.c_int64), ("states", C.c_void_p), ("shared_initial", C.c_int32), ("method", C.c_int32),
                ("t1", C.c_void_p), ("t2", C.c_void_p), ("a1", C.c_void_p), ("a2", C.c_void_p),
                ("d1", C.c_void_p), ("d2", C.c_void_p), ("width", C.c_double), ("freq", C.c_double),
                ("T0", C.c_double), ("dt", C.c_double), ("n_steps", C.c_int64), ("save_interval", C.c_int64),
                ("obs", C.c_void_p), ("final_states", C.c_void_p), ("pulse4", C.c_void_p)]


class TrajSpec(C.Structure):
    _fields_ = [("lattice", C.c_void_p), ("state", C.c_void_p), ("T0", C.c_double), ("T1", C.c_double),
                ("dt", C.c_double), ("t1", C.c_double), ("t2", C.c_double), ("a1", C.c_double), ("a2", C.c_double),
                ("rows", C.c_void_p), ("max_rows", C.c_int64), ("final_state", C.c_void_p),
                ("stats", C.c_int64 * 4)]


class MixedDesc(C.Structure):
    """cmd_mixed_desc (include/cmd_mixed.h)."""
    _fields_ = [("n_su2", C.c_int64), ("n_su3", C.c_int64), ("spin_dim_su2", C.c_int32),
                ("spin_dim_su3", C.c_int32), ("n_atoms_su2", C.c_int32), ("n_atoms_su3", C.c_int32),
                ("max_bilinear_su2", C.c_int32), ("max_bilinear_su3", C.c_int32), ("max_mixed_su2", C.c_int32),
                ("max_mixed_su3", C.c_int32),
                ("field_su2", C.c_void_p), ("onsite_su2", C.c_void_p), ("bilinear_su2", C.c_void_p),
                ("partners_su2", C.c_void_p), ("counts_su2", C.c_void_p),
                ("field_su3", C.c_void_p), ("onsite_su3", C.c_void_p), ("bilinear_su3", C.c_void_p),
                ("partners_su3", C.c_void_p), ("counts_su3", C.c_void_p),
                ("mixed_su2", C.c_void_p), ("mixed_partners_su3", C.c_void_p), ("mixed_counts_su2", C.c_void_p),
                ("mixed_su3", C.c_void_p), ("mixed_partners_su2", C.c_void_p), ("mixed_counts_su3", C.c_void_p)]


class CmdError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_SIGS = {
    "cmd_create": (C.c_int, [C.POINTER(LatticeDesc), C.POINTER(C.c_void_p)]),
    "cmd_destroy": (C.c_int, [C.c_void_p]),
    "cmd_set_pulse": (C.c_int, [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
    "cmd_set_spins": (C.c_int, [C.c_void_p, _D, C.c_int64]),
    "cmd_get_spins": (C.c_int, [C.c_void_p, _D, C.c_int64]),
    "cmd_step": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int]),
    "cmd_integrate": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_int, _D, _D, _D,
                                C.c_int64, _I64]),
    "cmd_set_tolerances": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int64]),
    "cmd_energy": (C.c_int, [C.c_void_p, _D]),
    "cmd_normalize": (C.c_int, [C.c_void_p, C.c_double]),
    "cmd_magnetization": (C.c_int, [C.c_void_p, _D, _D]),
    "cmd_observables": (C.c_int, [C.c_void_p, _D]),
    "cmd_integrate_batched": (C.c_int, [C.c_void_p, _D, _D, C.c_int64, _D, _D, C.c_double, C.c_double,
                                        C.c_double, C.c_int64, C.c_int, _D, _D, C.c_int64, _I64]),
    "cmd_run_batch": (C.c_int, [C.c_void_p, C.POINTER(BatchDesc)]),
    "cmd_batch_rows": (C.c_int64, [C.c_int64, C.c_int64]),
    "cmd_run_batch_device": (C.c_int, [C.c_void_p, C.POINTER(BatchDesc), C.c_void_p, _I32]),
    "cmd_run_batch_device_noalloc": (C.c_int, [C.c_void_p, C.POINTER(BatchDesc), C.c_void_p, _I32]),
    "cmd_max_dsdt_no_drive": (C.c_int, [C.c_void_p, _D]),
    "cmd_nonlinear_spectrum": (C.c_int, [_D, _D, _D, C.c_int64, C.c_int64, C.c_int32, _D, _D]),
    "cmd_layout_info": (C.c_int, [C.c_void_p, _I64]),
    "cmd_plan_layout": (C.c_int, [C.POINTER(LatticeDesc), _I64]),
    "cmd_run_uneven": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_double, C.c_double, C.c_int64]),
    "cmd_adjoint_rk4": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cmd_variant_count": (C.c_int, []),
    "cmd_variant_info": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32, _I32]),
    "cmd_set_variant": (C.c_int, [C.c_void_p, C.c_int32]),
    "cmd_get_variant": (C.c_int, [C.c_void_p, _I32]),
    "cmd_autotune": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, _I32, _D]),
    "cmd_set_graphs": (C.c_int, [C.c_void_p, C.c_int32]),
    "cmd_rk45_variant_count": (C.c_int, []),
    "cmd_rk45_variant_info": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32, _I32]),
    "cmd_set_rk45_variant": (C.c_int, [C.c_void_p, C.c_int32]),
    "cmd_get_rk45_variant": (C.c_int, [C.c_void_p, _I32]),
    "cmd_autotune_rk45": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, _I32, _D]),
    "cmd_last_error": (C.c_char_p, []),
    "cmd_version": (C.c_char_p, []),
    # host lattice construction (cmd_lattice.h)
    "cmd_lattice_kitaev": (C.c_int, [_D, C.c_double, _D, _D, C.c_int32, C.c_int32, C.c_int32,
                                     C.POINTER(C.c_void_p)]),
    "cmd_lattice_pyrochlore_nk": (C.c_int, [_D, C.c_double, _D, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                            C.POINTER(C.c_void_p)]),
    "cmd_lattice_generic": (C.c_int, [C.c_int32, _I32, _D, C.c_int32, _D, _D, _D, _D, C.c_int32, C.c_int32,
                                      C.c_int32, C.POINTER(C.c_void_p)]),
    "cmd_lattice_sizes": (C.c_int, [C.c_void_p, _I64, _I32, _I32, _I32]),
    "cmd_lattice_export": (C.c_int, [C.c_void_p, _D, _D, _D, _I64, _I64, _D, _D]),
    "cmd_lattice_geometry": (C.c_int, [C.c_void_p, _D, _D]),
    "cmd_lattice_desc_of": (C.c_int, [C.c_void_p, C.POINTER(LatticeDesc)]),
    "cmd_lattice_rotate_pulse": (C.c_int, [C.c_void_p, _D, _D, _D]),
    "cmd_lattice_random_spins": (C.c_int, [C.c_int64, C.c_uint64, C.c_double, _D]),
    "cmd_mixed_create": (C.c_int, [C.POINTER(MixedDesc), C.POINTER(C.c_void_p)]),
    "cmd_mixed_destroy": (C.c_int, [C.c_void_p]),
    "cmd_mixed_set_pulse": (C.c_int, [C.c_void_p, C.c_int32, _D, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double]),
    "cmd_mixed_set_spins": (C.c_int, [C.c_void_p, _D, C.c_int64]),
    "cmd_mixed_get_spins": (C.c_int, [C.c_void_p, _D, C.c_int64]),
    "cmd_mixed_step": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int]),
    "cmd_mixed_integrate": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_int, _D, _D,
                                      C.c_int64, _I64]),
    "cmd_mixed_magnetization": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "cmd_mixed_normalize": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "cmd_mixed_dims": (C.c_int, [C.c_void_p, _I64]),
    "cmd_lattice_free": (None, [C.c_void_p]),
}

EXPORTED = tuple(_SIGS)

_lib = None


def lib() -> C.CDLL:
    """Load libcmd_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m classical_mcmc_spin_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code: int, where: str) -> None:
    if code != CMD_OK:
        raise CmdError(code, where, lib().cmd_last_error().decode(errors="replace"))


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_D) if a is not None else None


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_I64) if a is not None else None


def f64(x, n=None) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a
