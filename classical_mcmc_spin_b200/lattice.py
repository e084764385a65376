"""Host-side lattice of the LL MD path (mirror of the reference ``Lattice`` MD slice).

Builds the reference's bond tables through libcmd_b200.so (include/cmd_lattice.h;
reference include/classical_spin/lattice/lattice.h:601-855 and
src/core/unitcell_builders.cpp) and hands them to the GPU boundary exactly as
``Lattice::ensure_gpu_data_initialized`` does (lattice.h:5429-5497).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from . import gpu_api
from ._native import check, dptr, f64, iptr

KITAEV_KEYS = ("K", "Gamma", "Gammap", "J", "J2_A", "J2_B", "J3", "J_perp", "Ka", "Kb", "Kc")
KITAEV_DEFAULTS = dict(K=-1.0, Gamma=0.25, Gammap=-0.02, J=0.0, J2_A=0.0, J2_B=0.0, J3=0.0, J_perp=0.0,
                       Ka=0.0, Kb=0.0, Kc=0.0)
PYRO_KEYS = ("Jpm", "Jzz", "Jpmpm", "J2", "delta1", "delta2")
PYRO_DEFAULTS = dict(Jpm=0.0, Jzz=1.0, Jpmpm=0.0, J2=0.0, delta1=0.0, delta2=0.0)


class Lattice:
    """Bond tables + sublattice frames of one lattice (spin_dim = 3)."""

    def __init__(self, ptr: C.c_void_p):
        self._ptr = ptr
        N = C.c_int64()
        na = C.c_int32()
        z = C.c_int32()
        dims = (C.c_int32 * 3)()
        check(nat.lib().cmd_lattice_sizes(ptr, C.byref(N), C.byref(na), C.byref(z), dims), "cmd_lattice_sizes")
        self.lattice_size = int(N.value)
        self.N_atoms = int(na.value)
        self.num_bi = int(z.value)
        self.dims = tuple(int(d) for d in dims)
        self.spin_dim = 3
        self.spins = np.zeros((self.lattice_size, 3))

    # ---- builders -------------------------------------------------------
    @classmethod
    def kitaev(cls, d1: int, d2: int, d3: int = 1, h: float = 0.0, field_direction=(0.0, 1.0, 0.0),
               g_factor=(1.0, 1.0, 1.0), **params) -> "Lattice":
        """build_kitaev_honeycomb (unitcell_builders.cpp:178-283); unknown keys -> KeyError."""
        p = dict(KITAEV_DEFAULTS)
        for k, v in params.items():
            if k not in p:
                raise KeyError(f"unknown Kitaev parameter {k!r}")
            p[k] = float(v)
        kp = f64([p[k] for k in KITAEV_KEYS])
        out = C.c_void_p()
        check(nat.lib().cmd_lattice_kitaev(dptr(kp), float(h), dptr(f64(field_direction, 3)),
                                           dptr(f64(g_factor, 3)), d1, d2, d3, C.byref(out)), "kitaev")
        return cls(out)

    @classmethod
    def pyrochlore_non_kramer(cls, d1: int, d2: int, d3: int, h: float = 0.0, field_direction=(0.0, 1.0, 0.0),
                              cubic: bool = False, **params) -> "Lattice":
        """build_pyrochlore_non_kramer (unitcell_builders.cpp:370-471)."""
        p = dict(PYRO_DEFAULTS)
        for k, v in params.items():
            if k not in p:
                raise KeyError(f"unknown pyrochlore parameter {k!r}")
            p[k] = float(v)
        pp = f64([p[k] for k in PYRO_KEYS])
        out = C.c_void_p()
        check(nat.lib().cmd_lattice_pyrochlore_nk(dptr(pp), float(h), dptr(f64(field_direction, 3)), d1, d2, d3,
                                                  int(bool(cubic)), C.byref(out)), "pyrochlore_non_kramer")
        return cls(out)

    def __del__(self):
        try:
            if self._ptr:
                nat.lib().cmd_lattice_free(self._ptr)
                self._ptr = None
        except Exception:
            pass

    # ---- tables ----------------------------------------------------------
    def export(self) -> dict:
        N, z, na = self.lattice_size, self.num_bi, self.N_atoms
        out = dict(field=np.zeros(3 * N), onsite=np.zeros(9 * N), bilinear=np.zeros(9 * N * z),
                   partners=np.zeros(N * z, np.int64), counts=np.zeros(N, np.int64), frames=np.zeros(9 * na),
                   afm=np.zeros(na), max_bilinear=z)
        check(nat.lib().cmd_lattice_export(self._ptr, dptr(out["field"]), dptr(out["onsite"]),
                                           dptr(out["bilinear"]), iptr(out["partners"]), iptr(out["counts"]),
                                           dptr(out["frames"]), dptr(out["afm"])), "cmd_lattice_export")
        return out

    @property
    def sublattice_frames(self) -> np.ndarray:
        return self.export()["frames"].reshape(self.N_atoms, 3, 3)

    @property
    def afm_sublattice_signs(self) -> np.ndarray:
        return self.export()["afm"]

    def rotate_pulse(self, field_in1, field_in2) -> np.ndarray:
        """Lattice::set_pulse's R*B rotation (lattice_md.cpp:214-217); returns [2*N_atoms*3]."""
        fd = np.zeros(6 * self.N_atoms)
        check(nat.lib().cmd_lattice_rotate_pulse(self._ptr, dptr(f64(field_in1, 3 * self.N_atoms)),
                                                 dptr(f64(field_in2, 3 * self.N_atoms)), dptr(fd)),
              "cmd_lattice_rotate_pulse")
        return fd

    def to_gpu(self) -> gpu_api.GPULatticeDataHandle:
        """ensure_gpu_data_initialized (lattice.h:5429-5497) -> device handle."""
        d = nat.LatticeDesc()
        check(nat.lib().cmd_lattice_desc_of(self._ptr, C.byref(d)), "cmd_lattice_desc_of")
        out = C.c_void_p()
        check(nat.lib().cmd_create(C.byref(d), C.byref(out)), "cmd_create")
        return gpu_api.GPULatticeDataHandle(out.value, self.lattice_size, self.N_atoms)

    # ---- spin configuration I/O (lattice.h:4687-4739) ---------------------
    def save_spin_config(self, filename: str) -> None:
        with open(filename, "w") as f:
            for s in self.spins:
                f.write(" ".join(f"{v:.16e}" for v in s) + "\n")

    def load_spin_config(self, filename: str) -> None:
        rows = []
        with open(filename) as f:
            for line in f:
                if len(rows) >= self.lattice_size:
                    break
                parts = line.split()
                if len(parts) < 3:
                    raise ValueError(f"incomplete spin data at line {len(rows)}")
                rows.append([float(x) for x in parts[:3]])
        if len(rows) != self.lattice_size:
            raise ValueError(f"file contained {len(rows)} spins, expected {self.lattice_size}")
        self.spins = np.array(rows)
