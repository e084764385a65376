"""Python mirror of the reference's host GPU API for mixed SU(2)/SU(3) lattices.

Same function names, argument meaning and result layout as ``namespace mixed_gpu``
in include/classical_spin/gpu/mixed_lattice_gpu_api.h (ze-bang/Classical_MCMC_Spin);
the work happens in libcmd_b200.so (include/cmd_mixed.h).  Differences, by design:
failures raise ``CmdError`` (the reference returns silently on a NULL handle or a
missing state), an unknown method raises instead of falling back to ssprk53, and
``integrate_mixed_gpu`` returns the times with the trajectory.

``synthetic_mixed_lattice`` builds seeded lattices in the reference's flattened form
(the arrays MixedLattice uploads) for tests and benchmarks.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import check, dptr, f64
from .gpu_api import METHODS


def _method(method: str | int) -> int:
    if isinstance(method, int):
        return method
    if method not in METHODS or method == "rk45":
        raise ValueError(f"unknown mixed-lattice method {method!r}; supported: "
                         f"{sorted(m for m in METHODS if m != 'rk45')}")
    return METHODS[method]


def _i64(a, n):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int64).ravel())
    if a.size != n:
        raise ValueError(f"expected {n} indices, got {a.size}")
    return a


class GPUMixedLatticeDataHandle:
    """Opaque handle (mixed_lattice_gpu_api.h:32); owns a cmd_mixed."""

    def __init__(self, ptr: int, n2: int, n3: int, na2: int, na3: int):
        self.ptr = C.c_void_p(ptr)
        self.n2, self.n3, self.na2, self.na3 = n2, n3, na2, na3
        self.V = 3 * n2 + 8 * n3

    def close(self):
        if self.ptr:
            nat.lib().cmd_mixed_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def create_gpu_mixed_lattice_data(lattice_size_SU2, spin_dim_SU2, N_atoms_SU2, lattice_size_SU3, spin_dim_SU3,
                                  N_atoms_SU3, max_bilinear_SU2, max_bilinear_SU3, max_mixed_bilinear,
                                  max_mixed_bilinear_SU3, flat_field_SU2, flat_onsite_SU2, flat_bilinear_SU2,
                                  flat_partners_SU2, num_bilinear_per_site_SU2, flat_field_SU3, flat_onsite_SU3,
                                  flat_bilinear_SU3, flat_partners_SU3, num_bilinear_per_site_SU3,
                                  flat_mixed_bilinear, flat_mixed_partners_SU2, flat_mixed_partners_SU3,
                                  num_mixed_per_site_SU2, flat_mixed_bilinear_SU3,
                                  flat_mixed_partners_SU2_from_SU3,
                                  num_mixed_per_site_SU3) -> GPUMixedLatticeDataHandle:
    """create_gpu_mixed_lattice_data (mixed_lattice_gpu_api.h:66-90).  flat_mixed_partners_SU2 is unused,
    as in the reference."""
    if spin_dim_SU2 != 3 or spin_dim_SU3 != 8:
        raise ValueError("spin dimensions must be 3 (SU(2)) and 8 (SU(3))")
    n2, n3 = int(lattice_size_SU2), int(lattice_size_SU3)
    z2, z3, zm2, zm3 = int(max_bilinear_SU2), int(max_bilinear_SU3), int(max_mixed_bilinear), \
        int(max_mixed_bilinear_SU3)
    keep = dict(f2=f64(flat_field_SU2, 3 * n2), o2=f64(flat_onsite_SU2, 9 * n2),
                j2=f64(flat_bilinear_SU2, 9 * n2 * z2), p2=_i64(flat_partners_SU2, n2 * z2),
                c2=_i64(num_bilinear_per_site_SU2, n2),
                f3=f64(flat_field_SU3, 8 * n3), o3=f64(flat_onsite_SU3, 64 * n3),
                j3=f64(flat_bilinear_SU3, 64 * n3 * z3), p3=_i64(flat_partners_SU3, n3 * z3),
                c3=_i64(num_bilinear_per_site_SU3, n3),
                m2=f64(flat_mixed_bilinear, 24 * n2 * zm2), mp2=_i64(flat_mixed_partners_SU3, n2 * zm2),
                mc2=_i64(num_mixed_per_site_SU2, n2),
                m3=f64(flat_mixed_bilinear_SU3, 24 * n3 * zm3), mp3=_i64(flat_mixed_partners_SU2_from_SU3, n3 * zm3),
                mc3=_i64(num_mixed_per_site_SU3, n3))
    d = nat.MixedDesc()
    d.n_su2, d.n_su3 = n2, n3
    d.spin_dim_su2, d.spin_dim_su3 = 3, 8
    d.n_atoms_su2, d.n_atoms_su3 = int(N_atoms_SU2), int(N_atoms_SU3)
    d.max_bilinear_su2, d.max_bilinear_su3, d.max_mixed_su2, d.max_mixed_su3 = z2, z3, zm2, zm3
    ptr = lambda k: keep[k].ctypes.data if keep[k].size else None
    d.field_su2, d.onsite_su2, d.bilinear_su2, d.partners_su2, d.counts_su2 = (ptr(k) for k in
                                                                               ("f2", "o2", "j2", "p2", "c2"))
    d.field_su3, d.onsite_su3, d.bilinear_su3, d.partners_su3, d.counts_su3 = (ptr(k) for k in
                                                                               ("f3", "o3", "j3", "p3", "c3"))
    d.mixed_su2, d.mixed_partners_su3, d.mixed_counts_su2 = ptr("m2"), ptr("mp2"), ptr("mc2")
    d.mixed_su3, d.mixed_partners_su2, d.mixed_counts_su3 = ptr("m3"), ptr("mp3"), ptr("mc3")
    out = C.c_void_p()
    check(nat.lib().cmd_mixed_create(C.byref(d), C.byref(out)), "create_gpu_mixed_lattice_data")
    return GPUMixedLatticeDataHandle(out.value, n2, n3, int(N_atoms_SU2), int(N_atoms_SU3))


def destroy_gpu_mixed_lattice_data(handle: GPUMixedLatticeDataHandle) -> None:
    handle.close()


def _set_pulse(handle, sub, flat_field_drive, pulse_amp, pulse_width, pulse_freq, t_pulse_1, t_pulse_2):
    n = 2 * (handle.na2 * 3 if sub == 2 else handle.na3 * 8)
    fd = f64(flat_field_drive, n)
    check(nat.lib().cmd_mixed_set_pulse(handle.ptr, sub, dptr(fd), float(pulse_amp), float(pulse_width),
                                        float(pulse_freq), float(t_pulse_1), float(t_pulse_2)), "set_gpu_pulse")


def set_gpu_pulse_SU2(handle, flat_field_drive, pulse_amp, pulse_width, pulse_freq, t_pulse_1, t_pulse_2):
    """set_gpu_pulse_SU2 (:97-104): flat_field_drive [2][N_atoms_SU2][3]."""
    _set_pulse(handle, 2, flat_field_drive, pulse_amp, pulse_width, pulse_freq, t_pulse_1, t_pulse_2)


def set_gpu_pulse_SU3(handle, flat_field_drive, pulse_amp, pulse_width, pulse_freq, t_pulse_1, t_pulse_2):
    """set_gpu_pulse_SU3 (:107-114): flat_field_drive [2][N_atoms_SU3][8]."""
    _set_pulse(handle, 3, flat_field_drive, pulse_amp, pulse_width, pulse_freq, t_pulse_1, t_pulse_2)


def set_gpu_mixed_spins(handle, flat_spins):
    s = f64(flat_spins, handle.V)
    check(nat.lib().cmd_mixed_set_spins(handle.ptr, dptr(s), s.size), "set_gpu_mixed_spins")


def get_gpu_mixed_spins(handle) -> np.ndarray:
    s = np.zeros(handle.V)
    check(nat.lib().cmd_mixed_get_spins(handle.ptr, dptr(s), s.size), "get_gpu_mixed_spins")
    return s


def step_mixed_gpu(handle, t, dt, method="ssprk53"):
    check(nat.lib().cmd_mixed_step(handle.ptr, float(t), float(dt), _method(method)), "step_mixed_gpu")


def integrate_mixed_gpu(handle, T_start, T_end, dt, save_interval, method="ssprk53"):
    """integrate_mixed_gpu (:154-162): ``(trajectory, times)`` with the reference's (t, state) pairs."""
    rows = C.c_int64()
    m = _method(method)
    L = nat.lib()
    rc = L.cmd_mixed_integrate(handle.ptr, float(T_start), float(T_end), float(dt), int(save_interval), m, None,
                               None, 0, C.byref(rows))
    if rc not in (nat.CMD_OK, nat.CMD_ERR_INVALID_ARG) or rows.value <= 0:
        check(rc, "integrate_mixed_gpu")
    n = rows.value
    times = np.zeros(n)
    states = np.zeros((n, handle.V))
    check(L.cmd_mixed_integrate(handle.ptr, float(T_start), float(T_end), float(dt), int(save_interval), m,
                                dptr(times), dptr(states), n, C.byref(rows)), "integrate_mixed_gpu")
    return [(float(times[r]), states[r]) for r in range(n)], times


def compute_magnetization_mixed_gpu(handle):
    """compute_magnetization_mixed_gpu (:188-194): (M_SU2, M_staggered_SU2, M_SU3, M_staggered_SU3)."""
    out = [np.zeros(3), np.zeros(3), np.zeros(8), np.zeros(8)]
    check(nat.lib().cmd_mixed_magnetization(handle.ptr, *(dptr(o) for o in out)), "compute_magnetization_mixed_gpu")
    return tuple(out)


def normalize_spins_mixed_gpu(handle, spin_length_SU2, spin_length_SU3):
    check(nat.lib().cmd_mixed_normalize(handle.ptr, float(spin_length_SU2), float(spin_length_SU3)),
          "normalize_spins_mixed_gpu")


def get_mixed_lattice_dims(handle):
    """get_mixed_lattice_dims (:208-212): (lattice_size_SU2, 3, N_atoms_SU2, lattice_size_SU3, 8, N_atoms_SU3)."""
    dims = np.zeros(6, dtype=np.int64)
    check(nat.lib().cmd_mixed_dims(handle.ptr, dims.ctypes.data_as(C.POINTER(C.c_int64))), "get_mixed_lattice_dims")
    return tuple(int(x) for x in dims)


def create_from(arr: dict) -> GPUMixedLatticeDataHandle:
    """create_gpu_mixed_lattice_data from a ``synthetic_mixed_lattice`` dictionary."""
    return create_gpu_mixed_lattice_data(
        arr["n2"], 3, arr["na2"], arr["n3"], 8, arr["na3"], arr["z2"], arr["z3"], arr["zm2"], arr["zm3"],
        arr["field2"], arr["onsite2"], arr["bil2"], arr["part2"], arr["cnt2"],
        arr["field3"], arr["onsite3"], arr["bil3"], arr["part3"], arr["cnt3"],
        arr["mix2"], np.zeros(0), arr["mpart2"], arr["mcnt2"], arr["mix3"], arr["mpart3"], arr["mcnt3"])


def synthetic_mixed_lattice(L=(6, 6, 6), na2=4, na3=4, seed=0, coupling=0.3, field=0.1, onsite=0.05) -> dict:
    """A seeded mixed lattice in the reference's flattened form, shaped like TmFeO3 (4 SU(2) and 4 SU(3)
    atoms per cell of an L1 x L2 x L3 periodic cubic lattice).

    SU(2) atom a couples to the same atom in the six neighbouring cells (3x3 J_{a,d} forward, its transpose
    backward); SU(3) atom b to the same atom in the two x-neighbours (8x8 K_b and transpose); SU(3) atom b of
    cell c to the four SU(2) atoms of cell c and of cell c + e_{b mod 3} (8x3 M from the SU(3) side, the 3x8
    transpose from the SU(2) side).  Fields and symmetric on-site matrices are random and small.  Every bond
    appears at both ends with transposed couplings, so the dynamics conserves the energy."""
    rng = np.random.default_rng(seed)
    L1, L2, L3 = L
    nc = L1 * L2 * L3
    n2, n3 = nc * na2, nc * na3
    E = np.eye(3, dtype=int)

    def cell(x, y, z):
        return ((x % L1) * L2 + (y % L2)) * L3 + (z % L3)

    def coords(c):
        return c // (L2 * L3), (c // L3) % L2, c % L3

    J = coupling * rng.normal(size=(na2, 3, 3, 3))            # [atom][direction] 3x3
    K = coupling * rng.normal(size=(na3, 8, 8)) / 2
    M = coupling * rng.normal(size=(na3, 2, na2, 8, 3)) / 2    # [SU3 atom][cell offset 0 / 1][SU2 atom] 8x3
    z2, z3, zm2, zm3 = 6, 2, 2 * na3, 2 * na2
    part2 = np.zeros((n2, z2), np.int64)
    bil2 = np.zeros((n2, z2, 3, 3))
    part3 = np.zeros((n3, z3), np.int64)
    bil3 = np.zeros((n3, z3, 8, 8))
    mpart3 = np.zeros((n3, zm3), np.int64)
    mix3 = np.zeros((n3, zm3, 8, 3))
    mlist2 = [[] for _ in range(n2)]
    for c in range(nc):
        x, y, z = coords(c)
        for a in range(na2):
            i = c * na2 + a
            for d in range(3):
                part2[i, 2 * d] = cell(x + E[d, 0], y + E[d, 1], z + E[d, 2]) * na2 + a
                bil2[i, 2 * d] = J[a, d]
                part2[i, 2 * d + 1] = cell(x - E[d, 0], y - E[d, 1], z - E[d, 2]) * na2 + a
                bil2[i, 2 * d + 1] = J[a, d].T
        for b in range(na3):
            s = c * na3 + b
            part3[s, 0], bil3[s, 0] = cell(x + 1, y, z) * na3 + b, K[b]
            part3[s, 1], bil3[s, 1] = cell(x - 1, y, z) * na3 + b, K[b].T
            d = b % 3
            for o, cc in enumerate((c, cell(x + E[d, 0], y + E[d, 1], z + E[d, 2]))):
                for a in range(na2):
                    k = o * na2 + a
                    p = cc * na2 + a
                    mpart3[s, k], mix3[s, k] = p, M[b, o, a]
                    mlist2[p].append((s, M[b, o, a].T))
    mpart2 = np.zeros((n2, zm2), np.int64)
    mix2 = np.zeros((n2, zm2, 3, 8))
    for p, lst in enumerate(mlist2):
        assert len(lst) == zm2
        for k, (s, m) in enumerate(lst):
            mpart2[p, k], mix2[p, k] = s, m
    A2 = onsite * rng.normal(size=(na2, 3, 3))
    A3 = onsite * rng.normal(size=(na3, 8, 8))
    A2 = (A2 + A2.transpose(0, 2, 1)) / 2
    A3 = (A3 + A3.transpose(0, 2, 1)) / 2
    B2 = field * rng.normal(size=(na2, 3))
    B3 = field * rng.normal(size=(na3, 8))
    return dict(n2=n2, n3=n3, na2=na2, na3=na3, z2=z2, z3=z3, zm2=zm2, zm3=zm3,
                field2=np.tile(B2, (nc, 1)).ravel(), onsite2=np.tile(A2, (nc, 1, 1)).ravel(),
                bil2=bil2.ravel(), part2=part2.ravel(), cnt2=np.full(n2, z2, np.int64),
                field3=np.tile(B3, (nc, 1)).ravel(), onsite3=np.tile(A3, (nc, 1, 1)).ravel(),
                bil3=bil3.ravel(), part3=part3.ravel(), cnt3=np.full(n3, z3, np.int64),
                mix2=mix2.ravel(), mpart2=mpart2.ravel(), mcnt2=np.full(n2, zm2, np.int64),
                mix3=mix3.ravel(), mpart3=mpart3.ravel(), mcnt3=np.full(n3, zm3, np.int64))


def random_mixed_state(arr: dict, seed: int) -> np.ndarray:
    """Unit SU(2) spins and unit 8-vectors for the SU(3) sites, seeded."""
    rng = np.random.default_rng(seed)
    s2 = rng.normal(size=(arr["n2"], 3))
    s3 = rng.normal(size=(arr["n3"], 8))
    s2 /= np.linalg.norm(s2, axis=1, keepdims=True)
    s3 /= np.linalg.norm(s3, axis=1, keepdims=True)
    return np.concatenate([s2.ravel(), s3.ravel()])
