"""Python mirror of the reference's host GPU API for the LL MD path.

Same function names, argument meaning and result layout as
``namespace gpu`` in include/classical_spin/gpu/lattice_gpu_api.h
(ze-bang/Classical_MCMC_Spin); the work happens in libcmd_b200.so on the GPU.
Differences, by design: failures raise ``CmdError`` (the reference silently
returns on a NULL handle or missing state, lattice_gpu.cu:660-723), the
energy is implemented (the reference throws, lattice_gpu.cu:298-303), and an
unknown method raises instead of falling back to ssprk53.  The default method
is the reference's, "ssprk53" (lattice_gpu_api.h:124, 139).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from ._native import check, dptr, f64, iptr

# The reference GPU method names (integrator.cuh:91-452) plus "rk45", the
# controlled Dormand-Prince of the reference CPU path.
METHODS = {"rk4": nat.CMD_RK4, "dopri5": nat.CMD_DOPRI5_FIXED, "rk54": nat.CMD_DOPRI5_FIXED,
           "rkf54": nat.CMD_DOPRI5_FIXED, "rk45": nat.CMD_RK45,
           "rk5": nat.CMD_CASH_KARP_FIXED, "rkck54": nat.CMD_CASH_KARP_FIXED,
           "euler": nat.CMD_EULER, "rk2": nat.CMD_MIDPOINT, "midpoint": nat.CMD_MIDPOINT,
           "ssprk53": nat.CMD_SSPRK53, "rk78": nat.CMD_RK78, "rkf78": nat.CMD_RK78,
           "bulirsch_stoer": nat.CMD_BULIRSCH_STOER, "bs": nat.CMD_BULIRSCH_STOER}


def _method(method: str | int) -> int:
    if isinstance(method, int):
        return method
    if method not in METHODS:
        raise ValueError(f"unknown integration method {method!r}; supported: {sorted(METHODS)}")
    return METHODS[method]


class GPULatticeDataHandle:
    """Opaque handle (lattice_gpu_api.h:30); owns a cmd_handle."""

    def __init__(self, ptr: int, N: int, n_atoms: int):
        self.ptr = C.c_void_p(ptr)
        self.N = N
        self.n_atoms = n_atoms

    def close(self):
        if self.ptr:
            nat.lib().cmd_destroy(self.ptr)
            self.ptr = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def variants(self) -> list:
        """[(index, name, fits this lattice)] of the resident-kernel variants."""
        L = nat.lib()
        out = []
        for i in range(L.cmd_variant_count()):
            buf = C.create_string_buffer(128)
            fits = C.c_int32()
            check(L.cmd_variant_info(self.ptr, i, buf, 128, C.byref(fits)), "cmd_variant_info")
            out.append((i, buf.value.decode(), bool(fits.value)))
        return out

    def set_variant(self, idx: int) -> None:
        check(nat.lib().cmd_set_variant(self.ptr, int(idx)), "cmd_set_variant")

    def get_variant(self) -> int:
        v = C.c_int32()
        check(nat.lib().cmd_get_variant(self.ptr, C.byref(v)), "cmd_get_variant")
        return v.value

    def autotune(self, B: int, n_steps: int) -> tuple:
        """Times every fitting variant; pins and returns (best index, ms per variant)."""
        n = nat.lib().cmd_variant_count()
        ms = np.zeros(n)
        best = C.c_int32()
        check(nat.lib().cmd_autotune(self.ptr, int(B), int(n_steps), C.byref(best), dptr(ms)), "cmd_autotune")
        return best.value, ms

    def set_graphs(self, enable: bool) -> None:
        """CUDA graphs (default on): streamed RK4 replays captured chunks of stage launches; batched resident
        runs and uneven batches run each call's launches as one captured graph.  Off: direct launches."""
        check(nat.lib().cmd_set_graphs(self.ptr, int(bool(enable))), "cmd_set_graphs")

    def rk45_variants(self) -> list:
        """[(index, name, holds this lattice)] of the on-chip controlled Dormand-Prince tilings."""
        L = nat.lib()
        out = []
        for i in range(L.cmd_rk45_variant_count()):
            buf = C.create_string_buffer(128)
            fits = C.c_int32()
            check(L.cmd_rk45_variant_info(self.ptr, i, buf, 128, C.byref(fits)), "cmd_rk45_variant_info")
            out.append((i, buf.value.decode(), bool(fits.value)))
        return out

    def set_rk45_variant(self, idx: int) -> None:
        """Pins an RK45 tiling (-1: default choice, -2: the global-memory kernel)."""
        check(nat.lib().cmd_set_rk45_variant(self.ptr, int(idx)), "cmd_set_rk45_variant")

    def get_rk45_variant(self) -> int:
        v = C.c_int32()
        check(nat.lib().cmd_get_rk45_variant(self.ptr, C.byref(v)), "cmd_get_rk45_variant")
        return v.value

    def autotune_rk45(self, B: int, n_steps: int) -> tuple:
        """Times every RK45 tiling that holds the lattice; pins and returns (best index, ms per tiling)."""
        n = nat.lib().cmd_rk45_variant_count()
        ms = np.zeros(n)
        best = C.c_int32()
        check(nat.lib().cmd_autotune_rk45(self.ptr, int(B), int(n_steps), C.byref(best), dptr(ms)),
              "cmd_autotune_rk45")
        return best.value, ms

    def layout_info(self) -> dict:
        info = np.zeros(6, np.int64)
        check(nat.lib().cmd_layout_info(self.ptr, iptr(info)), "cmd_layout_info")
        return dict(sites_per_group=int(info[0]), groups=int(info[1]), bonds_per_site=int(info[2]),
                    threads=int(info[3]), groups_per_thread=int(info[4]), smem_bytes=int(info[5]))


def _desc(N, n_atoms, max_bilinear, field_, onsite, bilinear, partners, counts, frames=None, afm=None):
    keep = dict(field=f64(field_, 3 * N), onsite=f64(onsite, 9 * N), bilinear=f64(bilinear, 9 * N * max_bilinear),
                partners=np.ascontiguousarray(partners, dtype=np.int64),
                counts=np.ascontiguousarray(counts, dtype=np.int64),
                frames=None if frames is None else f64(frames, 9 * n_atoms),
                afm=None if afm is None else f64(afm, n_atoms))
    d = nat.LatticeDesc()
    d.lattice_size = N
    d.spin_dim = 3
    d.n_atoms = n_atoms
    d.max_bilinear = max_bilinear
    d.field = dptr(keep["field"])
    d.onsite = dptr(keep["onsite"])
    d.bilinear = dptr(keep["bilinear"])
    d.partners = iptr(keep["partners"])
    d.counts = iptr(keep["counts"])
    d.frames = dptr(keep["frames"]) if keep["frames"] is not None else None
    d.afm_signs = dptr(keep["afm"]) if keep["afm"] is not None else None
    return d, keep


def create_gpu_lattice_data(lattice_size, spin_dim, N_atoms, max_bilinear, flat_field, flat_onsite,
                            flat_bilinear, flat_partners, num_bilinear_per_site, sublattice_frames=None,
                            afm_signs=None) -> GPULatticeDataHandle:
    """create_gpu_lattice_data (lattice_gpu_api.h:47-57)."""
    if spin_dim != 3:
        raise ValueError("only spin_dim = 3 is supported")
    d, _keep = _desc(int(lattice_size), int(N_atoms), int(max_bilinear), flat_field, flat_onsite, flat_bilinear,
                     flat_partners, num_bilinear_per_site, sublattice_frames, afm_signs)
    out = C.c_void_p()
    check(nat.lib().cmd_create(C.byref(d), C.byref(out)), "create_gpu_lattice_data")
    return GPULatticeDataHandle(out.value, int(lattice_size), int(N_atoms))


def destroy_gpu_lattice_data(handle: GPULatticeDataHandle) -> None:
    handle.close()


def set_gpu_pulse(handle, flat_field_drive, pulse_amp, pulse_width, pulse_freq, t_pulse_1, t_pulse_2):
    fd = f64(flat_field_drive, 6 * handle.n_atoms)
    check(nat.lib().cmd_set_pulse(handle.ptr, dptr(fd), float(pulse_amp), float(pulse_width), float(pulse_freq),
                                  float(t_pulse_1), float(t_pulse_2)), "set_gpu_pulse")


def set_gpu_spins(handle, flat_spins):
    s = f64(flat_spins, 3 * handle.N)
    check(nat.lib().cmd_set_spins(handle.ptr, dptr(s), s.size), "set_gpu_spins")


def get_gpu_spins(handle) -> np.ndarray:
    s = np.zeros(3 * handle.N)
    check(nat.lib().cmd_get_spins(handle.ptr, dptr(s), s.size), "get_gpu_spins")
    return s


def step_gpu(handle, t, dt, method="ssprk53"):
    check(nat.lib().cmd_step(handle.ptr, float(t), float(dt), _method(method)), "step_gpu")


def set_tolerances(handle, abs_tol, rel_tol, max_steps=0):
    check(nat.lib().cmd_set_tolerances(handle.ptr, float(abs_tol), float(rel_tol), int(max_steps)),
          "set_tolerances")


def integrate_gpu(handle, T_start, T_end, dt, save_interval, method="ssprk53", with_states=True, max_rows=None):
    """integrate_gpu (lattice_gpu_api.h:117-125).

    Returns ``(trajectory, obs, times)``: ``trajectory`` is the reference's list
    of ``(t, state)`` pairs (empty when ``with_states`` is False), ``obs`` the
    per-row observables {M_af, M_local, M_global, E/N} computed on the device.
    Methods: the reference GPU's fixed-step ones ("ssprk53", the default,
    "rk4", "dopri5" / "rk54", "rk5" / "rkck54", "euler", "rk2" / "midpoint",
    "rk78" / "rkf78", "bs" / "bulirsch_stoer") and "rk45" (controlled
    Dormand-Prince with the CPU path's step control; ``dt`` is the initial
    step, one row per accepted step).
    """
    rows = C.c_int64()
    m = _method(method)
    L = nat.lib()
    n = int(max_rows) if max_rows else 0
    if n <= 0:
        rc = L.cmd_integrate(handle.ptr, float(T_start), float(T_end), float(dt), int(save_interval), m,
                             None, None, None, 0, C.byref(rows))
        if rc not in (nat.CMD_OK, nat.CMD_ERR_INVALID_ARG) or rows.value <= 0:
            check(rc, "integrate_gpu")
        n = rows.value
    times = np.zeros(n)
    obs = np.zeros((n, 10))
    states = np.zeros((n, 3 * handle.N)) if with_states else None
    # A controlled run that needs more than max_rows rows has advanced the state
    # already; the error carries the row count it needed.
    check(L.cmd_integrate(handle.ptr, float(T_start), float(T_end), float(dt), int(save_interval), m,
                          dptr(times), dptr(obs), dptr(states), n, C.byref(rows)), "integrate_gpu")
    n = rows.value
    times, obs = times[:n], obs[:n]
    traj = [(float(times[r]), states[r]) for r in range(n)] if with_states else []
    return traj, obs, times


def compute_energy_gpu(handle) -> float:
    e = C.c_double()
    check(nat.lib().cmd_energy(handle.ptr, C.byref(e)), "compute_energy_gpu")
    return e.value


def normalize_spins_gpu(handle, spin_length):
    check(nat.lib().cmd_normalize(handle.ptr, float(spin_length)), "normalize_spins_gpu")


def compute_magnetization_gpu(handle):
    ml = np.zeros(3)
    ms = np.zeros(3)
    check(nat.lib().cmd_magnetization(handle.ptr, dptr(ml), dptr(ms)), "compute_magnetization_gpu")
    return ml, ms


def observables_gpu(handle) -> np.ndarray:
    row = np.zeros(10)
    check(nat.lib().cmd_observables(handle.ptr, dptr(row)), "observables_gpu")
    return row


@dataclass
class BatchedMagResult:
    """BatchedMagResult (lattice_gpu_api.h:171-177)."""
    B: int
    spin_dim: int
    n_time_points: int
    times: np.ndarray = field(repr=False)
    mag_data: np.ndarray = field(repr=False)   # [n_time_points][B][3][spin_dim]


def integrate_gpu_batched(handle, flat_initial_state, tau2_values, afm_signs, sublattice_frames, T_start, T_end,
                          dt, save_interval=1, method="rk4") -> BatchedMagResult:
    """integrate_gpu_batched (lattice_gpu_api.h:205-214)."""
    init = f64(flat_initial_state, 3 * handle.N)
    tau2 = f64(tau2_values)
    B = tau2.size
    afm = None if afm_signs is None else f64(afm_signs, handle.n_atoms)
    fr = None if sublattice_frames is None else f64(sublattice_frames, 9 * handle.n_atoms)
    rows = C.c_int64()
    m = _method(method)
    rc = nat.lib().cmd_integrate_batched(handle.ptr, dptr(init), dptr(tau2), B, dptr(afm), dptr(fr),
                                         float(T_start), float(T_end), float(dt), int(save_interval), m, None,
                                         None, 0, C.byref(rows))
    if rc not in (nat.CMD_OK, nat.CMD_ERR_INVALID_ARG) or rows.value <= 0:
        check(rc, "integrate_gpu_batched")
    n = rows.value
    times = np.zeros(n)
    mags = np.zeros((n, B, 3, 3))
    check(nat.lib().cmd_integrate_batched(handle.ptr, dptr(init), dptr(tau2), B, dptr(afm), dptr(fr),
                                          float(T_start), float(T_end), float(dt), int(save_interval), m,
                                          dptr(times), dptr(mags), n, C.byref(rows)), "integrate_gpu_batched")
    return BatchedMagResult(B=B, spin_dim=3, n_time_points=n, times=times, mag_data=mags)


def run_batch(handle, states, n_steps, dt, T0=0.0, save_interval=1, t1=None, t2=None, a1=None, a2=None,
              d1=None, d2=None, width=1.0, freq=0.0, shared_initial=False, want_final=True):
    """Generalised batch (cmd_run_batch): per-trajectory pulse pairs, RK4.

    Returns ``(obs[B][rows][10], final_states[B][N*3] or None)``.
    """
    st = f64(states)
    B = st.size // (3 * handle.N) if not shared_initial else (len(t1) if t1 is not None else 1)
    if shared_initial and st.size != 3 * handle.N:
        raise ValueError("shared_initial needs one state of N*3 doubles")
    if not shared_initial and st.size != B * 3 * handle.N:
        raise ValueError("states must be [B][N*3]")
    rows = int(nat.lib().cmd_batch_rows(int(n_steps), int(save_interval)))
    obs = np.zeros((B, rows, 10))
    fin = np.zeros((B, 3 * handle.N)) if want_final else None
    keep = {}
    d = nat.BatchDesc()
    d.B = B
    d.states = st.ctypes.data
    d.shared_initial = int(bool(shared_initial))
    d.method = nat.CMD_RK4
    drive = d1 is not None or d2 is not None
    if drive:
        for name, arr, n in (("t1", t1, B), ("t2", t2, B), ("a1", a1, B), ("a2", a2, B),
                             ("d1", d1 if d1 is not None else np.zeros(3 * handle.n_atoms), 3 * handle.n_atoms),
                             ("d2", d2 if d2 is not None else np.zeros(3 * handle.n_atoms), 3 * handle.n_atoms)):
            keep[name] = f64(arr, n)
            setattr(d, name, keep[name].ctypes.data)
    d.width = float(width)
    d.freq = float(freq)
    d.T0 = float(T0)
    d.dt = float(dt)
    d.n_steps = int(n_steps)
    d.save_interval = int(save_interval)
    d.obs = obs.ctypes.data
    d.final_states = fin.ctypes.data if fin is not None else None
    check(nat.lib().cmd_run_batch(handle.ptr, C.byref(d)), "cmd_run_batch")
    return obs, fin


def run_uneven(specs, method="rk45", abs_tol=1e-10, rel_tol=1e-10, max_steps=0):
    """Uneven batch (cmd_run_uneven): one persistent launch over trajectories on
    different lattices.  ``specs``: list of dicts with keys handle, state, T0, T1,
    dt and optional t1, t2, a1, a2, max_rows, want_final.  Returns a list of
    (rows[n][11] = {t, M_af, M_local, M_global, E/N}, final_state or None, stats)."""
    B = len(specs)
    arr = (nat.TrajSpec * B)()
    keep = []
    mrs = [int(sp.get("max_rows", (max_steps + 2) if max_steps else int((sp["T1"] - sp["T0"]) / sp["dt"]) + 2))
           for sp in specs]
    # one block for every trajectory's rows (views per trajectory): a large allocation is backed by huge pages,
    # so filling it costs far fewer page faults than many small arrays
    block = np.empty((sum(mrs), 11))
    offs = np.concatenate(([0], np.cumsum(mrs)))
    for b, sp in enumerate(specs):
        h = sp["handle"]
        st = f64(sp["state"], 3 * h.N)
        mr = mrs[b]
        rows = block[offs[b]:offs[b] + mr]
        fin = np.zeros(3 * h.N) if sp.get("want_final", True) else None
        keep.append((st, rows, fin))
        a = arr[b]
        a.lattice = h.ptr.value
        a.state = st.ctypes.data
        a.T0, a.T1, a.dt = float(sp["T0"]), float(sp["T1"]), float(sp["dt"])
        a.t1, a.t2 = float(sp.get("t1", 0.0)), float(sp.get("t2", 0.0))
        a.a1, a.a2 = float(sp.get("a1", 0.0)), float(sp.get("a2", 0.0))
        a.rows = rows.ctypes.data
        a.max_rows = mr
        a.final_state = fin.ctypes.data if fin is not None else None
    check(nat.lib().cmd_run_uneven(C.cast(arr, C.c_void_p), B, _method(method), float(abs_tol), float(rel_tol),
                                   int(max_steps)), "cmd_run_uneven")
    out = []
    for b in range(B):
        st, rows, fin = keep[b]
        stats = tuple(int(x) for x in arr[b].stats)
        out.append((rows[:stats[0]], fin, stats))
    return out
