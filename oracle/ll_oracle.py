"""ctypes binding of the CPU oracle (oracle/libll_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the B200 path.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module;
the product package never does.  See ll_oracle.h for what each function
restates from the reference and how the restatement is pinned.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libll_oracle.so"
REF_DIR = HERE / "_ref"

MAX_ATOMS = 32
MAX_BONDS = 512


class Bond(C.Structure):
    _fields_ = [("src", C.c_int), ("dst", C.c_int), ("off", C.c_int * 3), ("J", C.c_double * 9)]


class UnitCell(C.Structure):
    _fields_ = [("n_atoms", C.c_int),
                ("pos", C.c_double * (MAX_ATOMS * 3)),
                ("lattice_vectors", C.c_double * 9),
                ("field", C.c_double * (MAX_ATOMS * 3)),
                ("onsite", C.c_double * (MAX_ATOMS * 9)),
                ("frames", C.c_double * (MAX_ATOMS * 9)),
                ("afm", C.c_double * MAX_ATOMS),
                ("n_bonds", C.c_int),
                ("bonds", Bond * MAX_BONDS)]


_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_L = C.POINTER(C.c_long)


def build(force: bool = False) -> Path:
    src = [HERE / "ll_oracle.cpp", HERE / "ll_oracle.h"]
    if force or not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in src):
        subprocess.run(["make", "-C", str(HERE), "libll_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "ora_uc_kitaev": (None, [_D, C.c_double, _D, _D, C.POINTER(UnitCell)]),
        "ora_uc_pyrochlore_nk": (None, [_D, C.c_double, _D, C.POINTER(UnitCell)]),
        "ora_uc_pyrochlore_nk_cubic": (None, [_D, C.c_double, _D, C.POINTER(UnitCell)]),
        "ora_lattice_create": (C.c_void_p, [C.POINTER(UnitCell), C.c_int, C.c_int, C.c_int]),
        "ora_lattice_destroy": (None, [C.c_void_p]),
        "ora_lattice_size": (C.c_size_t, [C.c_void_p]),
        "ora_lattice_nnz": (C.c_size_t, [C.c_void_p]),
        "ora_lattice_max_bilinear": (C.c_int, [C.c_void_p]),
        "ora_lattice_csr": (None, [C.c_void_p, _I64, _I64, _D]),
        "ora_lattice_ell": (None, [C.c_void_p, _D, _D, _D, _I64, _I64]),
        "ora_lattice_frames": (None, [C.c_void_p, _D, _D]),
        "ora_set_pulse": (None, [C.c_void_p, _D, C.c_double, _D, C.c_double, C.c_double, C.c_double, C.c_double]),
        "ora_clear_pulse": (None, [C.c_void_p]),
        "ora_set_gilbert": (None, [C.c_void_p, C.c_double]),
        "ora_set_threads": (None, [C.c_int]),
        "ora_rhs": (None, [C.c_void_p, _D, C.c_double, _D]),
        "ora_local_field": (None, [C.c_void_p, _D, _D]),
        "ora_energy": (C.c_double, [C.c_void_p, _D]),
        "ora_magnetizations": (None, [C.c_void_p, _D, _D]),
        "ora_max_dsdt_no_drive": (C.c_double, [C.c_void_p, _D]),
        "ora_rk4_step": (None, [C.c_void_p, _D, C.c_double, C.c_double]),
        "ora_rk4_step_gpu_form": (None, [C.c_void_p, _D, C.c_double, C.c_double]),
        "ora_md_rk4_const": (C.c_long, [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_long, _D, C.c_long]),
        "ora_md_rk4_gpu_loop": (C.c_long, [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_long, _D, C.c_long]),
        "ora_md_dopri5_adaptive": (C.c_long, [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.c_long, _D, C.c_long, _L]),
        "ora_md_dopri5_const": (C.c_long, [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_double,
                                           C.c_double, _D, C.c_long, _L]),
        "ora_pulse_segments": (C.c_int, [C.c_double, C.c_double, _D, C.c_int, C.c_double, C.c_double,
                                         C.c_double, _D, C.c_int]),
        "ora_pulse_drive": (C.c_long, [C.c_void_p, _D, _D, C.c_double, _D, C.c_double, C.c_int, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_int, C.c_double, C.c_double, _D, C.c_long]),
        "ora_loss": (C.c_double, [C.c_void_p, _D, C.c_double, C.c_double, C.c_long, _D]),
        "ora_loss_grad_tlm": (C.c_double, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, _D, C.c_double, C.c_double,
                                           C.c_long, _D, _D]),
        "ora_batch_rk4": (None, [C.c_void_p, _D, C.c_int, _D, _D, _D, _D, C.c_double, C.c_double, C.c_double,
                                 _D, _D, C.c_double, C.c_double, C.c_long, _D, C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _pi(a: np.ndarray):
    return a.ctypes.data_as(_I64)


def _arr(x, n=None) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    if n is not None:
        assert a.size == n, (a.size, n)
    return a


KITAEV_DEFAULT = dict(K=-1.0, Gamma=0.25, Gammap=-0.02, J=0.0, J2_A=0.0, J2_B=0.0, J3=0.0, J_perp=0.0,
                      Ka=0.0, Kb=0.0, Kc=0.0)
PYRO_DEFAULT = dict(Jpm=0.0, Jzz=1.0, Jpmpm=0.0, J2=0.0, delta1=0.0, delta2=0.0)


def kitaev_params(**kw) -> np.ndarray:
    p = dict(KITAEV_DEFAULT)
    p.update(kw)
    return np.array([p[k] for k in ("K", "Gamma", "Gammap", "J", "J2_A", "J2_B", "J3", "J_perp",
                                     "Ka", "Kb", "Kc")], dtype=np.float64)


def pyro_params(**kw) -> np.ndarray:
    p = dict(PYRO_DEFAULT)
    p.update(kw)
    return np.array([p[k] for k in ("Jpm", "Jzz", "Jpmpm", "J2", "delta1", "delta2")], dtype=np.float64)


class OracleLattice:
    """The reference Lattice's MD slice, restated on the CPU."""

    def __init__(self, uc: UnitCell, d1: int, d2: int, d3: int):
        self._L = lib()
        self.uc = uc
        self.h = self._L.ora_lattice_create(C.byref(uc), d1, d2, d3)
        if not self.h:
            raise ValueError("oracle lattice construction failed")
        self.n_atoms = uc.n_atoms
        self.dims = (d1, d2, d3)
        self.N = int(self._L.ora_lattice_size(self.h))

    @classmethod
    def kitaev(cls, d1, d2, d3=1, h=0.0, direction=(0, 1, 0), g=(1, 1, 1), **kw):
        uc = UnitCell()
        lib().ora_uc_kitaev(_p(kitaev_params(**kw)), float(h), _p(_arr(direction, 3)), _p(_arr(g, 3)), C.byref(uc))
        return cls(uc, d1, d2, d3)

    @classmethod
    def pyrochlore_nk(cls, d1, d2, d3, h=0.0, direction=(0, 1, 0), cubic=False, **kw):
        uc = UnitCell()
        f = lib().ora_uc_pyrochlore_nk_cubic if cubic else lib().ora_uc_pyrochlore_nk
        f(_p(pyro_params(**kw)), float(h), _p(_arr(direction, 3)), C.byref(uc))
        return cls(uc, d1, d2, d3)

    def __del__(self):
        if getattr(self, "h", None):
            self._L.ora_lattice_destroy(self.h)
            self.h = None

    # ---- tables -------------------------------------------------------
    def csr(self):
        nnz = int(self._L.ora_lattice_nnz(self.h))
        off = np.zeros(self.N + 1, np.int64)
        part = np.zeros(nnz, np.int64)
        J = np.zeros(nnz * 9)
        self._L.ora_lattice_csr(self.h, _pi(off), _pi(part), _p(J))
        return off, part, J.reshape(nnz, 3, 3)

    def ell(self):
        z = int(self._L.ora_lattice_max_bilinear(self.h))
        N = self.N
        field = np.zeros(N * 3)
        onsite = np.zeros(N * 9)
        bil = np.zeros(N * z * 9)
        part = np.zeros(N * z, np.int64)
        cnt = np.zeros(N, np.int64)
        self._L.ora_lattice_ell(self.h, _p(field), _p(onsite), _p(bil), _pi(part), _pi(cnt))
        return dict(field=field, onsite=onsite, bilinear=bil, partners=part, counts=cnt, max_bilinear=z)

    def frames(self):
        fr = np.zeros(self.n_atoms * 9)
        afm = np.zeros(self.n_atoms)
        self._L.ora_lattice_frames(self.h, _p(fr), _p(afm))
        return fr, afm

    # ---- physics ------------------------------------------------------
    def set_pulse(self, field_in1, t1, field_in2, t2, amp, width, freq):
        self._L.ora_set_pulse(self.h, _p(_arr(field_in1, 3 * self.n_atoms)), float(t1),
                              _p(_arr(field_in2, 3 * self.n_atoms)), float(t2), float(amp), float(width),
                              float(freq))

    def clear_pulse(self):
        self._L.ora_clear_pulse(self.h)

    def rhs(self, state, t=0.0):
        s = _arr(state, 3 * self.N)
        out = np.zeros_like(s)
        self._L.ora_rhs(self.h, _p(s), float(t), _p(out))
        return out

    def local_field(self, state):
        s = _arr(state, 3 * self.N)
        out = np.zeros_like(s)
        self._L.ora_local_field(self.h, _p(s), _p(out))
        return out

    def max_dsdt_no_drive(self, state) -> float:
        return float(self._L.ora_max_dsdt_no_drive(self.h, _p(_arr(state, 3 * self.N))))

    def energy(self, state) -> float:
        return float(self._L.ora_energy(self.h, _p(_arr(state, 3 * self.N))))

    def magnetizations(self, state) -> np.ndarray:
        out = np.zeros(9)
        self._L.ora_magnetizations(self.h, _p(_arr(state, 3 * self.N)), _p(out))
        return out

    def rk4_step(self, state, t, dt, gpu_form=False) -> np.ndarray:
        s = _arr(state, 3 * self.N).copy()
        f = self._L.ora_rk4_step_gpu_form if gpu_form else self._L.ora_rk4_step
        f(self.h, _p(s), float(t), float(dt))
        return s

    def md_rk4(self, state, T0, T1, dt, save_interval=1, gpu_loop=False):
        """Rows {t, M_af, M_loc, M_glob, E/N} and the final state."""
        s = _arr(state, 3 * self.N).copy()
        nmax = int((T1 - T0) / dt / save_interval) + 4
        rows = np.zeros((nmax, 11))
        f = self._L.ora_md_rk4_gpu_loop if gpu_loop else self._L.ora_md_rk4_const
        n = f(self.h, _p(s), float(T0), float(T1), float(dt), int(save_interval), _p(rows), nmax)
        return rows[:n], s

    def md_dopri5(self, state, T0, T1, dt0, abs_tol, rel_tol, max_accepted=0, max_rows=200000, const=False):
        s = _arr(state, 3 * self.N).copy()
        rows = np.zeros((max_rows, 11))
        stats = (C.c_long * 3)()
        if const:
            n = self._L.ora_md_dopri5_const(self.h, _p(s), float(T0), float(T1), float(dt0), float(abs_tol),
                                            float(rel_tol), _p(rows), max_rows, stats)
        else:
            n = self._L.ora_md_dopri5_adaptive(self.h, _p(s), float(T0), float(T1), float(dt0), float(abs_tol),
                                               float(rel_tol), int(max_accepted), _p(rows), max_rows, stats)
        if n < 0:
            raise RuntimeError("step-size control failed (500 rejections)")
        return rows[:n], s, tuple(stats)

    def pulse_drive(self, state, field_in1, t1, field_in2, t2, n_pulses, amp, width, freq, T0, T1, step,
                    method="rk4", chunking=False, abs_tol=1e-8, rel_tol=1e-8):
        nmax = int((T1 - T0) / step) + 8
        rows = np.zeros((nmax, 10))
        z = np.zeros(3 * self.n_atoms)
        n = self._L.ora_pulse_drive(self.h, _p(_arr(state, 3 * self.N)), _p(_arr(field_in1)), float(t1),
                                    _p(_arr(field_in2) if field_in2 is not None else z), float(t2), int(n_pulses),
                                    float(amp), float(width), float(freq), float(T0), float(T1), float(step),
                                    0 if method == "rk4" else 1, int(bool(chunking)), float(abs_tol),
                                    float(rel_tol), _p(rows), nmax)
        if n < 0:
            raise RuntimeError("pulse drive failed")
        return rows[:min(n, nmax)]

    def batch_rk4(self, states, t1, t2, s1, s2, amp, width, freq, dir1, dir2, T0, dt, nsteps,
                  with_obs=True, with_energy=True):
        st = np.ascontiguousarray(states, dtype=np.float64).copy()
        B = st.shape[0]
        obs = np.zeros((B, nsteps + 1, 10)) if with_obs else None
        self._L.ora_batch_rk4(self.h, _p(st), B, _p(_arr(t1, B)), _p(_arr(t2, B)), _p(_arr(s1, B)),
                              _p(_arr(s2, B)), float(amp), float(width), float(freq),
                              _p(_arr(dir1, 3 * self.n_atoms)), _p(_arr(dir2, 3 * self.n_atoms)), float(T0),
                              float(dt), int(nsteps), _p(obs) if obs is not None else None, int(with_energy))
        return st, obs


def loss(L, state0, T0, dt, nsteps, target):
    return float(lib().ora_loss(L.h, _p(_arr(state0, 3 * L.N)), float(T0), float(dt), int(nsteps),
                                _p(_arr(target, 3 * (nsteps + 1)))))


def loss_grad_tlm(L, dparams, state0, T0, dt, nsteps, target):
    """(loss, dL/dtheta) by the tangent-linear model; dparams: OracleLattices built at theta = e_q."""
    nq = len(dparams)
    arr = (C.c_void_p * nq)(*[d.h for d in dparams])
    g = np.zeros(nq)
    val = lib().ora_loss_grad_tlm(L.h, arr, nq, _p(_arr(state0, 3 * L.N)), float(T0), float(dt), int(nsteps),
                                  _p(_arr(target, 3 * (nsteps + 1))), _p(g))
    return float(val), g


def set_threads(n: int):
    lib().ora_set_threads(int(n))


def pulse_segments(T_start, T_end, centers, window, T_step, free_dt_factor=20.0):
    c = _arr(centers)
    segs = np.zeros(3 * 128)
    n = lib().ora_pulse_segments(float(T_start), float(T_end), _p(c), len(c), float(window), float(T_step),
                                 float(free_dt_factor), _p(segs), 128)
    return segs[:3 * n].reshape(n, 3)


# ---- reference code compiled in place (oracle/_ref) -------------------------

def ref_available(name: str) -> bool:
    return (REF_DIR / name).exists()


def ref_pulse_segments(T_start, T_end, centers, window, T_step, free_dt_factor=20.0):
    L = C.CDLL(str(REF_DIR / "libref_chunking.so"))
    L.refchunk_segments.restype = C.c_int
    L.refchunk_segments.argtypes = [C.c_double, C.c_double, _D, C.c_int, C.c_double, C.c_double, C.c_double,
                                    _D, C.c_int]
    c = _arr(centers)
    segs = np.zeros(3 * 128)
    n = L.refchunk_segments(float(T_start), float(T_end), _p(c), len(c), float(window), float(T_step),
                            float(free_dt_factor), _p(segs), 128)
    return segs[:3 * n].reshape(n, 3)


class RefGPU:
    """The reference's own gpu:: integrator (oracle/_ref/libref_gpu.so); needs a GPU."""

    def __init__(self, ell: dict, n_atoms: int):
        L = C.CDLL(str(REF_DIR / "libref_gpu.so"))
        L.refgpu_create.restype = C.c_void_p
        L.refgpu_create.argtypes = [C.c_int64, C.c_int64, C.c_int64, _D, _D, _D, _I64, _I64]
        L.refgpu_destroy.argtypes = [C.c_void_p]
        L.refgpu_set_pulse.argtypes = [C.c_void_p, _D, C.c_int64, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double]
        L.refgpu_set_spins.argtypes = [C.c_void_p, _D, C.c_int64]
        L.refgpu_get_spins.argtypes = [C.c_void_p, _D, C.c_int64]
        L.refgpu_integrate.restype = C.c_int64
        L.refgpu_integrate.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_char_p,
                                       _D, _D, C.c_int64, C.c_int64]
        L.refgpu_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_char_p]
        L.refgpu_batched.restype = C.c_int64
        L.refgpu_batched.argtypes = [C.c_void_p, _D, C.c_int64, _D, C.c_int64, _D, _D, C.c_int64, C.c_double,
                                     C.c_double, C.c_double, C.c_int64, _D, _D, C.c_int64]
        self._L = L
        self.n_atoms = n_atoms
        self.N = ell["counts"].size
        self._keep = ell
        self.h = L.refgpu_create(self.N, n_atoms, ell["max_bilinear"], _p(ell["field"]), _p(ell["onsite"]),
                                 _p(ell["bilinear"]), _pi(ell["partners"]), _pi(ell["counts"]))
        if not self.h:
            raise RuntimeError("reference create_gpu_lattice_data failed")

    def close(self):
        if self.h:
            self._L.refgpu_destroy(self.h)
            self.h = None

    def set_pulse(self, field_drive, amp, width, freq, t1, t2):
        fd = _arr(field_drive)
        assert self._L.refgpu_set_pulse(self.h, _p(fd), fd.size, amp, width, freq, t1, t2) == 0

    def set_spins(self, s):
        s = _arr(s, 3 * self.N)
        assert self._L.refgpu_set_spins(self.h, _p(s), s.size) == 0

    def get_spins(self):
        s = np.zeros(3 * self.N)
        assert self._L.refgpu_get_spins(self.h, _p(s), s.size) == 0
        return s

    def integrate(self, T0, T1, dt, save_interval=1, method="rk4", max_rows=None):
        n_est = int((T1 - T0) / dt) // save_interval + 4 if max_rows is None else max_rows
        times = np.zeros(n_est)
        states = np.zeros((n_est, 3 * self.N))
        n = self._L.refgpu_integrate(self.h, T0, T1, dt, save_interval, method.encode(), _p(times), _p(states),
                                     3 * self.N, n_est)
        assert 0 <= n <= n_est, n
        return times[:n], states[:n]

    def step(self, t, dt, method="rk4"):
        assert self._L.refgpu_step(self.h, t, dt, method.encode()) == 0

    def batched(self, init, tau2, afm, frames, T0, T1, dt, save_interval=1):
        tau2 = _arr(tau2)
        B = tau2.size
        n_est = int((T1 - T0) / dt) // save_interval + 4
        times = np.zeros(n_est)
        mags = np.zeros((n_est, B, 9))
        n = self._L.refgpu_batched(self.h, _p(_arr(init, 3 * self.N)), 3 * self.N, _p(tau2), B,
                                   _p(_arr(afm, self.n_atoms)), _p(_arr(frames, 9 * self.n_atoms)),
                                   self.n_atoms, T0, T1, dt, save_interval, _p(times), _p(mags), n_est)
        assert 0 <= n <= n_est, n
        return times[:n], mags[:n]
