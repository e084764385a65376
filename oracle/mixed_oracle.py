"""Test oracle: numpy restatement of the reference's mixed SU(2)/SU(3) GPU dynamics.

Test infrastructure only (imported by tests/).  Follows src/gpu/mixed_lattice_gpu.cu
of the reference: local fields of SU(2) sites (:54-121) and SU(3) sites (:127-187),
the two-pulse drive of each kind (gpu_common_helpers.cuh:355-377), and the equations
of motion dS/dt = H x S (SU(2)) and (dS/dt)_a = f_abc H_b S_c (SU(3),
gpu_common_helpers.cuh:386-399), integrated with oracle/fixed_methods.py.  The
structure constants are derived here from the Gell-Mann matrices,
f_abc = Tr([l_a, l_b] l_c) / (4i), not copied from a table.

``RefMixedGPU`` wraps the reference's own mixed GPU code (oracle/_ref/libref_mixed.so,
built from its sources by oracle/Makefile); it needs a GPU.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / "_ref"


def gell_mann() -> np.ndarray:
    """The eight Gell-Mann matrices, [8][3][3] complex."""
    l = np.zeros((8, 3, 3), complex)
    l[0][0, 1] = l[0][1, 0] = 1
    l[1][0, 1], l[1][1, 0] = -1j, 1j
    l[2][0, 0], l[2][1, 1] = 1, -1
    l[3][0, 2] = l[3][2, 0] = 1
    l[4][0, 2], l[4][2, 0] = -1j, 1j
    l[5][1, 2] = l[5][2, 1] = 1
    l[6][1, 2], l[6][2, 1] = -1j, 1j
    l[7] = np.diag([1, 1, -2]) / np.sqrt(3)
    return l


def structure_constants() -> np.ndarray:
    """f_abc from [l_a, l_b] = 2i f_abc l_c."""
    l = gell_mann()
    f = np.zeros((8, 8, 8))
    for a in range(8):
        for b in range(8):
            com = l[a] @ l[b] - l[b] @ l[a]
            for c in range(8):
                f[a, b, c] = (np.trace(com @ l[c]) / 4j).real
    return f


F_SU3 = structure_constants()


def drive_factor(amp, x, width, freq):
    """gpu_common_helpers.cuh:363-372."""
    u = x / (2.0 * width)
    return amp * np.exp(-(u * u)) * np.cos(freq * x)


class MixedOracle:
    """The mixed lattice of a ``synthetic_mixed_lattice`` dictionary (the reference's flattened arrays)."""

    def __init__(self, arr: dict):
        self.a = arr
        self.n2, self.n3 = arr["n2"], arr["n3"]
        self.pulse = {2: None, 3: None}

    def set_pulse(self, sub, field_drive, amp, width, freq, t1, t2):
        self.pulse[sub] = (np.asarray(field_drive, float).reshape(2, -1, 3 if sub == 2 else 8), amp, width, freq,
                           t1, t2)

    def _ell(self, key_part, key_cnt, key_val, n, z, shape):
        a = self.a
        part = np.asarray(a[key_part]).reshape(n, z)
        cnt = np.asarray(a[key_cnt]).reshape(n)
        val = np.asarray(a[key_val]).reshape((n, z) + shape)
        return part, cnt, val

    def fields(self, Y, t):
        """(H2 [n2][3], H3 [n3][8]) at state Y and time t."""
        a = self.a
        n2, n3 = self.n2, self.n3
        S2 = Y[:3 * n2].reshape(n2, 3)
        S3 = Y[3 * n2:].reshape(n3, 8)
        H2 = -np.asarray(a["field2"]).reshape(n2, 3) + 2.0 * np.einsum(
            "nij,nj->ni", np.asarray(a["onsite2"]).reshape(n2, 3, 3), S2)
        H3 = -np.asarray(a["field3"]).reshape(n3, 8) + 2.0 * np.einsum(
            "nij,nj->ni", np.asarray(a["onsite3"]).reshape(n3, 8, 8), S3)
        for (H, n, S_other, kp, kc, kv, z, shape, limit) in (
                (H2, n2, S2, "part2", "cnt2", "bil2", a["z2"], (3, 3), n2),
                (H3, n3, S3, "part3", "cnt3", "bil3", a["z3"], (8, 8), n3),
                (H2, n2, S3, "mpart2", "mcnt2", "mix2", a["zm2"], (3, 8), n3),
                (H3, n3, S2, "mpart3", "mcnt3", "mix3", a["zm3"], (8, 3), n2)):
            if n == 0 or z == 0:
                continue
            part, cnt, val = self._ell(kp, kc, kv, n, z, shape)
            for k in range(z):
                ok = (k < cnt) & (part[:, k] >= 0) & (part[:, k] < limit)
                if ok.any():
                    H[ok] += np.einsum("mij,mj->mi", val[ok, k], S_other[part[ok, k]])
        for sub, H, n, na in ((2, H2, n2, a["na2"]), (3, H3, n3, a["na3"])):
            p = self.pulse[sub]
            if p is None or p[1] == 0.0 or n == 0:
                continue
            fd, amp, width, freq, t1, t2 = p
            f1, f2 = drive_factor(amp, t - t1, width, freq), drive_factor(amp, t - t2, width, freq)
            atom = np.arange(n) % na
            H -= f1 * fd[0][atom] + f2 * fd[1][atom]
        return H2, H3

    def rhs(self, Y, t=0.0):
        n2, n3 = self.n2, self.n3
        H2, H3 = self.fields(Y, t)
        S2 = Y[:3 * n2].reshape(n2, 3)
        S3 = Y[3 * n2:].reshape(n3, 8)
        return np.concatenate([np.cross(H2, S2).ravel(), np.einsum("abc,nb,nc->na", F_SU3, H3, S3).ravel()])

    def energy(self, Y):
        """Static energy (no drive): the local fields are its gradient, each bond counted once."""
        a = self.a
        n2, n3 = self.n2, self.n3
        S2 = Y[:3 * n2].reshape(n2, 3)
        S3 = Y[3 * n2:].reshape(n3, 8)
        E = -np.sum(np.asarray(a["field2"]).reshape(n2, 3) * S2) - np.sum(np.asarray(a["field3"]).reshape(n3, 8) * S3)
        E += np.einsum("ni,nij,nj->", S2, np.asarray(a["onsite2"]).reshape(n2, 3, 3), S2)
        E += np.einsum("ni,nij,nj->", S3, np.asarray(a["onsite3"]).reshape(n3, 8, 8), S3)
        for (n, S, S_o, kp, kc, kv, z, shape, w) in (
                (n2, S2, S2, "part2", "cnt2", "bil2", a["z2"], (3, 3), 0.5),
                (n3, S3, S3, "part3", "cnt3", "bil3", a["z3"], (8, 8), 0.5),
                (n2, S2, S3, "mpart2", "mcnt2", "mix2", a["zm2"], (3, 8), 1.0)):
            if n == 0 or z == 0:
                continue
            part, cnt, val = self._ell(kp, kc, kv, n, z, shape)
            for k in range(z):
                ok = k < cnt
                E += w * np.einsum("mi,mij,mj->", S[ok], val[ok, k], S_o[part[ok, k]])
        return float(E)

    def magnetizations(self, Y):
        """(m2, ms2, m3, ms3): means and staggered means, sign (-1)^(site mod atoms) (gpu_common_helpers.cu:163-211)."""
        a = self.a
        out = []
        for S, na in ((Y[:3 * self.n2].reshape(self.n2, 3), a["na2"]), (Y[3 * self.n2:].reshape(self.n3, 8), a["na3"])):
            sign = np.where((np.arange(len(S)) % na) % 2 == 0, 1.0, -1.0)
            out += [S.mean(0), (S * sign[:, None]).mean(0)]
        return tuple(out)


class RefMixedGPU:
    """The reference's own mixed_gpu:: integrator (oracle/_ref/libref_mixed.so); needs a GPU."""

    def __init__(self, arr: dict):
        L = C.CDLL(str(REF_DIR / "libref_mixed.so"))
        P = C.c_void_p
        L.refmix_create.restype = P
        L.refmix_create.argtypes = [P] * 17
        L.refmix_destroy.argtypes = [P]
        L.refmix_set_pulse.argtypes = [P, C.c_int, P, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double]
        L.refmix_set_spins.argtypes = [P, P, C.c_int64]
        L.refmix_get_spins.argtypes = [P, P, C.c_int64]
        L.refmix_step.argtypes = [P, C.c_double, C.c_double, C.c_char_p]
        L.refmix_integrate.restype = C.c_int64
        L.refmix_integrate.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_char_p, P, P, C.c_int64,
                                       C.c_int64]
        L.refmix_magnetization.argtypes = [P] * 5
        L.refmix_normalize.argtypes = [P, C.c_double, C.c_double]
        self._L = L
        self.V = 3 * arr["n2"] + 8 * arr["n3"]
        f = lambda k: np.ascontiguousarray(arr[k], dtype=np.float64)
        i = lambda k: np.ascontiguousarray(arr[k], dtype=np.int64)
        self._keep = [np.array([arr["n2"], arr["na2"], arr["n3"], arr["na3"], arr["z2"], arr["z3"], arr["zm2"],
                                arr["zm3"]], np.int64),
                      f("field2"), f("onsite2"), f("bil2"), i("part2"), i("cnt2"),
                      f("field3"), f("onsite3"), f("bil3"), i("part3"), i("cnt3"),
                      f("mix2"), i("mpart2"), i("mcnt2"), f("mix3"), i("mpart3"), i("mcnt3")]
        self.h = L.refmix_create(*[k.ctypes.data for k in self._keep])
        if not self.h:
            raise RuntimeError("reference create_gpu_mixed_lattice_data failed")

    def close(self):
        if self.h:
            self._L.refmix_destroy(self.h)
            self.h = None

    def set_pulse(self, sub, field_drive, amp, width, freq, t1, t2):
        fd = np.ascontiguousarray(field_drive, dtype=np.float64).ravel()
        assert self._L.refmix_set_pulse(self.h, sub, fd.ctypes.data, fd.size, amp, width, freq, t1, t2) == 0

    def set_spins(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        assert self._L.refmix_set_spins(self.h, s.ctypes.data, s.size) == 0

    def get_spins(self):
        s = np.zeros(self.V)
        assert self._L.refmix_get_spins(self.h, s.ctypes.data, s.size) == 0
        return s

    def step(self, t, dt, method="ssprk53"):
        assert self._L.refmix_step(self.h, t, dt, method.encode()) == 0

    def integrate(self, T0, T1, dt, save_interval=1, method="ssprk53"):
        n_est = int((T1 - T0) / dt) // save_interval + 4
        times = np.zeros(n_est)
        states = np.zeros((n_est, self.V))
        n = self._L.refmix_integrate(self.h, T0, T1, dt, save_interval, method.encode(), times.ctypes.data,
                                     states.ctypes.data, self.V, n_est)
        assert 0 <= n <= n_est, n
        return times[:n], states[:n]

    def magnetization(self):
        out = [np.zeros(3), np.zeros(3), np.zeros(8), np.zeros(8)]
        assert self._L.refmix_magnetization(self.h, *(o.ctypes.data for o in out)) == 0
        return tuple(out)

    def normalize(self, l2, l3):
        assert self._L.refmix_normalize(self.h, l2, l3) == 0
